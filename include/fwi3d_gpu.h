/*
 * fwi3d_gpu.h -- C ABI of the B200 wave-propagation engine (libfwi3d_b200.so).
 *
 * Drop-in for the time-stepping hot path of nmbader/fwi3d: the acoustic
 * variable-density, elastic isotropic and elastic VTI propagators and their
 * adjoint-state gradients.  Entry points replace, one for one, the reference
 * operator calls a caller makes:
 *
 *   fwi_op_create     <- nl_we_op_{a,e,vti}(domain, allsrc, s, par)
 *                        src/include/we_op.hpp:59-79 (elastic), :106 (VTI), :139-151 (acoustic)
 *   fwi_op_forward    <- nl_we_op_e::apply_forward(add, pmod, pdat)
 *                        we_op.hpp:50, src/cpp/we_op.cpp:872-946
 *   fwi_op_jacobianT  <- nl_we_op_e::apply_jacobianT(add, pmod, pmod0, pdat)
 *                        we_op.hpp:51, src/cpp/we_op.cpp:948-1078
 *   fwi_op_destroy    <- delete op   (src/main/we_modeling.cpp:98, src/cpp/optimization.cpp:183)
 *   fwi_forward_batch <- the rank-strided shot loop of WE_MODELING_3D
 *                        (src/main/we_modeling.cpp:72-109) for shots sharing one model
 *
 * Errors: the reference aborts through successCheck -> exit(123)
 * (src/include/misc.hpp:4-12).  Here every call returns FWI_OK (0) or a negative
 * status and leaves a message for fwi_last_error().
 *
 * Conventions (the reference's): units km, km/s, g/cc, s; model layout
 * [nmodels][ny][nx][nz] (z fastest) holding vp,rho (nmodels=2), vp,vs,rho (3) or
 * vp,vs,rho,delta,epsilon,gamma (6); data layout [nrcomp][nr][nt_data]; wavelet
 * [ncomp][nt_data] or a single trace duplicated as analyzeWavelet does
 * (we_op.cpp:138-232).  Host buffers are owned by the caller; the operator owns
 * its device model, wavefields, snapshots and traces.
 */
#ifndef FWI3D_GPU_H
#define FWI3D_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FWI_OK 0
#define FWI_ERR_ARG (-1)         /* bad shape / argument (reference: successCheck) */
#define FWI_ERR_OOM (-2)         /* device memory exhausted */
#define FWI_ERR_CUDA (-3)        /* CUDA runtime or launch failure */
#define FWI_ERR_NAN (-4)         /* non-finite value in model or wavefield */
#define FWI_ERR_STATE (-5)       /* adjoint requested without stored forward state */
#define FWI_ERR_UNSUPPORTED (-6) /* option the GPU path does not implement */
#define FWI_ERR_NOGPU (-7)       /* no CUDA device */

/* Computational grid: model axes Z (fast), X, Y (src/cpp/we_op.cpp:28-30). */
typedef struct fwi_grid {
    int nx, ny, nz;
    float ox, oy, oz;
    float dx, dy, dz;
} fwi_grid;

/* Propagation knobs; field meaning and defaults as in `struct param`
 * (src/include/param.hpp:8-71).  fwi_param_default() fills the defaults. */
typedef struct fwi_param {
    float courant, dt;        /* dt <= 0: CFL-derived (analyzeModel, we_op.cpp:405-425) */
    int sub;                  /* snapshot/imaging sub-sampling; <0: derived; 0: none */
    int resampling_linear;    /* 0 sinc (default), 1 linear */
    int sinc_half_length;
    int mt;                   /* moment-tensor source (6 components) */
    float fangle, fazimuth;   /* vector-force direction */
    float mxx, myy, mzz, mxy, mxz, myz;
    int seismotype;           /* 0 displacement/pressure, 1 velocity (time derivative) */
    float gl;                 /* DAS gauge length; > 0 unsupported on the GPU path */
    int bc[6];                /* top, bottom, left, right, front, back: 0 none, 1 free, 2 absorbing, 3 rigid */
    int taper[6];
    float free_surface_stiffness, taper_strength;
    float vpmin, vpmax, vsmin, vsmax, rhomin, rhomax;
    float deltamin, deltamax, epsilonmin, epsilonmax, gammamin, gammamax;
    int soft_clip;
    int verbose;
    int snapshot_storage;     /* gradient snapshots: 0 FP32 (as the reference), 1 FP16 second-difference
                                 residuals with per-snapshot scales (half the memory); no reference counterpart */
    float snapshot_budget_gb; /* HBM budget of the gradient's forward-wavefield storage (0: unlimited); above it
                                 binomial checkpointing with as many slots as fit replaces full storage */
    int checkpoint_slots;     /* > 0: binomial checkpointing (Griewank-Walther revolve schedule) with this many
                                 restart states (prev, curr) on the device, whatever the budget; no reference
                                 counterpart (the reference keeps every snapshot, zfpWrapper.hpp:24-116) */
    int checkpoint_precision; /* checkpoint storage: 0 FP32, 1 BF16, 2 FP16, the 16-bit forms scaled per
                                 (state, level, shot, component) by the field's max |value| */
} fwi_param;

void fwi_param_default(fwi_param *p);

typedef struct fwi_op fwi_op;

typedef struct fwi_op_info {
    float dt;       /* propagation time step */
    int nt;         /* propagation samples */
    int sub;        /* snapshot interval */
    int nscomp;     /* source components (1, 3 or 6) */
    int nrcomp;     /* receiver components (1 or 3) */
    int nr;         /* receivers */
    int64_t device_bytes;
} fwi_op_info;

/* One shot on one device.  `rxyz` is [nr][5] (x, y, z, dip, azimuth), as the
 * reference's par.rxyz[s]; `sxyz` is [3]. */
int fwi_op_create(fwi_op **op, int device, const fwi_grid *grid, int nmodels, const fwi_param *par,
                  const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data, const float *sxyz, int nr,
                  const float *rxyz);

/* data (+)= F(model); keeps the forward snapshots for a following jacobianT when sub > 0. */
int fwi_op_forward(fwi_op *op, int add, const float *model, float *data);

/* grad (+)= J^T data at model0 (needs the preceding forward of the same op with sub > 0). */
int fwi_op_jacobianT(fwi_op *op, int add, float *grad, const float *model0, const float *data);

int fwi_op_get_info(const fwi_op *op, fwi_op_info *info);
void fwi_op_destroy(fwi_op *op);

/* Modeling of nshots shots that share one model, batched on the device.
 * sxyz: [nshots][3]; nr: receivers per shot (same for all shots);
 * rxyz: [nshots][nr][5]; data: [nshots][nrcomp][nr][nt_data]. */
int fwi_forward_batch(int device, const fwi_grid *grid, int nmodels, const fwi_param *par, const float *model,
                      const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data, int nshots,
                      const float *sxyz, int nr, const float *rxyz, float *data);

/* Batched modeling session: nshots shots sharing one device-resident model
 * advance in lockstep, one kernel launch per operator per time step for the
 * whole batch.  fwi_forward_batch is create + reset + run(all) + traces.
 * Calls on one session must come from one host thread at a time. */
typedef struct fwi_batch fwi_batch;

int fwi_batch_create(fwi_batch **b, int device, const fwi_grid *grid, int nmodels, const fwi_param *par,
                     const float *model, const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data,
                     int nshots, const float *sxyz, int nr, const float *rxyz);
/* Zero the wavefields and apply the initial condition (time index 0). */
int fwi_batch_reset(fwi_batch *b);
/* Enqueue nsteps time steps on the session's stream (asynchronous). */
int fwi_batch_run(fwi_batch *b, int nsteps);
int fwi_batch_sync(fwi_batch *b);
/* *ready = 1 when the session's enqueued work has finished (then as
 * fwi_batch_sync, without waiting), else 0: a dispatcher polls its sessions
 * and gives each its next steps as soon as it is idle.  Serving; no
 * counterpart in the reference. */
int fwi_batch_ready(fwi_batch *b, int *ready);
/* The cudaStream_t the session launches on (for event timing). */
int fwi_batch_stream(fwi_batch *b, void **stream);
/* Data [nshots][nrcomp][nr][nt_data] after the full time axis was run. */
int fwi_batch_traces(fwi_batch *b, float *data);
/* Shot slots (serving; no counterpart in the reference, whose modeling runs
 * one survey at a time).  fwi_batch_enable_slots, right after a reset, turns
 * the session's shots into slots with their own start steps (all 0 then).
 * fwi_batch_join restarts `slot` with a new shot (sxyz [3], rxyz [nr][5]) at
 * the session's current step while the other slots run on; a run is then no
 * longer bounded by nt, every slot's sources and receivers follow its own
 * time axis, and its data come from fwi_batch_slot_traces once
 * fwi_batch_slot_time reports 0 steps remaining (fwi_batch_traces refuses).
 * fwi_batch_release makes a slot idle: no kernel advances it until the next
 * join (a session opened with spare slots releases them; a slot whose data
 * were read is released).  A shot whose source lies in a taper zone cannot
 * join (FWI_ERR_UNSUPPORTED): its first step would taper its initial state,
 * which a shot started at time 0 does not see; it needs a session of its own. */
int fwi_batch_enable_slots(fwi_batch *b);
int fwi_batch_join(fwi_batch *b, int slot, const float *sxyz, const float *rxyz);
int fwi_batch_release(fwi_batch *b, int slot);
int fwi_batch_slot_time(const fwi_batch *b, int slot, int *t0, int *remaining);
int fwi_batch_slot_traces(fwi_batch *b, int slot, float *data);
int fwi_batch_get_info(const fwi_batch *b, fwi_op_info *info, int *launches_per_step);
/* Diagnostics (no counterpart in the reference): time each launch of the
 * step's main kernel with a pair of CUDA events on the session stream, for up
 * to max_launches launches (0: off); read back the summed time, the number of
 * launches timed, the grid-point updates one launch performs and the kernel
 * name.  The read-back synchronises the session stream. */
int fwi_batch_time_main_kernel(fwi_batch *b, int max_launches);
int fwi_batch_main_kernel_time(fwi_batch *b, double *ms, int *launches, int64_t *points, const char **name);
void fwi_batch_destroy(fwi_batch *b);

/* One elastic (nmodels 3) or VTI (nmodels 6) leapfrog step on caller-owned
 * device buffers that allocates nothing, device or host.  No counterpart in
 * the reference: there the step lives inside nl_we_op_*::propagate
 * (src/cpp/we_op.cpp:623-836) on arrays the operator allocates itself.  For
 * callers whose device memory is owned by another allocator (a PyTorch
 * caching allocator, a serving loop that has budgeted all HBM to admitted
 * requests): the library's own paths cudaMalloc and cudaFree, and cudaFree
 * synchronises the whole device.
 *   model: converted [nmodels][ny][nx][nz] (lambda, mu, rho[, c13, eps, c66]);
 *   prev, curr (read), next (written at every point): [3][ny][nx][nz];
 *   all on the current device; stream: a cudaStream_t (0: legacy default).
 *   next may be prev itself (the leapfrog in place: prev is read only at the
 *   point written) but must not overlap curr, the model, or prev in part
 *   (FWI_ERR_ARG).
 * Limits: at most 262,144 grid points (the static scratch is 9 x 2^18 floats,
 * 9 MiB, reserved with the library's device code when that loads), each axis >= 12, bc[6] each 0 (none) or 1 (traction-free), no taper
 * (FWI_ERR_ARG / FWI_ERR_UNSUPPORTED otherwise).  Nothing needs to start at
 * zero.  The first call on a device does a one-time synchronous set-up
 * (scratch address, coefficient tables): make it before any stream capture.
 * All calls on a device share the one scratch array, so calls that overlap
 * in time (other streams, other threads) race: serialise them. */
int fwi_elastic_step_static(const fwi_grid *grid, int nmodels, const int *bc, float dt, const float *model,
                            const float *prev, const float *curr, float *next, void *stream);

/* Full-waveform-inversion objective of a shot gather on the device: the
 * nlls_fwi objective of the reference (src/cpp/optimization.cpp:5-197,
 * src/include/optimization.hpp:403-430) without data weights, filters,
 * envelopes or source scaling.  Shots are processed `batch` at a time in
 * lockstep; per evaluation
 *   f    = 0.5 dt_data (sum r^2 - 0.5 sum_traces (r_0^2 + r_{nt-1}^2)) / dnorm,
 *   grad = J^T Ht(r) summed over shots / dnorm, in (vp, vs, rho) like jacobianT,
 * with r = synthetic - observed, dnorm = dt_data |observed|^2 when `normalize`
 * (else 1).  Misfit and gradient sums are FP64 (the reference sums in data_t);
 * the gradient is the sum of the per-shot gradients (the reference's
 * apply_jacobianT(add=true) chaining, we_op.cpp:968-972 and 1069-1075, also
 * passes the earlier shots' sum through H and the chain rule again; the
 * per-shot operator path above reproduces that when a caller needs it).
 * observed: [nshots][nrcomp][nr][nt_data]; residual (optional, may be null):
 * same layout; grad: [min(3,nmodels)][ny][nx][nz]. */
typedef struct fwi_objective fwi_objective;
int fwi_objective_create(fwi_objective **o, int device, const fwi_grid *grid, int nmodels, const fwi_param *par,
                         const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data, int nshots,
                         const float *sxyz, int nr, const float *rxyz, const float *observed, int normalize,
                         int batch);
int fwi_objective_evaluate(fwi_objective *o, const float *model, double *f, float *grad, float *residual);
/* Serving (no counterpart in the reference).  fwi_objective_evaluate_shots:
 * one objective per shot -- f [nshots], grad [nshots][min(3,nmodels)][nxyz],
 * each normalised by its own shot's data -- from the same batched launches
 * (independent gradient requests on one model in one evaluation).
 * fwi_objective_set_shots: new shots for the same counts (sxyz [nshots][3],
 * rxyz [nshots][nr][5], observed data); the evaluations after it reuse the
 * objective's device buffers (wavefields, snapshot or checkpoint stores,
 * residual state), so a server allocates no device memory per request. */
int fwi_objective_evaluate_shots(fwi_objective *o, const float *model, double *f, float *grad);
int fwi_objective_set_shots(fwi_objective *o, const float *sxyz, const float *rxyz, const float *observed);
/* Device bytes of the last evaluation (wavefields, snapshots, model, tables). */
int64_t fwi_objective_device_bytes(const fwi_objective *o);
void fwi_objective_destroy(fwi_objective *o);

/* Message of the last failing call on this thread. */
const char *fwi_last_error(void);

/* Library version string. */
const char *fwi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FWI3D_GPU_H */
