// Device engine: owns the GPU state of one propagation problem (model, tables,
// wavefields of a batch of shots, snapshots) and runs the time loops on a
// CUDA stream.  All shots of a batch share the model and step in lockstep;
// one kernel launch advances every shot.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_ops.h"

namespace fwi {

struct FwiError : std::runtime_error {
    int code;
    FwiError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Device buffer (RAII).
// Device residual of the FWI objective, one trace per CUDA block: from the
// synthetic traces at the propagation sampling to the misfit partial of each
// trace and the adjoint sources, with the host path's arithmetic (capi.cpp,
// fwi_objective_evaluate): [Dt], *alpha, sinc resampling to the data axis,
// - observed, sum of squares minus the half end samples (FP64), Ht, sinc
// resampling back, Ht^-1, time reversal, *(-alpha), [Dt^T].
struct ResidualArgs {
    const float *rcv;      // [ntraces][nt] synthetic traces
    const float *obs;      // [ntraces][ntd] observed
    float *asrc;           // [ntraces][nt] adjoint sources (out)
    float *resid;          // [ntraces][ntd] residual (out, may be null)
    double *part;          // [ntraces] misfit partials (out)
    int *bad;              // set when a synthetic sample is not finite
    const int *first, *count;  // sinc taps per propagation sample (data -> propagation axis)
    const int *off;            // start of each propagation sample's taps in s / win
    const float *s;
    const double *win;
    const int *jlo, *jhi;      // propagation samples whose taps reach data sample j
    int nt, ntd, seismotype;
    float alpha, dt, dtd;
};
// Largest trace length (either axis) the device residual keeps in shared memory.
constexpr int kResidualMaxSamples = 12000;

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n);
    ~DevBuf();
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept;
    void alloc(size_t n);
    void zero(void *stream = nullptr);
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Static description of a propagation problem.
struct Problem {
    int nmodels;     // 2, 3, 6
    int nx, ny, nz;
    float dx, dy, dz;
    float dt;
    int nt;          // propagation samples (steps + 1)
    int sub;         // snapshot interval (0: none)
    int bc[6];
    int taper[6];
    float taper_strength;
    float free_surface_stiffness;
    int nshots = 1;
    int ncomp() const { return nmodels == 2 ? 1 : 3; }
    int64_t nxyz() const { return (int64_t)nx * ny * nz; }
};

// Injection table on the device: entry k adds w[k]*src[trace[k]][it] to field
// component c at global point gidx[k] = shot*nxyz + point.
struct DevInj {
    int n[3] = {0, 0, 0};
    DevBuf gidx[3], trace[3], w[3];
    int ntrace = 0;
};
// Extraction table: receiver row k (= shot*nr + r) reads 27 weighted points.
struct DevExt {
    int nrec = 0;   // total rows over the batch
    int nr = 0;     // receivers per shot
    int ntap = 27;  // weights per row
    DevBuf gidx, w;
};

class Engine {
public:
    Engine(int device, const Problem &pb);
    ~Engine();

    const Problem &problem() const { return pb_; }
    void *stream() const { return stream_; }

    // Converted model [nmodels][nxyz] (host); boundary divisors and taper tables are built here.
    void set_model(const float *conv_model);

    // --- batched modeling -------------------------------------------------
    // Tables of all shots (gidx already offset by shot), sources [ntrace][nt]
    // at the propagation sampling, receivers per shot.
    void set_sources(const InjTable &inj, int ntrace, const float *src);
    void set_receivers(const ExtTable &ext, int nr_per_shot);
    void reset();                         // zero wavefields, apply the initial condition
    void run(int it0, int nsteps);        // advance all shots by nsteps from time index it0 (async)
    void extract_last();                  // receivers at it = nt-1 (after the last step)
    void copy_traces(float *rcv);         // [nshots][nrcomp][nr][nt] raw traces (host)
    int launches_per_step() const;

    // Shot slots: in continuous mode every shot of the batch carries its own
    // start step t0 (all 0 when the mode begins); its sources and receivers
    // run on its local time it - t0, and a run is no longer bounded by nt.
    // join_shot replaces the geometry of one slot (tables of all shots,
    // gidx offset by shot as in set_sources/set_receivers, the same source
    // traces) and restarts it at step t0: its three wavefield levels and its
    // traces are zeroed and its initial condition applied.  Throws when one
    // of its source points lies in a taper zone, where the first step of a
    // restarted shot would taper its initial state (the reference tapers
    // prev only after the first step).  An idle slot (release_shot) is
    // advanced by no kernel until a shot joins it.
    void set_continuous();
    bool continuous() const { return continuous_; }
    void join_shot(int slot, const InjTable &inj, const ExtTable &ext, int t0);
    void release_shot(int slot);
    void copy_shot_traces(int slot, float *rcv);  // [nrcomp][nr][nt] raw traces of one slot (host)

    // DAS (fibre) receivers: the strain along each fibre from the three
    // components of its dipole rows (dipole_to_strain, misc.cpp:11-42), on
    // the device.  w: [nshots][nr][3] projection weights (cos dip cos az,
    // cos dip sin az, sin dip, as floats), gl the gauge length.
    void set_das(const std::vector<float> &w, int nr, float gl);
    // strain [nsh][nr][nt] of shots [s0, s0+nsh) of the raw traces
    // [nshots][3][nr][nt] (device; kept until the next call)
    const float *strain_traces(int s0, int nsh);
    // its adjoint: strain sources [nshots][nr][nt] to dipole sources
    // [nshots][3][nr][nt] (device; kept until the next call)
    const float *strain_adjoint(const float *src_dev);
    void copy_strain(int s0, int nsh, float *rcv);  // strain_traces to the host

    // --- operator / gradient path (one shot or a batch of shots) -------------
    // Snapshot storage of the forward wavefield for the imaging condition.
    enum Storage { STORE_FP32 = 0, STORE_FP16P = 1 };
    void set_storage(int mode) { storage_ = mode; }
    // HBM budget of the forward-wavefield storage of the gradient path (bytes,
    // 0: unlimited).  When full storage exceeds it, binomial checkpointing
    // (below) replaces it with as many checkpoint slots as fit the budget.
    void set_snapshot_budget(int64_t bytes) { budget_ = bytes; }
    // Binomial checkpointing (the schedule of Griewank and Walther's revolve):
    // `slots` restart states (prev, curr) of the batch held on the device,
    // stored in FP32 (precision 0) or per-(state, level, shot, component)
    // scaled BF16 (1) or FP16 (2); the adjoint recomputes the forward states
    // it needs from them, placing new checkpoints on the way so that the
    // number of recomputed steps is the minimum for that many slots.
    // slots 0: full storage unless the budget forces checkpointing.
    void set_checkpointing(int slots, int precision) { rv_C_req_ = slots; rv_prec_ = precision; }
    int checkpoint_slots() const { return rv_C_; }        // 0: full storage
    int64_t recomputed_steps() const { return rv_steps_; }  // chain steps recomputed by the last adjoint
    // forward: full time loop; keeps snapshots when store && sub > 0.  Tables of
    // all shots (as set_sources/set_receivers); rcv [nshots][ncomp][nr][nt].
    void forward(const InjTable &inj, int ntrace, const float *src, const ExtTable &ext, float *rcv, bool store);
    // adjoint + imaging of every shot of the batch; grad out: [min(3,nm)][nxyz]
    // float, summed over the shots in FP64 (before H quadrature and chain
    // rule), or with per-shot gradients [nshots][min(3,nm)][nxyz]
    void set_per_shot_gradient(bool on) { per_shot_grad_ = on; }
    void adjoint(const InjTable &inj, int ntrace, const float *adj_src, float *grad);
    // the same with the adjoint sources [ntrace][nt] already on the device
    // (stream-ordered after the engine's earlier work)
    void adjoint_dev(const InjTable &inj, int ntrace, const float *adj_src_dev, float *grad);
    // traces of the last forward [nshots][ncomp][nr][nt] on the device (a
    // forward called with rcv == nullptr leaves them there)
    const float *traces_dev() const { return rcv_dev_.as<float>(); }

private:
    void adjoint_impl(const InjTable &inj, int ntrace, const float *adj_src, const float *adj_src_dev, float *grad);

public:
    int64_t snapshot_bytes() const
    {
        return snaps_.bytes + snapq_.bytes + enc_.bytes + snapz_.bytes + rv_store_.bytes + rv_scale_.bytes +
               rec_fields_.bytes;
    }

    // Diagnostic timing of the step's main kernel (the fused interior kernel,
    // else the per-point step kernel): a pair of CUDA events on the engine
    // stream around each of its launches, up to max_launches (0: off).
    void time_main_kernel(int max_launches);
    // Summed event time since time_main_kernel(); launches timed, grid-point
    // updates per launch and the kernel's name.  Synchronises the stream.
    double main_kernel_ms(int *launches, int64_t *points, const char **name);

    bool has_snapshots() const { return snaps_valid_; }
    int64_t device_bytes() const;
    void sync();

private:
    void upload_inj(const InjTable &t, int ntrace, DevInj &d);
    void init_prev(const DevInj &inj, const float *src_dev, float *prev, int only_shot = -1);
    void upload_tables(const InjTable &inj, const ExtTable &ext);
    void step(float *prev, float *curr, float *next, bool taper_prev);
    void inject(const DevInj &inj, const float *src_dev, int it, float *next);
    void extract(const DevExt &ext, const float *curr, float *rcv_dev, int it);
    void image(int itl, const float *curr, const float *prevl);
    float *level(int l) const;

    int device_;
    int sm_count_ = 148;           // streaming multiprocessors of the device
    Problem pb_;
    void *stream_ = nullptr;
    // second stream of a step: the edge tiles and y-wall slabs run beside the
    // interior tiles (fork and join events on stream_); FWI_CONCURRENT=0 keeps
    // one stream
    void *side_ = nullptr, *ev_fork_ = nullptr, *ev_join_ = nullptr;
    bool conc_ = true;
    bool continuous_ = false;     // shot slots with their own start steps (shot_t0_)
    bool per_shot_grad_ = false;  // the adjoint keeps one gradient per shot
    bool image_split_ = true;     // imaging in an interior-box and a shell launch (FWI_IMAGE_SPLIT=0: one)
    DevBuf shot_t0_, shot_active_;
    DevBuf das_w_, das_rcv_, das_src_;  // DAS projection weights, strain traces, dipole sources
    int das_nr_ = 0;
    float das_gl_ = 0.f;
    DevBuf model_;                 // [nm][nxyz]
    DevBuf w2c_;                   // closure weights of the D2var coefficients per axis (StepArgs::w2c)
    const float *w2c_ptr_[3][3] = {};
    DevBuf fields_;                // [3 levels][nshots][ncomp][nxyz]
    int rot_ = 0;                  // rotation of the three time levels
    DevBuf aux_;                   // elastic derivative scratch [nshots][naux][nxyz] (per-point path)
    DevBuf snaps_;                 // FP32 storage: [nsnap][nshots][ncomp][nxyz]; FP16P: 3-slot decode ring
    DevBuf snapq_;                 // FP16P: second-difference residuals [nsnap][nshots][ncomp][nxyz] (half)
    DevBuf snaps_scale_;           // FP16P: residual scales [nsnap][nshots*ncomp] (float)
    DevBuf enc_;                   // FP16P: encoder/decoder state, two FP64 levels [2][nshots][ncomp][nxyz]
    DevBuf amax_;                  // FP16P: per (shot, comp) max |residual| of one snapshot
    DevBuf snapz_;                 // FP16P: zero snapshot (indices past the last forward state)
    int storage_ = STORE_FP32;
    int nsnap_ = 0;
    int nwritten_ = 0;             // snapshots 0..nwritten_-1 hold forward states, the rest are zero
    int dec_lo_ = 0;               // FP16P decoder: state holds snapshots dec_lo_, dec_lo_+1
    void snap_store(int k);
    int64_t budget_ = 0;
    // binomial checkpointing over the chain of snapshot states 0..rv_K_
    // (state k: the time levels (prev, curr) at step k*sub)
    int rv_C_req_ = 0, rv_prec_ = 0;
    int rv_C_ = 0;                 // slots in use for this forward (0: full storage)
    int rv_K_ = 0;
    int rv_pos_ = -1;              // state held by the recomputation levels (-1: none)
    int rv_rot_ = 0;               // their rotation
    std::vector<int> rv_pos_stack_, rv_slot_stack_, rv_free_;  // checkpoints (positions increase up the stack)
    std::vector<int> rv_mark_;     // forward sweep: 1 where a checkpoint is taken
    const int32_t *rv_split_ = nullptr;  // optimal first advance for (length, free slots)
    int64_t rv_steps_ = 0;
    int ring_[3] = {-1, -1, -1};   // snapshot index held by each slot of the FP32 ring (snaps_)
    DevBuf rv_store_;              // [C][2 levels][nshots][ncomp][nxyz], FP32 or 16-bit
    DevBuf rv_scale_;              // [C][2][nshots*ncomp] scales of the 16-bit slots
    DevBuf rec_fields_;            // time levels of the recomputation
    bool no_extract_ = false;
    void rv_store(int slot, const float *prev, const float *curr);
    void rv_restore(int slot);
    void rv_advance(int d);        // recomputation levels: d chain steps forward
    void rv_goto(int t);           // recomputation levels to state t (t below the last visited)
    const float *snap_fp32(int kk);  // FP32 view of snapshot kk (decoding as needed)
    bool snaps_valid_ = false;
    DevBuf grad_;                  // [3][nxyz] double
    DevBuf sdiv_;                  // boundary divisors, packed
    const float *sdiv_ptr_[6][3] = {};
    DevBuf taper_;                 // packed taper tables
    const float *taper_ptr_[6] = {};
    int scale_ = 0;
    bool march_ = false;           // marching elastic kernel over all planes
    bool afused_ = false;          // acoustic marching kernel (else the per-point kernel)
    bool slab_march_ = false;      // fused path: y-wall slabs by the marching kernel (else per-point kernels)
    bool fused_ = false;           // fused elastic kernel for the interior planes
    int fused_minb_ = 2;           // resident CTAs per SM the fused kernel is compiled for
    bool graphs_ = true;           // modeling runs replay captured three-step graphs
    void *graph_exec_ = nullptr;   // cudaGraphExec_t of the captured steps
    uint64_t graph_key_ = 0;       // graph_key() at capture
    DevBuf it_dev_;                // device time index of replayed steps
    int *itp_ = nullptr;           // non-null while capturing: kernels read the time index there
    void run_step(int it, bool taper_prev);
    uint64_t graph_key() const;
    bool capture_graph();
    void drop_graph();
    bool pair_ = true;             // isotropic interior tiles by the paired kernel (pair.cuh)
    int pair_edge_ = 2;            // its edge tiles: 0 one-point kernel, 1 x-face-only tiles paired, 2 all paired
    bool fused_split_ = true;      // interior and edge tiles of the fused kernel in separate launches
    int fused_waves_ = 8;          // y chunks per tile column: about this many waves of resident CTAs
    int pair_waves_ = 4;           // the same for the paired kernel's launches
    bool slabs_last_ = true;       // the y-wall slabs after the side stream's edge tiles (FWI_SLABS_LAST=0: first)
    int side_modes_ = 0x30;        // bit m: edge mode m of the paired kernel on the second stream
    bool fused_split_active() const;
    bool tma_ = false;             // fused kernel copies planes with bulk-tensor copies
    DevBuf tma_err_;               // int: a fused-kernel wait for a plane copy gave up
    DevBuf src_dev_, rcv_dev_;
    std::vector<void *> kev_;      // event pairs (begin, end) of the timed main-kernel launches
    int kev_used_ = 0;
    bool ktime_ = false;
    const char *kname_ = "";
    int64_t kpts_ = 0;
    void kmark(bool begin, const char *name, int64_t pts);
    DevInj inj_;
    DevInj adj_inj_;                  // adjoint source tables (reused between adjoints)
    DevBuf adj_src_buf_, grad_f32_;   // host adjoint sources on the device, FP32 gradient
    DevExt ext_;
};

// One elastic (nmodels 3) or VTI (6) leapfrog step next = F(prev, curr) on
// caller-owned device buffers of the current device, with the derivative
// scratch in a static device array: no device or host allocation.  Faces bc 0
// or 1 only, no taper, at most 2^18 grid points (fwi_elastic_step_static).
void static_elastic_step(const fwi_grid &grid, int nmodels, const int bc[6], float dt, const float *model,
                         const float *prev, const float *curr, float *next, void *stream);

// The FWI objective's residual on the device, batch by batch: observed
// traces kept on the device, the sinc taps of the data and propagation axes,
// the adjoint sources of the last batch (kernel k_residual, engine.cu).
class DeviceResidual {
public:
    // upload the observed traces [nshots][ntr][ntd] once per device
    void set_observed(int device, const std::vector<float> &obs);
    // sinc taps between the data axis (ntd, dtd) and the propagation axis (nt, dt)
    void set_axes(int hl, int ntd, float dtd, int nt, float dt);
    // residual of the ntraces traces of eng's last forward against the observed
    // traces from obs_offset on; returns the FP64 misfit sum (before 0.5 dt /
    // dnorm), leaves the adjoint sources on the device and, when residual is
    // not null, copies the residual [ntraces][ntd] there.  Synchronises eng's stream.
    double run(Engine &eng, size_t obs_offset, int ntraces, int seismotype, float alpha, float *residual,
               double *per_trace = nullptr, const float *traces = nullptr);
    const float *adjoint_sources() const { return asrc_.as<float>(); }
    // Data of ntraces raw traces [ntraces][nt] on the device (modeling output,
    // we_op.cpp:929-941): Dt for velocity data, times alpha, adjoint
    // resampling to the data axis, into out [ntraces][ntd] on the host; the
    // host formulation's operations in its order (same values bit for bit).
    // Synchronises eng's stream.
    void data(Engine &eng, const float *traces, int ntraces, int seismotype, float alpha, float *out);

private:
    int device_ = -1, nt_ = -1, ntd_ = -1, hl_ = -1;
    float dt_ = 0.f, dtd_ = 0.f;
    DevBuf obs_, first_, count_, off_, s_, win_, jlo_, jhi_, asrc_, resid_, part_, bad_;
};

}  // namespace fwi
