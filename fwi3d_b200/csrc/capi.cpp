// extern "C" entry points of libfwi3d_b200.so (declared in include/fwi3d_gpu.h).
//
// fwi_op mirrors one nl_we_op_{a,e,vti} object: it holds the per-shot
// wavelet and geometry (we_op.hpp:59-79), a mutable copy of the parameters
// that analyzeModel updates on every call (dt, courant, sub), and the device
// state the forward pass leaves for the adjoint (the reference keeps it in
// the mutable _zfp_wfld member, we_op.hpp:23).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fwi3d_gpu.h"
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "engine.h"
#include "host_ops.h"

using namespace fwi;

namespace {
thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

template <class F>
int guarded(F &&f)
{
    try {
        f();
        g_err.clear();
        return FWI_OK;
    } catch (const FwiError &e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(FWI_ERR_OOM, "host allocation failed");
    } catch (const std::invalid_argument &e) {
        return fail(FWI_ERR_ARG, e.what());
    } catch (const std::exception &e) {
        return fail(FWI_ERR_CUDA, e.what());
    }
}

bool finite_all(const float *p, int64_t n)
{
    int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
    for (int64_t i = 0; i < n; i++) bad |= !std::isfinite(p[i]);
    return !bad;
}
}  // namespace

struct fwi_op {
    int device = 0;
    fwi_grid grid{};
    int nmodels = 3;
    fwi_param par{};
    int nt_data = 0;
    float dt_data = 0.f;
    int nscomp = 1, nrcomp = 1;
    std::vector<float> wavelet;  // [nscomp][nt_data]
    float sxyz[3] = {0, 0, 0};
    int nr = 0;
    std::vector<float> rxyz;     // [nr][5]
    Problem pb{};
    std::unique_ptr<Engine> eng;
    std::vector<float> conv;     // converted model of the last call

    int64_t nxyz() const { return (int64_t)grid.nx * grid.ny * grid.nz; }
    int ncomp() const { return nmodels == 2 ? 1 : 3; }

    // analyzeModel + convert_model on a copy of `model`, then make sure the
    // engine matches the resulting time axis (we_op.cpp:874-878, 951-958).
    void prepare(const float *model)
    {
        std::vector<float> m(model, model + nmodels * nxyz());
        TimeAxis ta = analyze_model(m, nmodels, grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz, nt_data, dt_data,
                                    par);
        par.dt = ta.dt;
        par.courant = ta.courant;
        par.sub = ta.sub;
        convert_model(m, nmodels, nxyz());
        Problem p{};
        p.nmodels = nmodels;
        p.nx = grid.nx;
        p.ny = grid.ny;
        p.nz = grid.nz;
        p.dx = grid.dx;
        p.dy = grid.dy;
        p.dz = grid.dz;
        p.dt = ta.dt;
        p.nt = ta.nt;
        p.sub = ta.sub;
        std::memcpy(p.bc, par.bc, sizeof(p.bc));
        for (int f = 0; f < 6; f++) p.bc[f] = std::max(0, p.bc[f]);
        std::memcpy(p.taper, par.taper, sizeof(p.taper));
        p.taper_strength = par.taper_strength;
        p.free_surface_stiffness = nmodels == 2 ? std::max(par.free_surface_stiffness, 1.0f) : par.free_surface_stiffness;
        const bool same = eng && pb.nt == p.nt && pb.dt == p.dt && pb.sub == p.sub;
        pb = p;
        if (!same) eng.reset(new Engine(device, pb));
        eng->set_storage(par.snapshot_storage);
        eng->set_snapshot_budget((int64_t)((double)par.snapshot_budget_gb * 1e9));
        eng->set_checkpointing(par.checkpoint_slots, par.checkpoint_precision);
        eng->set_model(m.data());
        conv.swap(m);
    }

    std::vector<Loc> receivers() const
    {
        std::vector<Loc> l(nr);
        for (int r = 0; r < nr; r++) l[r] = Loc{rxyz[5 * r], rxyz[5 * r + 1], rxyz[5 * r + 2]};
        return l;
    }
    bool das() const { return nmodels != 2 && par.gl > 0; }
    std::vector<Loc5> fibres() const
    {
        std::vector<Loc5> l(nr);
        for (int r = 0; r < nr; r++)
            l[r] = Loc5{rxyz[5 * r], rxyz[5 * r + 1], rxyz[5 * r + 2], rxyz[5 * r + 3], rxyz[5 * r + 4]};
        return l;
    }
    std::vector<float> rcv_angle(int k) const
    {
        std::vector<float> v(nr);
        for (int r = 0; r < nr; r++) v[r] = rxyz[5 * r + k];
        return v;
    }
};

struct fwi_batch {
    int device = 0;
    fwi_grid grid{};
    int nmodels = 3;
    fwi_param par{};
    int nt_data = 0;
    float dt_data = 0.f;
    int nshots = 1, nr = 0, nscomp = 1, nrcomp = 1;
    int it = 0;  // time steps run since reset
    Problem pb{};
    std::unique_ptr<Engine> eng;
    std::vector<float> sxyz, rxyz;  // geometry of every slot: [nshots][3], [nshots][nr][5]
    std::vector<int> t0;            // start step of every slot (shot slots)
    DeviceResidual out;             // modeling output on the device (sinc resampling)
};

namespace {
// FWI_BATCH_TIMING=1: host-clock times of the phases of a batch call on
// stderr (the device work of a phase is synchronised only where the phase
// ends in a synchronisation anyway).
struct PhaseClock {
    bool on = false;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    PhaseClock()
    {
        const char *e = std::getenv("FWI_BATCH_TIMING");
        on = e && e[0] == '1';
    }
    void mark(const char *what)
    {
        if (!on) return;
        const auto n = std::chrono::steady_clock::now();
        std::fprintf(stderr, "fwi batch: %-28s %8.3f s\n", what, std::chrono::duration<double>(n - t).count());
        t = n;
    }
};

// DAS channel s*nr + r of a [nshots][nr][5] receiver array: its fibre, and
// the projection weights of dipole_to_strain (misc.cpp:11-42) as that
// routine forms them in float.
std::vector<Loc5> shot_fibres(const float *rxyz, int s, int nr)
{
    std::vector<Loc5> l(nr);
    const float *r5 = rxyz + (size_t)5 * nr * s;
    for (int r = 0; r < nr; r++) l[r] = Loc5{r5[5 * r], r5[5 * r + 1], r5[5 * r + 2], r5[5 * r + 3], r5[5 * r + 4]};
    return l;
}
std::vector<float> das_weights(const float *rxyz, int s0, int nsh, int nr)
{
    std::vector<float> w((size_t)nsh * nr * 3);
    for (int b = 0; b < nsh; b++)
        for (int r = 0; r < nr; r++) {
            const float *r5 = rxyz + ((size_t)(s0 + b) * nr + r) * 5;
            const float cd = (float)std::cos((double)r5[3]), sd = (float)std::sin((double)r5[3]);
            const float ca = (float)std::cos((double)r5[4]), sa = (float)std::sin((double)r5[4]);
            float *o = w.data() + ((size_t)b * nr + r) * 3;
            o[0] = cd * ca;
            o[1] = cd * sa;
            o[2] = sd;
        }
    return w;
}

// Injection and extraction tables of a batch's current geometry (gidx offset
// by shot; source traces shot * nscomp + component).
void batch_tables(const fwi_batch &b, InjTable &all, ExtTable &ext)
{
    const Problem &p = b.pb;
    const int64_t n = p.nxyz();
    const int nc = p.ncomp();
    ext.nrec = b.nshots * b.nr;
    for (int s = 0; s < b.nshots; s++) {
        const float *sx = b.sxyz.data() + 3 * s;
        PointOp inj = make_delta(p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, b.grid.ox, b.grid.oy, b.grid.oz,
                                 {Loc{sx[0], sx[1], sx[2]}}, b.par.mt != 0);
        InjTable t = injection_table(inj, p.nx, p.ny, p.nz, nc);
        for (int c = 0; c < nc; c++)
            for (size_t k = 0; k < t.gidx[c].size(); k++) {
                all.gidx[c].push_back(t.gidx[c][k] + s * n);
                all.trace[c].push_back(t.trace[c][k] + s * b.nscomp);
                all.w[c].push_back(t.w[c][k]);
            }
        ExtTable e;
        if (b.par.gl > 0) {
            // DAS: the channel's two dipole ends (dipole_m3, injector.cpp:313-493)
            e = dipole_extraction_table(make_dipole(p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, b.grid.ox, b.grid.oy, b.grid.oz,
                                                    shot_fibres(b.rxyz.data(), s, b.nr), b.par.gl),
                                        p.nx, p.ny, p.nz);
        } else {
            std::vector<Loc> rl(b.nr);
            const float *rs = b.rxyz.data() + (size_t)5 * b.nr * s;
            for (int r = 0; r < b.nr; r++) rl[r] = Loc{rs[5 * r], rs[5 * r + 1], rs[5 * r + 2]};
            PointOp rop = make_delta(p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, b.grid.ox, b.grid.oy, b.grid.oz, rl, false);
            e = extraction_table(rop, p.nx, p.ny, p.nz);
        }
        ext.ntap = e.ntap;
        for (auto g : e.gidx) ext.gidx.push_back(g + s * n);
        ext.w.insert(ext.w.end(), e.w.begin(), e.w.end());
    }
}

// Raw traces [nrcomp*nr][nt] of one shot to data [nrcomp*nr][nt_data]: time
// derivative for velocity data, dt/dt_data, resampling (as fwi_batch_traces).
void batch_shot_output(const fwi_batch &b, float *r, float *d)
{
    const int nt = b.pb.nt;
    const int ntr = b.nrcomp * b.nr;
    std::vector<float> v;
    if (b.par.seismotype == 1) {
        v.resize((size_t)ntr * nt);
        apply_dt(false, r, v.data(), ntr, nt, b.pb.dt);
        r = v.data();
    }
    const float alpha = b.pb.dt / b.dt_data;
    for (size_t i = 0; i < (size_t)ntr * nt; i++) r[i] *= alpha;
    std::fill(d, d + (size_t)ntr * b.nt_data, 0.f);
    resample_adjoint(b.par.resampling_linear == 0, b.par.sinc_half_length, d, b.nt_data, b.dt_data, r, nt, b.pb.dt,
                     ntr);
}

// Data of shots [s0, s0+nsh) to data [nsh][nrcomp][nr][nt_data] on the device
// (sinc resampling and traces that fit the kernel's shared memory), false
// where the host path must take them.
bool batch_device_output(fwi_batch &b, int s0, int nsh, float *data)
{
    const int nt = b.pb.nt;
    const char *he = std::getenv("FWI_HOST_OUTPUT");  // =1: the host path (the same values bit for bit)
    if ((he && he[0] == '1') || b.par.resampling_linear != 0 || std::max(nt, b.nt_data) > kResidualMaxSamples)
        return false;
    const int ntr = b.nrcomp * b.nr;
    const float *src = b.par.gl > 0 ? b.eng->strain_traces(s0, nsh)
                                    : b.eng->traces_dev() + (size_t)s0 * b.pb.ncomp() * b.nr * nt;
    b.out.set_axes(b.par.sinc_half_length, b.nt_data, b.dt_data, nt, b.pb.dt);
    b.out.data(*b.eng, src, nsh * ntr, b.par.seismotype, b.pb.dt / b.dt_data, data);
    return true;
}
}  // namespace

struct fwi_objective {
    int device = 0;
    fwi_grid grid{};
    int nmodels = 3;
    fwi_param par{};
    int nt_data = 0;
    float dt_data = 0.f;
    int nshots = 1, nr = 0, nscomp = 1, nrcomp = 1, batch = 1;
    std::vector<float> wavelet, sxyz, rxyz, observed;
    double dnorm = 1.0;
    int normalize = 1;
    Problem pb{};
    std::map<int, std::unique_ptr<Engine>> eng;  // one engine per batch size
    int64_t device_bytes = 0;
    DeviceResidual dres;  // residual on the device (observed traces, resampling taps)
};

namespace {
// Normalisation of the misfit (nlls_fwi::_dnorm, optimization.hpp:386-393):
// sum of the squared observed data times dt, or 1; over all shots, or (sh
// >= 0) over shot sh alone (each request of a batched gradient is normalised
// by its own data).
double data_norm(const fwi_objective &o, int sh = -1)
{
    if (!o.normalize) return 1.0;
    const size_t nd = (size_t)o.nrcomp * o.nr * o.nt_data;
    const size_t b = sh < 0 ? 0 : (size_t)sh * nd, e = sh < 0 ? o.observed.size() : b + nd;
    double ss = 0;
    for (size_t i = b; i < e; i++) ss += (double)o.observed[i] * o.observed[i];
    const double dn = ss * o.dt_data;
    return dn < 1e-16 ? 1.0 : dn;
}
}  // namespace

extern "C" {

void fwi_param_default(fwi_param *p)
{
    std::memset(p, 0, sizeof(*p));
    p->courant = 0.5f;
    p->dt = -1.f;
    p->sub = 0;
    p->resampling_linear = 0;
    p->sinc_half_length = 11;
    p->mt = 0;
    p->mxx = p->myy = p->mzz = p->mxy = p->mxz = p->myz = 1.f;
    p->seismotype = 0;
    p->gl = 0.f;
    for (int f = 0; f < 6; f++) {
        p->bc[f] = 1;
        p->taper[f] = 0;
    }
    p->free_surface_stiffness = 1.05f;
    p->taper_strength = 0.05f;
    p->vpmin = 0.2f;
    p->vpmax = 8.f;
    p->vsmin = 0.1f;
    p->vsmax = 5.f;
    p->rhomin = 0.1f;
    p->rhomax = 8.f;
    p->deltamin = -0.5f;
    p->deltamax = 1.f;
    p->epsilonmin = 0.f;
    p->epsilonmax = 1.f;
    p->gammamin = 0.f;
    p->gammamax = 1.f;
    p->soft_clip = 0;
    p->verbose = 0;
    p->snapshot_storage = 0;
    p->snapshot_budget_gb = 0.f;
    p->checkpoint_slots = 0;
    p->checkpoint_precision = 0;
}

const char *fwi_last_error(void) { return g_err.c_str(); }

const char *fwi_version(void) { return "fwi3d_b200 0.1 (sm_100a)"; }

int fwi_op_create(fwi_op **out, int device, const fwi_grid *grid, int nmodels, const fwi_param *par,
                  const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data, const float *sxyz, int nr,
                  const float *rxyz)
{
    if (!out || !grid || !par || !wavelet || !sxyz || (nr > 0 && !rxyz)) return fail(FWI_ERR_ARG, "null argument");
    *out = nullptr;
    if (nmodels != 2 && nmodels != 3 && nmodels != 6)
        return fail(FWI_ERR_ARG, "The model must contain 2, 3, or 6 parameters");
    if (grid->nx < 12 || grid->ny < 12 || grid->nz < 12)
        return fail(FWI_ERR_ARG, "each grid axis needs at least 12 points");
    if (nt_data < 2 || !(dt_data > 0)) return fail(FWI_ERR_ARG, "the wavelet needs at least 2 samples and dt > 0");
    if (nr < 1) return fail(FWI_ERR_ARG, "at least one receiver is required");
    return guarded([&] {
        std::unique_ptr<fwi_op> op(new fwi_op());
        op->device = device;
        op->grid = *grid;
        op->nmodels = nmodels;
        op->par = *par;
        if (nmodels == 2) op->par.mt = 0;
        op->nt_data = nt_data;
        op->dt_data = dt_data;
        if (nmodels == 2) op->par.gl = 0.f;  // analyzeGeometry, we_op.cpp:11-14
        op->nscomp = nmodels == 2 ? 1 : (op->par.mt ? 6 : 3);
        op->nrcomp = nmodels == 2 ? 1 : (op->par.gl > 0 ? 1 : 3);
        op->wavelet = expand_wavelet(wavelet, wavelet_ncomp, nt_data, nmodels, op->par);
        std::memcpy(op->sxyz, sxyz, sizeof(op->sxyz));
        op->nr = nr;
        op->rxyz.assign(rxyz, rxyz + 5 * nr);
        // source / receivers inside the model (analyzeGeometry, we_op.cpp:84-108)
        const fwi_grid &g = *grid;
        const float prec = std::min(g.dx, g.dz) * 1e-3f;
        auto inside = [&](float x, float y, float z) {
            return (x - g.ox >= -prec) && (-prec <= -x + g.ox + (g.nx - 1) * g.dx) && (y - g.oy >= -prec) &&
                   (-prec <= -y + g.oy + (g.ny - 1) * g.dy) && (z - g.oz >= -prec) &&
                   (-prec <= -z + g.oz + (g.nz - 1) * g.dz);
        };
        if (!inside(sxyz[0], sxyz[1], sxyz[2]))
            throw FwiError(FWI_ERR_ARG, "Shot falls outside subsurface model boundaries");
        for (int r = 0; r < nr; r++) {
            if (!inside(rxyz[5 * r], rxyz[5 * r + 1], rxyz[5 * r + 2]))
                throw FwiError(FWI_ERR_ARG, "Receiver " + std::to_string(r) + " falls outside subsurface model boundaries");
            if (op->das() && !dipole_inside(Loc5{rxyz[5 * r], rxyz[5 * r + 1], rxyz[5 * r + 2], rxyz[5 * r + 3],
                                                 rxyz[5 * r + 4]},
                                            op->par.gl, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.ox, g.oy, g.oz))
                throw FwiError(FWI_ERR_ARG, "DAS channel " + std::to_string(r) +
                                                " has its gauge length falling outside subsurface model boundaries");
        }
        *out = op.release();
    });
}

int fwi_op_forward(fwi_op *op, int add, const float *model, float *data)
{
    if (!op || !model || !data) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] {
        if (!finite_all(model, op->nmodels * op->nxyz())) throw FwiError(FWI_ERR_NAN, "model contains non-finite values");
        op->prepare(model);
        const Problem &pb = op->pb;
        const int nt = pb.nt;
        const bool sinc = op->par.resampling_linear == 0;
        // wavelet -> propagation sampling (we_op.cpp:907-911)
        std::vector<float> src((size_t)op->nscomp * nt);
        resample_forward(sinc, op->par.sinc_half_length, op->wavelet.data(), op->nt_data, op->dt_data, src.data(), nt,
                         pb.dt, op->nscomp);
        PointOp inj = make_delta(pb.nx, pb.ny, pb.nz, pb.dx, pb.dy, pb.dz, op->grid.ox, op->grid.oy, op->grid.oz,
                                 {Loc{op->sxyz[0], op->sxyz[1], op->sxyz[2]}}, op->par.mt != 0);
        const InjTable it = injection_table(inj, pb.nx, pb.ny, pb.nz, op->ncomp());
        ExtTable et;
        if (op->das()) {
            et = dipole_extraction_table(make_dipole(pb.nx, pb.ny, pb.nz, pb.dx, pb.dy, pb.dz, op->grid.ox, op->grid.oy,
                                                     op->grid.oz, op->fibres(), op->par.gl),
                                         pb.nx, pb.ny, pb.nz);
        } else {
            PointOp ext = make_delta(pb.nx, pb.ny, pb.nz, pb.dx, pb.dy, pb.dz, op->grid.ox, op->grid.oy, op->grid.oz,
                                     op->receivers(), false);
            et = extraction_table(ext, pb.nx, pb.ny, pb.nz);
        }
        const int ncr = op->ncomp();
        std::vector<float> rcv((size_t)ncr * op->nr * nt);
        op->eng->forward(it, op->nscomp, src.data(), et, rcv.data(), pb.sub > 0);
        if (!finite_all(rcv.data(), (int64_t)rcv.size())) throw FwiError(FWI_ERR_NAN, "non-finite values in the traces");
        if (op->das()) {
            // strain along the fibre (we_op.cpp:929)
            const std::vector<float> dip = op->rcv_angle(3), az = op->rcv_angle(4);
            dipole_to_strain(false, rcv.data(), dip.data(), az.data(), op->nr, nt, op->par.gl);
            rcv.resize((size_t)op->nr * nt);
        }
        const int ntr = op->nrcomp * op->nr;
        if (op->par.seismotype == 1) {
            // particle velocity (we_op.cpp:932-938)
            std::vector<float> v(rcv.size());
            apply_dt(false, rcv.data(), v.data(), ntr, nt, pb.dt);
            rcv.swap(v);
        }
        const float alpha = pb.dt / op->dt_data;
        for (auto &v : rcv) v *= alpha;
        if (!add) std::fill(data, data + (size_t)ntr * op->nt_data, 0.f);
        resample_adjoint(sinc, op->par.sinc_half_length, data, op->nt_data, op->dt_data, rcv.data(), nt, pb.dt, ntr);
    });
}

int fwi_op_jacobianT(fwi_op *op, int add, float *grad, const float *model0, const float *data)
{
    if (!op || !grad || !model0 || !data) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] {
        if (!op->eng || !op->eng->has_snapshots())
            throw FwiError(FWI_ERR_STATE, "jacobianT needs a preceding forward on this operator with sub > 0");
        if (!finite_all(model0, op->nmodels * op->nxyz())) throw FwiError(FWI_ERR_NAN, "model contains non-finite values");
        const int64_t n = op->nxyz();
        const int nm = std::min(3, op->nmodels);
        // analyzeModel must reproduce the forward's time axis (same model in FWI)
        const Problem before = op->pb;
        {
            std::vector<float> m(model0, model0 + op->nmodels * n);
            TimeAxis ta = analyze_model(m, op->nmodels, op->grid.nx, op->grid.ny, op->grid.nz, op->grid.dx, op->grid.dy,
                                        op->grid.dz, op->nt_data, op->dt_data, op->par);
            if (ta.nt != before.nt || ta.dt != before.dt || ta.sub != before.sub)
                throw FwiError(FWI_ERR_STATE, "the background model changes the time axis of the stored forward pass");
            op->par.dt = ta.dt;
            op->par.courant = ta.courant;
            op->par.sub = ta.sub;
            convert_model(m, op->nmodels, n);
            op->eng->set_model(m.data());
            op->conv.swap(m);
        }
        const Problem &pb = op->pb;
        const int nt = pb.nt;
        const int ncr = op->ncomp();
        const int ntr = ncr * op->nr;
        const bool sinc = op->par.resampling_linear == 0;
        std::vector<float> temp;
        if (add) temp.assign(grad, grad + nm * n);
        else std::fill(grad, grad + nm * n, 0.f);
        // data -> propagation sampling, Ht^-1, time reversal, -alpha (we_op.cpp:994-1003);
        // DAS data fill component 0 of the three
        std::vector<float> rcv((size_t)ntr * nt, 0.f);
        resample_forward(sinc, op->par.sinc_half_length, data, op->nt_data, op->dt_data, rcv.data(), nt, pb.dt,
                         op->nrcomp * op->nr);
        apply_ht(true, rcv.data(), rcv.data(), ntr, nt, pb.dt);
        for (int tr = 0; tr < ntr; tr++) std::reverse(rcv.begin() + (size_t)tr * nt, rcv.begin() + (size_t)(tr + 1) * nt);
        const float alpha = pb.dt / op->dt_data;
        for (auto &v : rcv) v *= -alpha;
        if (op->par.seismotype == 1) {
            std::vector<float> v(rcv.size());
            apply_dt(true, rcv.data(), v.data(), ntr, nt, pb.dt);
            rcv.swap(v);
        }
        InjTable it;
        if (op->das()) {
            // strain back to the dipole components (we_op.cpp:1015), dipole injection
            const std::vector<float> dip = op->rcv_angle(3), az = op->rcv_angle(4);
            dipole_to_strain(true, rcv.data(), dip.data(), az.data(), op->nr, nt, op->par.gl);
            it = dipole_injection_table(make_dipole(pb.nx, pb.ny, pb.nz, pb.dx, pb.dy, pb.dz, op->grid.ox, op->grid.oy,
                                                    op->grid.oz, op->fibres(), op->par.gl),
                                        pb.nx, pb.ny, pb.nz, ncr);
        } else {
            PointOp inj = make_delta(pb.nx, pb.ny, pb.nz, pb.dx, pb.dy, pb.dz, op->grid.ox, op->grid.oy, op->grid.oz,
                                     op->receivers(), false);
            it = injection_table(inj, pb.nx, pb.ny, pb.nz, ncr);
        }
        std::vector<float> g((size_t)nm * n);
        op->eng->adjoint(it, ntr, rcv.data(), g.data());
        // The reference accumulates the imaging sums into pmod itself, so with
        // add the previous content also goes through H and the chain rule
        // before `temp` is added back (we_op.cpp:968-972, 1027-1075).
        for (int64_t i = 0; i < nm * n; i++) grad[i] += g[i];
        for (int p = 0; p < nm; p++) apply_h3(grad + p * n, pb.nx, pb.ny, pb.nz, pb.dx, pb.dy, pb.dz);
        gradient_to_velocity(grad, op->conv.data(), op->nmodels, n);
        if (add)
            for (int64_t i = 0; i < nm * n; i++) grad[i] += temp[i];
        if (!finite_all(grad, nm * n)) throw FwiError(FWI_ERR_NAN, "non-finite values in the gradient");
    });
}

int fwi_op_get_info(const fwi_op *op, fwi_op_info *info)
{
    if (!op || !info) return fail(FWI_ERR_ARG, "null argument");
    info->dt = op->pb.dt;
    info->nt = op->pb.nt;
    info->sub = op->pb.sub;
    info->nscomp = op->nscomp;
    info->nrcomp = op->nrcomp;
    info->nr = op->nr;
    info->device_bytes = op->eng ? op->eng->device_bytes() : 0;
    return FWI_OK;
}

void fwi_op_destroy(fwi_op *op) { delete op; }

int fwi_batch_create(fwi_batch **out, int device, const fwi_grid *grid, int nmodels, const fwi_param *par,
                     const float *model, const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data,
                     int nshots, const float *sxyz, int nr, const float *rxyz)
{
    if (!out || !grid || !par || !model || !wavelet || !sxyz || !rxyz || nshots < 1 || nr < 1)
        return fail(FWI_ERR_ARG, "null argument, no shot or no receiver");
    *out = nullptr;
    if (nmodels != 2 && nmodels != 3 && nmodels != 6)
        return fail(FWI_ERR_ARG, "The model must contain 2, 3, or 6 parameters");
    return guarded([&] {
        std::unique_ptr<fwi_batch> b(new fwi_batch());
        b->device = device;
        b->grid = *grid;
        b->nmodels = nmodels;
        b->par = *par;
        if (nmodels == 2) b->par.mt = 0;
        if (nmodels == 2) b->par.gl = 0.f;  // analyzeGeometry, we_op.cpp:11-14
        b->nt_data = nt_data;
        b->dt_data = dt_data;
        b->nshots = nshots;
        b->nr = nr;
        b->nscomp = nmodels == 2 ? 1 : (b->par.mt ? 6 : 3);
        b->nrcomp = nmodels == 2 ? 1 : (b->par.gl > 0 ? 1 : 3);  // DAS: strain along each fibre
        if (b->par.gl > 0)
            for (int s = 0; s < nshots; s++)
                for (const Loc5 &l : shot_fibres(rxyz, s, nr))
                    if (!dipole_inside(l, b->par.gl, grid->nx, grid->ny, grid->nz, grid->dx, grid->dy, grid->dz,
                                       grid->ox, grid->oy, grid->oz))
                        throw FwiError(FWI_ERR_ARG, "a DAS channel has its gauge length falling outside subsurface "
                                                    "model boundaries");
        const int64_t n = (int64_t)grid->nx * grid->ny * grid->nz;
        if (!finite_all(model, nmodels * n)) throw FwiError(FWI_ERR_NAN, "model contains non-finite values");
        std::vector<float> m(model, model + nmodels * n);
        PhaseClock clk;
        TimeAxis ta = analyze_model(m, nmodels, grid->nx, grid->ny, grid->nz, grid->dx, grid->dy, grid->dz, nt_data,
                                    dt_data, b->par);
        convert_model(m, nmodels, n);
        Problem &p = b->pb;
        p.nmodels = nmodels;
        p.nx = grid->nx;
        p.ny = grid->ny;
        p.nz = grid->nz;
        p.dx = grid->dx;
        p.dy = grid->dy;
        p.dz = grid->dz;
        p.dt = ta.dt;
        p.nt = ta.nt;
        p.sub = 0;
        for (int f = 0; f < 6; f++) p.bc[f] = std::max(0, b->par.bc[f]);
        std::memcpy(p.taper, b->par.taper, sizeof(p.taper));
        p.taper_strength = b->par.taper_strength;
        p.free_surface_stiffness =
            nmodels == 2 ? std::max(b->par.free_surface_stiffness, 1.0f) : b->par.free_surface_stiffness;
        p.nshots = nshots;
        clk.mark("model analysis + convert");
        b->eng.reset(new Engine(device, p));
        clk.mark("engine (device buffers)");
        b->eng->set_model(m.data());
        clk.mark("set_model (tables)");
        // sources: the same wavelet for every shot, resampled once
        std::vector<float> w = expand_wavelet(wavelet, wavelet_ncomp, nt_data, nmodels, b->par);
        std::vector<float> w1((size_t)b->nscomp * p.nt);
        const bool sinc = b->par.resampling_linear == 0;
        resample_forward(sinc, b->par.sinc_half_length, w.data(), nt_data, dt_data, w1.data(), p.nt, p.dt, b->nscomp);
        std::vector<float> src((size_t)nshots * b->nscomp * p.nt);
        for (int s = 0; s < nshots; s++) std::memcpy(src.data() + (size_t)s * w1.size(), w1.data(), sizeof(float) * w1.size());
        b->sxyz.assign(sxyz, sxyz + 3 * (size_t)nshots);
        b->rxyz.assign(rxyz, rxyz + 5 * (size_t)nr * nshots);
        b->t0.assign(nshots, 0);
        InjTable all;
        ExtTable ext;
        clk.mark("wavelet");
        batch_tables(*b, all, ext);
        clk.mark("geometry tables (host)");
        b->eng->set_sources(all, nshots * b->nscomp, src.data());
        b->eng->set_receivers(ext, nr);
        if (b->par.gl > 0) b->eng->set_das(das_weights(rxyz, 0, nshots, nr), nr, b->par.gl);
        b->eng->sync();
        clk.mark("tables upload");
        *out = b.release();
    });
}

int fwi_batch_reset(fwi_batch *b)
{
    if (!b) return fail(FWI_ERR_ARG, "null batch");
    return guarded([&] {
        b->eng->reset();
        b->it = 0;
        std::fill(b->t0.begin(), b->t0.end(), 0);
    });
}

int fwi_batch_run(fwi_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return fail(FWI_ERR_ARG, "bad argument");
    return guarded([&] {
        // shot slots: no common end, each slot's sources and receivers stop at its own
        const int k = b->eng->continuous() ? nsteps : std::min(nsteps, b->pb.nt - 1 - b->it);
        if ((int64_t)b->it + k > INT32_MAX - 2 * (int64_t)b->pb.nt)
            throw FwiError(FWI_ERR_ARG, "time index range of the batch exhausted");
        b->eng->run(b->it, k);
        b->it += k;
    });
}

int fwi_batch_enable_slots(fwi_batch *b)
{
    if (!b) return fail(FWI_ERR_ARG, "null batch");
    return guarded([&] {
        if (b->it != 0) throw FwiError(FWI_ERR_STATE, "shot slots are enabled at time index 0 (after a reset)");
        b->eng->set_continuous();
        std::fill(b->t0.begin(), b->t0.end(), 0);
    });
}

int fwi_batch_join(fwi_batch *b, int slot, const float *sxyz, const float *rxyz)
{
    if (!b || !sxyz || !rxyz) return fail(FWI_ERR_ARG, "null argument");
    if (slot < 0 || slot >= b->nshots) return fail(FWI_ERR_ARG, "slot out of range");
    return guarded([&] {
        const std::vector<float> s0(b->sxyz), r0(b->rxyz);
        std::memcpy(b->sxyz.data() + 3 * (size_t)slot, sxyz, sizeof(float) * 3);
        std::memcpy(b->rxyz.data() + 5 * (size_t)b->nr * slot, rxyz, sizeof(float) * 5 * b->nr);
        InjTable all;
        ExtTable ext;
        try {
            if (b->par.gl > 0) {
                for (const Loc5 &l : shot_fibres(b->rxyz.data(), slot, b->nr))
                    if (!dipole_inside(l, b->par.gl, b->grid.nx, b->grid.ny, b->grid.nz, b->grid.dx, b->grid.dy,
                                       b->grid.dz, b->grid.ox, b->grid.oy, b->grid.oz))
                        throw FwiError(FWI_ERR_ARG, "a DAS channel has its gauge length falling outside subsurface "
                                                    "model boundaries");
            }
            batch_tables(*b, all, ext);
            b->eng->join_shot(slot, all, ext, b->it);
            if (b->par.gl > 0) b->eng->set_das(das_weights(b->rxyz.data(), 0, b->nshots, b->nr), b->nr, b->par.gl);
        } catch (...) {
            b->sxyz = s0;  // the slot keeps its shot
            b->rxyz = r0;
            throw;
        }
        b->t0[slot] = b->it;
    });
}

int fwi_batch_release(fwi_batch *b, int slot)
{
    if (!b || slot < 0 || slot >= b->nshots) return fail(FWI_ERR_ARG, "bad argument");
    return guarded([&] { b->eng->release_shot(slot); });
}

int fwi_batch_slot_time(const fwi_batch *b, int slot, int *t0, int *remaining)
{
    if (!b || slot < 0 || slot >= b->nshots) return fail(FWI_ERR_ARG, "bad argument");
    if (t0) *t0 = b->t0[slot];
    // the last sample (local nt-1) is read by the step run at t0 + nt - 1
    if (remaining) *remaining = std::max(0, b->t0[slot] + b->pb.nt - b->it);
    return FWI_OK;
}

int fwi_batch_slot_traces(fwi_batch *b, int slot, float *data)
{
    if (!b || !data || slot < 0 || slot >= b->nshots) return fail(FWI_ERR_ARG, "bad argument");
    return guarded([&] {
        if (!b->eng->continuous()) throw FwiError(FWI_ERR_STATE, "slot traces need a batch with shot slots");
        if (b->it < b->t0[slot] + b->pb.nt) throw FwiError(FWI_ERR_STATE, "the slot's time axis has not been run to the end");
        if (batch_device_output(*b, slot, 1, data)) return;
        std::vector<float> rcv((size_t)b->nrcomp * b->nr * b->pb.nt);
        if (b->par.gl > 0) b->eng->copy_strain(slot, 1, rcv.data());  // strain along the fibres, on the device
        else b->eng->copy_shot_traces(slot, rcv.data());
        batch_shot_output(*b, rcv.data(), data);
    });
}

int fwi_batch_sync(fwi_batch *b)
{
    if (!b) return fail(FWI_ERR_ARG, "null batch");
    return guarded([&] { b->eng->sync(); });
}

int fwi_batch_ready(fwi_batch *b, int *ready)
{
    if (!b || !ready) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] {
        const cudaError_t e = cudaStreamQuery((cudaStream_t)b->eng->stream());
        if (e == cudaErrorNotReady) {
            *ready = 0;
            return;
        }
        if (e != cudaSuccess) throw FwiError(FWI_ERR_CUDA, cudaGetErrorString(e));
        b->eng->sync();  // idle: surfaces the kernels' error flags
        *ready = 1;
    });
}

int fwi_batch_stream(fwi_batch *b, void **stream)
{
    if (!b || !stream) return fail(FWI_ERR_ARG, "null argument");
    *stream = b->eng->stream();
    return FWI_OK;
}

int fwi_batch_traces(fwi_batch *b, float *data)
{
    if (!b || !data) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] {
        if (b->eng->continuous()) throw FwiError(FWI_ERR_STATE, "a batch with shot slots returns traces per slot");
        if (b->it != b->pb.nt - 1) throw FwiError(FWI_ERR_STATE, "the time axis has not been run to the end");
        b->eng->extract_last();
        if (batch_device_output(*b, 0, b->nshots, data)) return;
        const int nt = b->pb.nt;
        const int ntr = b->nrcomp * b->nr;
        std::vector<float> rcv((size_t)b->nshots * ntr * nt);
        if (b->par.gl > 0) b->eng->copy_strain(0, b->nshots, rcv.data());  // strain along the fibres, on the device
        else b->eng->copy_traces(rcv.data());
        for (int s = 0; s < b->nshots; s++)
            batch_shot_output(*b, rcv.data() + (size_t)s * ntr * nt, data + (size_t)s * ntr * b->nt_data);
    });
}

int fwi_batch_get_info(const fwi_batch *b, fwi_op_info *info, int *launches)
{
    if (!b || !info) return fail(FWI_ERR_ARG, "null argument");
    info->dt = b->pb.dt;
    info->nt = b->pb.nt;
    info->sub = 0;
    info->nscomp = b->nscomp;
    info->nrcomp = b->nrcomp;
    info->nr = b->nr;
    info->device_bytes = b->eng->device_bytes();
    if (launches) *launches = b->eng->launches_per_step();
    return FWI_OK;
}

void fwi_batch_destroy(fwi_batch *b) { delete b; }

int fwi_forward_batch(int device, const fwi_grid *grid, int nmodels, const fwi_param *par, const float *model,
                      const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data, int nshots,
                      const float *sxyz, int nr, const float *rxyz, float *data)
{
    fwi_batch *b = nullptr;
    int rc = fwi_batch_create(&b, device, grid, nmodels, par, model, wavelet, wavelet_ncomp, nt_data, dt_data, nshots,
                              sxyz, nr, rxyz);
    if (rc != FWI_OK) return rc;
    PhaseClock clk;
    rc = fwi_batch_reset(b);
    clk.mark("reset (+ graph capture)");
    if (rc == FWI_OK) rc = fwi_batch_run(b, b->pb.nt - 1);
    if (rc == FWI_OK) rc = fwi_batch_sync(b);
    clk.mark("time steps");
    if (rc == FWI_OK) rc = fwi_batch_traces(b, data);
    clk.mark("traces (copy + host)");
    fwi_batch_destroy(b);
    clk.mark("destroy");
    return rc;
}

int fwi_batch_time_main_kernel(fwi_batch *b, int max_launches)
{
    if (!b || max_launches < 0) return fail(FWI_ERR_ARG, "bad argument");
    return guarded([&] { b->eng->time_main_kernel(max_launches); });
}

int fwi_batch_main_kernel_time(fwi_batch *b, double *ms, int *launches, int64_t *points, const char **name)
{
    if (!b || !ms) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] { *ms = b->eng->main_kernel_ms(launches, points, name); });
}

int fwi_objective_create(fwi_objective **out, int device, const fwi_grid *grid, int nmodels, const fwi_param *par,
                         const float *wavelet, int wavelet_ncomp, int nt_data, float dt_data, int nshots,
                         const float *sxyz, int nr, const float *rxyz, const float *observed, int normalize, int batch)
{
    if (!out || !grid || !par || !wavelet || !sxyz || !rxyz || !observed || nshots < 1 || nr < 1)
        return fail(FWI_ERR_ARG, "null argument, no shot or no receiver");
    *out = nullptr;
    if (nmodels != 2 && nmodels != 3 && nmodels != 6)
        return fail(FWI_ERR_ARG, "The model must contain 2, 3, or 6 parameters");
    if (grid->nx < 12 || grid->ny < 12 || grid->nz < 12) return fail(FWI_ERR_ARG, "each grid axis needs at least 12 points");
    if (nt_data < 2 || !(dt_data > 0)) return fail(FWI_ERR_ARG, "the wavelet needs at least 2 samples and dt > 0");
    return guarded([&] {
        std::unique_ptr<fwi_objective> o(new fwi_objective());
        o->device = device;
        o->grid = *grid;
        o->nmodels = nmodels;
        o->par = *par;
        if (nmodels == 2) o->par.mt = 0;
        o->nt_data = nt_data;
        o->dt_data = dt_data;
        o->nshots = nshots;
        o->nr = nr;
        o->nscomp = nmodels == 2 ? 1 : (o->par.mt ? 6 : 3);
        if (nmodels == 2) o->par.gl = 0.f;  // analyzeGeometry, we_op.cpp:11-14
        o->nrcomp = nmodels == 2 ? 1 : (o->par.gl > 0 ? 1 : 3);  // DAS: strain along each fibre
        if (o->par.gl > 0)
            for (int s = 0; s < nshots; s++)
                for (const Loc5 &l : shot_fibres(rxyz, s, nr))
                    if (!dipole_inside(l, o->par.gl, grid->nx, grid->ny, grid->nz, grid->dx, grid->dy, grid->dz,
                                       grid->ox, grid->oy, grid->oz))
                        throw FwiError(FWI_ERR_ARG, "a DAS channel has its gauge length falling outside subsurface "
                                                    "model boundaries");
        o->batch = batch < 1 ? nshots : std::min(batch, nshots);
        o->wavelet = expand_wavelet(wavelet, wavelet_ncomp, nt_data, nmodels, o->par);
        o->sxyz.assign(sxyz, sxyz + 3 * nshots);
        o->rxyz.assign(rxyz, rxyz + (size_t)5 * nr * nshots);
        const size_t nd = (size_t)nshots * o->nrcomp * nr * nt_data;
        o->observed.assign(observed, observed + nd);
        if (!finite_all(observed, (int64_t)nd)) throw FwiError(FWI_ERR_NAN, "observed data contain non-finite values");
        o->normalize = normalize;
        o->dnorm = data_norm(*o);
        *out = o.release();
    });
}

int fwi_objective_set_shots(fwi_objective *o, const float *sxyz, const float *rxyz, const float *observed)
{
    if (!o || !sxyz || !rxyz || !observed) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] {
        const size_t nd = o->observed.size();
        if (!finite_all(observed, (int64_t)nd)) throw FwiError(FWI_ERR_NAN, "observed data contain non-finite values");
        o->sxyz.assign(sxyz, sxyz + o->sxyz.size());
        o->rxyz.assign(rxyz, rxyz + o->rxyz.size());
        o->observed.assign(observed, observed + nd);
        o->dnorm = data_norm(*o);
    });
}

// The objective of all shots (f, grad: summed over the shots, residual
// optional) or, with gs, one objective per shot: fs [nshots] and gs
// [nshots][nm][nxyz], each normalised by its own data.
static void objective_eval(fwi_objective *o, const float *model, double *f, float *grad, float *residual, double *fs,
                           float *gs)
{
    {
        const bool per_shot = gs != nullptr;
        const fwi_grid &g = o->grid;
        const int64_t n = (int64_t)g.nx * g.ny * g.nz;
        const int nm = std::min(3, o->nmodels);
        if (!finite_all(model, o->nmodels * n)) throw FwiError(FWI_ERR_NAN, "model contains non-finite values");
        std::vector<float> m(model, model + o->nmodels * n);
        fwi_param par = o->par;
        TimeAxis ta = analyze_model(m, o->nmodels, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, o->nt_data, o->dt_data, par);
        if (ta.sub < 1) ta.sub = std::max(1, (int)std::lround((double)(o->dt_data / ta.dt)));
        convert_model(m, o->nmodels, n);
        Problem p{};
        p.nmodels = o->nmodels;
        p.nx = g.nx;
        p.ny = g.ny;
        p.nz = g.nz;
        p.dx = g.dx;
        p.dy = g.dy;
        p.dz = g.dz;
        p.dt = ta.dt;
        p.nt = ta.nt;
        p.sub = ta.sub;
        for (int k = 0; k < 6; k++) p.bc[k] = std::max(0, par.bc[k]);
        std::memcpy(p.taper, par.taper, sizeof(p.taper));
        p.taper_strength = par.taper_strength;
        p.free_surface_stiffness =
            o->nmodels == 2 ? std::max(par.free_surface_stiffness, 1.0f) : par.free_surface_stiffness;
        const int nt = p.nt, ntd = o->nt_data;
        const int ncr = p.ncomp();
        const int ntr = o->nrcomp * o->nr;  // data traces of a shot
        const int ntr_raw = ncr * o->nr;    // extracted rows of a shot (DAS: the dipoles' three components)
        const bool das = par.gl > 0;
        const bool sinc = par.resampling_linear == 0;
        const float alpha = p.dt / o->dt_data;
        // wavelet at the propagation sampling (same for every shot)
        std::vector<float> w1((size_t)o->nscomp * nt);
        resample_forward(sinc, par.sinc_half_length, o->wavelet.data(), ntd, o->dt_data, w1.data(), nt, p.dt, o->nscomp);
        std::vector<double> gsum(per_shot ? 0 : (size_t)nm * n, 0.0);
        std::vector<double> fshot(o->nshots, 0.0);
        double fsum = 0.0;
        o->device_bytes = 0;
        // FWI_OBJ_TIMING=1: per-batch phase times on stderr (host clock)
        const char *tenv = std::getenv("FWI_OBJ_TIMING");
        const bool timing = tenv && tenv[0] == '1';
        auto now = [] { return std::chrono::steady_clock::now(); };
        auto secs = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double>(b - a).count();
        };
        // Residual on the device (sinc resampling, traces that fit in shared
        // memory; FWI_HOST_RESIDUAL=1 keeps the host path)
        const char *hre = std::getenv("FWI_HOST_RESIDUAL");
        const bool on_device = sinc && std::max(nt, ntd) <= kResidualMaxSamples && !(hre && hre[0] == '1');
        if (on_device) {
            o->dres.set_observed(o->device, o->observed);
            o->dres.set_axes(par.sinc_half_length, ntd, o->dt_data, nt, p.dt);
        }
        for (int s0 = 0; s0 < o->nshots; s0 += o->batch) {
            const auto t0 = now();
            const int B = std::min(o->batch, o->nshots - s0);
            p.nshots = B;
            auto &eng = o->eng[B];
            const bool same = eng && o->pb.nt == p.nt && o->pb.dt == p.dt && o->pb.sub == p.sub;
            if (!same) eng.reset(new Engine(o->device, p));
            eng->set_storage(par.snapshot_storage);
            eng->set_snapshot_budget((int64_t)((double)par.snapshot_budget_gb * 1e9));
            eng->set_checkpointing(par.checkpoint_slots, par.checkpoint_precision);
            eng->set_per_shot_gradient(per_shot);
            eng->set_model(m.data());
            // tables of the batch (shot b of the batch at wavefield offset b)
            InjTable inj, adj;
            ExtTable ext;
            ext.nrec = B * o->nr;
            std::vector<float> src((size_t)B * o->nscomp * nt);
            for (int b = 0; b < B; b++) {
                const int sh = s0 + b;
                std::memcpy(src.data() + (size_t)b * w1.size(), w1.data(), sizeof(float) * w1.size());
                const float *sx = &o->sxyz[3 * sh];
                PointOp pi = make_delta(p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, g.ox, g.oy, g.oz, {Loc{sx[0], sx[1], sx[2]}},
                                        par.mt != 0);
                InjTable t = injection_table(pi, p.nx, p.ny, p.nz, ncr);
                std::vector<Loc> rl(o->nr);
                const float *rs = &o->rxyz[(size_t)5 * o->nr * sh];
                for (int r = 0; r < o->nr; r++) rl[r] = Loc{rs[5 * r], rs[5 * r + 1], rs[5 * r + 2]};
                PointOp pr = make_delta(p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, g.ox, g.oy, g.oz, rl, false);
                InjTable ta2;
                ExtTable e;
                if (das) {
                    // the channels' dipoles (dipole_m3, injector.cpp:313-493; we_op.cpp:1015)
                    const Dipole dp = make_dipole(p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, g.ox, g.oy, g.oz,
                                                  shot_fibres(o->rxyz.data(), sh, o->nr), par.gl);
                    ta2 = dipole_injection_table(dp, p.nx, p.ny, p.nz, ncr);
                    e = dipole_extraction_table(dp, p.nx, p.ny, p.nz);
                } else {
                    ta2 = injection_table(pr, p.nx, p.ny, p.nz, ncr);
                    e = extraction_table(pr, p.nx, p.ny, p.nz);
                }
                ext.ntap = e.ntap;
                for (int c = 0; c < ncr; c++) {
                    for (size_t k = 0; k < t.gidx[c].size(); k++) {
                        inj.gidx[c].push_back(t.gidx[c][k] + b * n);
                        inj.trace[c].push_back(t.trace[c][k] + b * o->nscomp);
                        inj.w[c].push_back(t.w[c][k]);
                    }
                    for (size_t k = 0; k < ta2.gidx[c].size(); k++) {
                        adj.gidx[c].push_back(ta2.gidx[c][k] + b * n);
                        adj.trace[c].push_back(ta2.trace[c][k] + b * ntr_raw);
                        adj.w[c].push_back(ta2.w[c][k]);
                    }
                }
                for (auto gi : e.gidx) ext.gidx.push_back(gi + b * n);
                ext.w.insert(ext.w.end(), e.w.begin(), e.w.end());
            }
            if (das) eng->set_das(das_weights(o->rxyz.data(), s0, B, o->nr), o->nr, par.gl);
            const auto t1 = now();
            if (on_device) {
                eng->forward(inj, B * o->nscomp, src.data(), ext, nullptr, true);
                // DAS: strain along the fibres, on the device (we_op.cpp:929)
                const float *strain = das ? eng->strain_traces(0, B) : nullptr;
                const auto t2 = now();
                const size_t ntrb = (size_t)B * ntr;
                nvtxRangePushA("fwi3d residual");
                std::vector<double> pt(ntrb);
                fsum += o->dres.run(*eng, (size_t)s0 * ntr * ntd, (int)ntrb, par.seismotype, alpha,
                                    residual ? residual + (size_t)s0 * ntr * ntd : nullptr, pt.data(), strain);
                nvtxRangePop();
                for (int b = 0; b < B; b++)
                    for (int tr = 0; tr < ntr; tr++) fshot[s0 + b] += pt[(size_t)b * ntr + tr];
                std::vector<float> gb((size_t)(per_shot ? B : 1) * nm * n);
                const auto t3 = now();
                if (das) {
                    // strain sources back to the dipoles' three components (we_op.cpp:1015)
                    eng->adjoint_dev(adj, B * ntr_raw, eng->strain_adjoint(o->dres.adjoint_sources()), gb.data());
                } else {
                    eng->adjoint_dev(adj, (int)ntrb, o->dres.adjoint_sources(), gb.data());
                }
                const auto t4 = now();
                if (per_shot) std::copy(gb.begin(), gb.end(), gs + (size_t)s0 * nm * n);
                else
                    for (size_t i = 0; i < gb.size(); i++) gsum[i] += gb[i];
                if (timing)
                    std::fprintf(stderr,
                                 "objective batch %d: prep %.3f s, forward %.3f s, device residual %.3f s, adjoint %.3f s\n",
                                 s0 / o->batch, secs(t0, t1), secs(t1, t2), secs(t2, t3), secs(t3, t4));
                o->device_bytes = std::max(o->device_bytes, eng->device_bytes());
                o->pb = p;
                continue;
            }
            std::vector<float> rcv((size_t)B * ntr_raw * nt);
            eng->forward(inj, B * o->nscomp, src.data(), ext, rcv.data(), true);
            const auto t2 = now();
            if (!finite_all(rcv.data(), (int64_t)rcv.size())) throw FwiError(FWI_ERR_NAN, "non-finite values in the traces");
            const auto tr0 = now();
            double t_ra = 0, t_rf = 0;
            std::vector<float> asrc((size_t)B * ntr_raw * nt);
            std::vector<float> syn((size_t)ntr * ntd), tmp;
            for (int b = 0; b < B; b++) {
                const int sh = s0 + b;
                float *r = rcv.data() + (size_t)b * ntr_raw * nt;
                if (das) {
                    // strain along the fibres into component 0 (we_op.cpp:929)
                    std::vector<float> dip(o->nr), az(o->nr);
                    for (int q = 0; q < o->nr; q++) {
                        dip[q] = o->rxyz[((size_t)sh * o->nr + q) * 5 + 3];
                        az[q] = o->rxyz[((size_t)sh * o->nr + q) * 5 + 4];
                    }
                    dipole_to_strain(false, r, dip.data(), az.data(), o->nr, nt, par.gl);
                }
                if (par.seismotype == 1) {
                    tmp.resize((size_t)ntr * nt);
                    apply_dt(false, r, tmp.data(), ntr, nt, p.dt);
                    std::memcpy(r, tmp.data(), sizeof(float) * tmp.size());
                }
                for (size_t i = 0; i < (size_t)ntr * nt; i++) r[i] *= alpha;
                std::fill(syn.begin(), syn.end(), 0.f);
                const auto ta0 = now();
                resample_adjoint(sinc, par.sinc_half_length, syn.data(), ntd, o->dt_data, r, nt, p.dt, ntr);
                t_ra += secs(ta0, now());
                // residual and misfit (optimization.cpp:111-115, optimization.hpp:410-424), FP64 sums
                const float *obs = &o->observed[(size_t)sh * ntr * ntd];
                for (size_t i = 0; i < syn.size(); i++) syn[i] -= obs[i];
                double ss = 0;
                for (size_t i = 0; i < syn.size(); i++) ss += (double)syn[i] * syn[i];
                for (int tr = 0; tr < ntr; tr++) {
                    const double a0 = syn[(size_t)tr * ntd], a1 = syn[(size_t)tr * ntd + ntd - 1];
                    ss -= 0.5 * (a0 * a0 + a1 * a1);
                }
                fsum += ss;
                fshot[sh] = ss;
                if (residual) std::memcpy(residual + (size_t)sh * ntr * ntd, syn.data(), sizeof(float) * syn.size());
                // adjoint sources: Ht(r) (optimization.cpp:118), then jacobianT's data path (we_op.cpp:994-1003)
                apply_ht(false, syn.data(), syn.data(), ntr, ntd, o->dt_data);
                float *as = asrc.data() + (size_t)b * ntr_raw * nt;
                const auto tf0 = now();
                resample_forward(sinc, par.sinc_half_length, syn.data(), ntd, o->dt_data, as, nt, p.dt, ntr);
                t_rf += secs(tf0, now());
                apply_ht(true, as, as, ntr, nt, p.dt);
                for (int tr = 0; tr < ntr; tr++) std::reverse(as + (size_t)tr * nt, as + (size_t)(tr + 1) * nt);
                for (size_t i = 0; i < (size_t)ntr * nt; i++) as[i] *= -alpha;
                if (par.seismotype == 1) {
                    tmp.resize((size_t)ntr * nt);
                    apply_dt(true, as, tmp.data(), ntr, nt, p.dt);
                    std::memcpy(as, tmp.data(), sizeof(float) * tmp.size());
                }
                if (das) {
                    // strain sources back to the dipoles' three components (we_op.cpp:1015)
                    std::vector<float> dip(o->nr), az(o->nr);
                    for (int q = 0; q < o->nr; q++) {
                        dip[q] = o->rxyz[((size_t)sh * o->nr + q) * 5 + 3];
                        az[q] = o->rxyz[((size_t)sh * o->nr + q) * 5 + 4];
                    }
                    dipole_to_strain(true, as, dip.data(), az.data(), o->nr, nt, par.gl);
                }
            }
            std::vector<float> gb((size_t)(per_shot ? B : 1) * nm * n);
            const auto t3 = now();
            eng->adjoint(adj, B * ntr_raw, asrc.data(), gb.data());
            const auto t4 = now();
            if (per_shot) std::copy(gb.begin(), gb.end(), gs + (size_t)s0 * nm * n);
            else
                for (size_t i = 0; i < gb.size(); i++) gsum[i] += gb[i];
            if (timing)
                std::fprintf(stderr,
                             "objective batch %d: prep %.3f s, forward %.3f s, residual %.3f s (check %.3f, "
                             "resample adj %.3f fwd %.3f; nt %d ntd %d ntr %d), adjoint %.3f s\n",
                             s0 / o->batch, secs(t0, t1), secs(t1, t2), secs(t2, t3), secs(t2, tr0), t_ra, t_rf, nt,
                             ntd, ntr, secs(t3, t4));
            o->device_bytes = std::max(o->device_bytes, eng->device_bytes());
            o->pb = p;
        }
        // H quadrature, chain rule to (vp, vs, rho), 1/dnorm (we_op.cpp:1027-1067, optimization.cpp:194)
        if (f) *f = 0.5 * o->dt_data * fsum / o->dnorm;
        if (per_shot) {
            for (int sh = 0; sh < o->nshots; sh++) {
                float *gsh = gs + (size_t)sh * nm * n;
                for (int q = 0; q < nm; q++) apply_h3(gsh + q * n, p.nx, p.ny, p.nz, p.dx, p.dy, p.dz);
                gradient_to_velocity(gsh, m.data(), o->nmodels, n);
                const double dn = data_norm(*o, sh);
                const float sc = (float)(1.0 / dn);
                for (int64_t i = 0; i < nm * n; i++) gsh[i] *= sc;
                fs[sh] = 0.5 * o->dt_data * fshot[sh] / dn;
            }
            if (!finite_all(gs, (int64_t)o->nshots * nm * n))
                throw FwiError(FWI_ERR_NAN, "non-finite values in the gradient");
            return;
        }
        for (int64_t i = 0; i < nm * n; i++) grad[i] = (float)gsum[i];
        for (int q = 0; q < nm; q++) apply_h3(grad + q * n, p.nx, p.ny, p.nz, p.dx, p.dy, p.dz);
        gradient_to_velocity(grad, m.data(), o->nmodels, n);
        const float sc = (float)(1.0 / o->dnorm);
        for (int64_t i = 0; i < nm * n; i++) grad[i] *= sc;
        if (!finite_all(grad, nm * n)) throw FwiError(FWI_ERR_NAN, "non-finite values in the gradient");
    }
}

int fwi_objective_evaluate(fwi_objective *o, const float *model, double *f, float *grad, float *residual)
{
    if (!o || !model || !f || !grad) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] { objective_eval(o, model, f, grad, residual, nullptr, nullptr); });
}

int fwi_objective_evaluate_shots(fwi_objective *o, const float *model, double *f, float *grad)
{
    if (!o || !model || !f || !grad) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] { objective_eval(o, model, nullptr, nullptr, nullptr, f, grad); });
}

int64_t fwi_objective_device_bytes(const fwi_objective *o) { return o ? o->device_bytes : 0; }

void fwi_objective_destroy(fwi_objective *o) { delete o; }

int fwi_elastic_step_static(const fwi_grid *grid, int nmodels, const int *bc, float dt, const float *model,
                            const float *prev, const float *curr, float *next, void *stream)
{
    if (!grid || !bc || !model || !prev || !curr || !next) return fail(FWI_ERR_ARG, "null argument");
    return guarded([&] { fwi::static_elastic_step(*grid, nmodels, bc, dt, model, prev, curr, next, stream); });
}

}  // extern "C"
