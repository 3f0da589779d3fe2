/*
 * oracle/ref_driver.cpp -- C-ABI driver over the UNMODIFIED reference library
 * (nmbader/fwi3d src/cpp/{we_op,spatial_operators,injector,param,misc,operator}.cpp),
 * compiled from the reference tree by oracle/Makefile into oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * the library it builds.
 *
 * The call sequence mirrors the reference's own drivers:
 *   modeling  : src/main/we_modeling.cpp:35-90  (analyzeGeometry, analyzeWavelet,
 *               new nl_we_op_{a,e,vti}(hyper, allsrc, s, par), op->forward)
 *   gradient  : src/cpp/optimization.cpp:41-50,181 (apply_forward on a fresh
 *               per-shot op, then apply_jacobianT(add=true, ...) on the same op,
 *               which consumes the snapshots the forward pass stored)
 * data_t is float in the FP32 build and double with -DDOUBLE_PRECISION; inputs
 * are float and outputs double in both builds so one ctypes binding serves both.
 */
#include <cstdio>
#include <cstring>
#include <vector>
#include <memory>
#include <exception>
#include <omp.h>
#include "we_op.hpp"
#include "misc.hpp"

extern "C" {

/* Mirrors the subset of `struct param` (src/include/param.hpp:8-71) that the
 * propagation path reads.  Field meaning and defaults follow param.hpp. */
typedef struct oracle_param {
    int nmodels;                 /* 2 acoustic (vp,rho), 3 elastic (vp,vs,rho), 6 VTI */
    int nx, ny, nz;
    float ox, oy, oz, dx, dy, dz;
    int nt_data;                 /* samples of the wavelet / data time axis */
    float dt_data;
    float courant, dt;           /* param.hpp:12 (dt=-1: CFL-derived) */
    int sub;                     /* param.hpp:11 (0: no snapshots; -1: derived) */
    int resampling_linear;       /* 0 sinc, 1 linear */
    int sinc_half_length;
    int mt;
    float fangle, fazimuth;
    float mxx, myy, mzz, mxy, mxz, myz;
    int seismotype;
    float gl;
    int bc[6];                   /* top, bottom, left, right, front, back */
    int taper[6];
    float free_surface_stiffness, taper_strength;
    float vpmin, vpmax, vsmin, vsmax, rhomin, rhomax;
    float deltamin, deltamax, epsilonmin, epsilonmax, gammamin, gammamax;
    int soft_clip;
    int verbose;
    int nthreads;
} oracle_param;

typedef struct oracle_info {
    double dt;         /* propagation time step chosen by analyzeModel */
    int nt;            /* propagation steps + 1 */
    int sub;
    double courant;
    int nscomp, nrcomp;
} oracle_info;

int oracle_data_t_size(void) { return (int)sizeof(data_t); }

}  // extern "C"

namespace {

void fill_param(const oracle_param *p, int nr, const float *sxyz, const float *rxyz, param &par)
{
    par.courant = p->courant;
    par.dt = p->dt;
    par.sub = p->sub;
    par.resampling = p->resampling_linear ? "linear" : "sinc";
    par.sinc_half_length = p->sinc_half_length;
    par.mt = p->mt != 0;
    par.fangle = p->fangle;
    par.fazimuth = p->fazimuth;
    par.mxx = p->mxx; par.myy = p->myy; par.mzz = p->mzz;
    par.mxy = p->mxy; par.mxz = p->mxz; par.myz = p->myz;
    par.seismotype = p->seismotype;
    par.gl = p->gl;
    par.bc_top = p->bc[0]; par.bc_bottom = p->bc[1]; par.bc_left = p->bc[2];
    par.bc_right = p->bc[3]; par.bc_front = p->bc[4]; par.bc_back = p->bc[5];
    par.taper_top = p->taper[0]; par.taper_bottom = p->taper[1]; par.taper_left = p->taper[2];
    par.taper_right = p->taper[3]; par.taper_front = p->taper[4]; par.taper_back = p->taper[5];
    par.free_surface_stiffness = p->free_surface_stiffness;
    par.taper_strength = p->taper_strength;
    par.vpmin = p->vpmin; par.vpmax = p->vpmax; par.vsmin = p->vsmin; par.vsmax = p->vsmax;
    par.rhomin = p->rhomin; par.rhomax = p->rhomax;
    par.deltamin = p->deltamin; par.deltamax = p->deltamax;
    par.epsilonmin = p->epsilonmin; par.epsilonmax = p->epsilonmax;
    par.gammamin = p->gammamin; par.gammamax = p->gammamax;
    par.soft_clip = p->soft_clip != 0;
    par.verbose = p->verbose;
    par.nthreads = p->nthreads;
    par.ns = 1;
    par.sxyz = {{(data_t)sxyz[0], (data_t)sxyz[1], (data_t)sxyz[2]}};
    std::vector<std::vector<data_t> > rec(nr);
    for (int r = 0; r < nr; r++)
        rec[r] = {(data_t)rxyz[5 * r], (data_t)rxyz[5 * r + 1], (data_t)rxyz[5 * r + 2],
                  (data_t)rxyz[5 * r + 3], (data_t)rxyz[5 * r + 4]};
    par.rxyz = {rec};
    par.nr = nr;
}

hypercube<data_t> model_hyper(const oracle_param *p)
{
    axis<data_t> Z(p->nz, p->oz, p->dz), X(p->nx, p->ox, p->dx), Y(p->ny, p->oy, p->dy);
    axis<data_t> C(p->nmodels, 0, 1);
    return hypercube<data_t>(Z, X, Y, C);
}

/* Wavelet: wavelet_ncomp==1 -> 1-D input duplicated by analyzeWavelet
 * (we_op.cpp:138-214); otherwise [ncomp][nt] used as given. */
std::shared_ptr<vecReg<data_t> > make_wavelet(const oracle_param *p, const float *w, int ncomp)
{
    axis<data_t> T(p->nt_data, 0, p->dt_data);
    std::shared_ptr<vecReg<data_t> > src;
    if (ncomp == 1) {
        src = std::make_shared<vecReg<data_t> >(hypercube<data_t>(T));
    } else {
        axis<data_t> C(ncomp, 0, 1), S(1, 0, 1);
        src = std::make_shared<vecReg<data_t> >(hypercube<data_t>(T, C, S));
    }
    data_t *ps = src->getVals();
    for (long i = 0; i < (long)ncomp * p->nt_data; i++) ps[i] = (data_t)w[i];
    return src;
}

nl_we_op_e *make_op(const hypercube<data_t> &hyp, std::shared_ptr<vecReg<data_t> > allsrc, param &par)
{
    if (par.nmodels == 2) return new nl_we_op_a(hyp, allsrc, 0, par);
    if (par.nmodels == 3) return new nl_we_op_e(hyp, allsrc, 0, par);
    return new nl_we_op_vti(hyp, allsrc, 0, par);
}

void fill_info(const nl_we_op_e *op, oracle_info *info)
{
    if (!info) return;
    info->dt = op->_par.dt;
    info->nt = op->_par.nt;
    info->sub = op->_par.sub;
    info->courant = op->_par.courant;
    info->nscomp = op->_par.nscomp;
    info->nrcomp = op->_par.nrcomp;
}

}  // namespace

extern "C" {

/* One shot of WE_MODELING_3D: returns data [nrcomp][nr][nt_data] (double). */
int oracle_modeling(const oracle_param *p, const float *model, const float *wavelet, int wavelet_ncomp,
                    const float *sxyz, int nr, const float *rxyz, double *data, oracle_info *info)
{
    try {
        if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
        param par;
        fill_param(p, nr, sxyz, rxyz, par);
        hypercube<data_t> hyp = model_hyper(p);
        analyzeGeometry(hyp, par, false);
        std::shared_ptr<vecReg<data_t> > src = make_wavelet(p, wavelet, wavelet_ncomp);
        std::shared_ptr<vecReg<data_t> > allsrc = analyzeWavelet(src, par, false);
        std::unique_ptr<nl_we_op_e> op(make_op(hyp, allsrc, par));
        std::shared_ptr<vecReg<data_t> > mod = std::make_shared<vecReg<data_t> >(hyp);
        data_t *pm = mod->getVals();
        for (long i = 0; i < hyp.getN123(); i++) pm[i] = (data_t)model[i];
        std::shared_ptr<vecReg<data_t> > rcv = std::make_shared<vecReg<data_t> >(*op->getRange());
        rcv->zero();
        op->forward(false, mod, rcv);
        const data_t *pr = rcv->getCVals();
        for (long i = 0; i < rcv->getN123(); i++) data[i] = (double)pr[i];
        fill_info(op.get(), info);
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "oracle_modeling: %s\n", e.what());
        return -1;
    }
}

/* apply_forward followed by apply_jacobianT on the same per-shot operator
 * (optimization.cpp:50,181).  `adj_data` [nrcomp][nr][nt_data] is the data-side
 * vector the adjoint consumes (e.g. Ht applied residual); `grad` receives
 * [min(3,nmodels)][nxyz] with add=false semantics.  `syn` (optional) receives the
 * forward data. */
int oracle_forward_jacobianT(const oracle_param *p, const float *model, const float *wavelet, int wavelet_ncomp,
                             const float *sxyz, int nr, const float *rxyz, const float *adj_data,
                             double *syn, double *grad, oracle_info *info)
{
    try {
        if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
        param par;
        fill_param(p, nr, sxyz, rxyz, par);
        hypercube<data_t> hyp = model_hyper(p);
        analyzeGeometry(hyp, par, false);
        std::shared_ptr<vecReg<data_t> > src = make_wavelet(p, wavelet, wavelet_ncomp);
        std::shared_ptr<vecReg<data_t> > allsrc = analyzeWavelet(src, par, false);
        std::unique_ptr<nl_we_op_e> op(make_op(hyp, allsrc, par));
        std::vector<data_t> m((size_t)hyp.getN123());
        for (size_t i = 0; i < m.size(); i++) m[i] = (data_t)model[i];
        long nd = op->getRange()->getN123();
        std::vector<data_t> d((size_t)nd, 0), a((size_t)nd);
        op->apply_forward(false, m.data(), d.data());
        if (syn) for (long i = 0; i < nd; i++) syn[i] = (double)d[i];
        for (long i = 0; i < nd; i++) a[i] = (data_t)adj_data[i];
        long nxyz = (long)p->nx * p->ny * p->nz;
        int nm = std::min(3, par.nmodels);
        std::vector<data_t> g((size_t)(nm * nxyz), 0);
        op->apply_jacobianT(false, g.data(), m.data(), a.data());
        for (long i = 0; i < nm * nxyz; i++) grad[i] = (double)g[i];
        fill_info(op.get(), info);
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "oracle_forward_jacobianT: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
