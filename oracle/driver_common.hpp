/*
 * oracle/driver_common.hpp -- shared by the oracle's C-ABI drivers
 * (ref_driver.cpp, refside_driver.cpp): the parameter struct of the ctypes
 * binding and its translation into the reference's `param`, hypercube and
 * wavelet vector.  TEST INFRASTRUCTURE ONLY.
 */
#pragma once

#include <memory>
#include <vector>

#include "we_op.hpp"

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

}  // extern "C"

namespace oracle_common {

inline void fill_param(const oracle_param *p, int nr, const float *sxyz, const float *rxyz, param &par)
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

inline hypercube<data_t> model_hyper(const oracle_param *p)
{
    axis<data_t> Z(p->nz, p->oz, p->dz), X(p->nx, p->ox, p->dx), Y(p->ny, p->oy, p->dy);
    axis<data_t> C(p->nmodels, 0, 1);
    return hypercube<data_t>(Z, X, Y, C);
}

/* Wavelet: wavelet_ncomp==1 -> 1-D input duplicated by analyzeWavelet
 * (we_op.cpp:138-214); otherwise [ncomp][nt] used as given. */
inline std::shared_ptr<vecReg<data_t> > make_wavelet(const oracle_param *p, const float *w, int ncomp)
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

}  // namespace oracle_common
