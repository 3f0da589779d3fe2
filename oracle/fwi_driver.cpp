/*
 * oracle/fwi_driver.cpp -- C-ABI driver over the UNMODIFIED reference FWI
 * objective and non-linear solvers (nmbader/fwi3d src/cpp/optimization.cpp,
 * src/cpp/nlsolver.cpp, src/include/optimization.hpp, nlsolver.hpp), compiled
 * with the propagation sources by oracle/Makefile into oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY: only tests/ load the library it builds.
 *
 * The set-up follows the reference's FWI program (src/main/fwi3d.cpp:72-79,
 * 247-253, 350-375): analyzeGeometry over all shots, analyzeWavelet, one
 * nl_we_op_{a,e,vti} on the model hypercube, the observed data on the range
 * (time axis, all traces of all shots), nlls_fwi(L, par, model, data) with no
 * model preconditioner (model_parameterization 1: vp, vs, rho), then either one
 * objective evaluation (res, getFunc, grad) or a solver run with the chosen
 * line search.  Inputs are float; outputs double (data_t is float in the FP32
 * build and double with -DDOUBLE_PRECISION).
 */
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <vector>
#include <omp.h>
#include "nlsolver.hpp"
#include "optimization.hpp"
#include "we_op.hpp"

extern "C" {

/* Propagation knobs: the same layout as ref_driver.cpp's oracle_param. */
typedef struct oracle_param {
    int nmodels;
    int nx, ny, nz;
    float ox, oy, oz, dx, dy, dz;
    int nt_data;
    float dt_data;
    float courant, dt;
    int sub;
    int resampling_linear;
    int sinc_half_length;
    int mt;
    float fangle, fazimuth;
    float mxx, myy, mzz, mxy, mxz, myz;
    int seismotype;
    float gl;
    int bc[6];
    int taper[6];
    float free_surface_stiffness, taper_strength;
    float vpmin, vpmax, vsmin, vsmax, rhomin, rhomax;
    float deltamin, deltamax, epsilonmin, epsilonmax, gammamin, gammamax;
    int soft_clip;
    int verbose;
    int nthreads;
} oracle_param;

/* Solver choice (param.hpp:55-63 names): solver 0 = objective and gradient
 * only, 1 lbfgs, 2 nlcg, 3 nlsd; lsearch 0 weak_wolfe, 1 regular_wolfe. */
typedef struct oracle_solver {
    int solver, lsearch, niter, max_trial;
    float threshold, ls_c1, ls_c2, ls_a0, ls_a1, ls_max_step;
    int ls_version, lbfgs_m, nlcg_method, normalize_obj_func;
} oracle_solver;

}  // extern "C"

namespace {

void fill_param(const oracle_param *p, int ns, const float *sxyz, int nr, const float *rxyz, param &par)
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
    par.ns = ns;
    par.sxyz.clear();
    par.rxyz.clear();
    for (int s = 0; s < ns; s++) {
        par.sxyz.push_back({(data_t)sxyz[3 * s], (data_t)sxyz[3 * s + 1], (data_t)sxyz[3 * s + 2]});
        std::vector<std::vector<data_t> > rec(nr);
        const float *r0 = rxyz + (size_t)s * nr * 5;
        for (int r = 0; r < nr; r++)
            rec[r] = {(data_t)r0[5 * r], (data_t)r0[5 * r + 1], (data_t)r0[5 * r + 2], (data_t)r0[5 * r + 3],
                      (data_t)r0[5 * r + 4]};
        par.rxyz.push_back(rec);
    }
}

}  // namespace

extern "C" {

/* The reference FWI objective on ns shots sharing the model, and optionally a
 * solver run.  obs: [ns][nrcomp][nr][nt_data].  Outputs: f_hist (niter+1
 * values; f_hist[0] the objective at the input model), nf (values written),
 * model_out [nmodels][nxyz] (the solver's final model), grad_out
 * [nmodels][nxyz] (the gradient at the last evaluated model), counts
 * {feval, geval}. */
int oracle_fwi(const oracle_param *p, const float *model, const float *wavelet, int wavelet_ncomp, int ns,
               const float *sxyz, int nr, const float *rxyz, const float *obs, const oracle_solver *sol,
               double *f_hist, int *nf, double *model_out, double *grad_out, int *counts)
{
    try {
        if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
        param par;
        fill_param(p, ns, sxyz, nr, rxyz, par);
        par.normalize_obj_func = sol->normalize_obj_func != 0;
        axis<data_t> Z(p->nz, p->oz, p->dz), X(p->nx, p->ox, p->dx), Y(p->ny, p->oy, p->dy), C(p->nmodels, 0, 1);
        hypercube<data_t> hyp(Z, X, Y, C);
        analyzeGeometry(hyp, par, false);
        axis<data_t> T(p->nt_data, 0, p->dt_data);
        std::shared_ptr<vecReg<data_t> > src;
        if (wavelet_ncomp == 1) {
            src = std::make_shared<vecReg<data_t> >(hypercube<data_t>(T));
        } else {
            axis<data_t> Cs(wavelet_ncomp, 0, 1), S(1, 0, 1);
            src = std::make_shared<vecReg<data_t> >(hypercube<data_t>(T, Cs, S));
        }
        for (long i = 0; i < (long)wavelet_ncomp * p->nt_data; i++) src->getVals()[i] = (data_t)wavelet[i];
        std::shared_ptr<vecReg<data_t> > allsrc = analyzeWavelet(src, par, false);
        analyzeNLInversion(par);
        std::unique_ptr<nl_we_op> L;
        if (par.nmodels == 2) L.reset(new nl_we_op_a(hyp, allsrc, 0, par));
        else if (par.nmodels == 3) L.reset(new nl_we_op_e(hyp, allsrc, 0, par));
        else L.reset(new nl_we_op_vti(hyp, allsrc, 0, par));
        axis<data_t> axR(par.nr * par.nrcomp, 0, 1);
        std::shared_ptr<vecReg<data_t> > data = std::make_shared<vecReg<data_t> >(hypercube<data_t>(T, axR));
        for (long i = 0; i < data->getN123(); i++) data->getVals()[i] = (data_t)obs[i];
        std::shared_ptr<vecReg<data_t> > m = std::make_shared<vecReg<data_t> >(hyp);
        for (long i = 0; i < hyp.getN123(); i++) m->getVals()[i] = (data_t)model[i];
        nlls_fwi prob(L.get(), par, m, data);
        int n = 0;
        if (sol->solver == 0) {
            prob.res();
            f_hist[n++] = (double)prob.getFunc();
            prob.grad();
            counts[0] = 1;
            counts[1] = 1;
        } else {
            lsearch *ls;
            if (sol->lsearch == 0) ls = new weak_wolfe(sol->ls_c1, sol->ls_a0, sol->ls_a1, sol->ls_version != 0);
            else
                ls = new regular_wolfe(sol->ls_c1, sol->ls_c2, sol->ls_a0, sol->ls_a1, sol->ls_max_step,
                                       sol->ls_version != 0);
            std::unique_ptr<nlsolver> solver;
            if (sol->solver == 1) solver.reset(new lbfgs(sol->niter, sol->max_trial, sol->threshold, ls, nullptr, sol->lbfgs_m));
            else if (sol->solver == 2) {
                nlcg *c = new nlcg(sol->niter, sol->max_trial, sol->threshold, ls);
                c->setMethod(sol->nlcg_method);
                solver.reset(c);
            } else {
                solver.reset(new nlsd(sol->niter, sol->max_trial, sol->threshold, ls));
            }
            delete ls;
            solver->run(&prob, false, "none");
            for (data_t v : solver->_func) f_hist[n++] = (double)v;
            counts[0] = (int)solver->getFeval();
            counts[1] = (int)solver->getGeval();
        }
        *nf = n;
        const data_t *pm = m->getCVals();
        const data_t *pg = prob.getGrad()->getCVals();
        for (long i = 0; i < hyp.getN123(); i++) {
            model_out[i] = (double)pm[i];
            grad_out[i] = (double)pg[i];
        }
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "oracle_fwi: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
