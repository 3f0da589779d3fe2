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

#include "driver_common.hpp"

extern "C" {
int oracle_data_t_size(void) { return (int)sizeof(data_t); }
}

namespace {
using namespace oracle_common;

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
