/*
 * oracle/refside_driver.cpp -- drives the reference-side GPU binding
 * (include/fwi3d_we_op_gpu.hpp) through the reference's own operator calls.
 *
 * TEST INFRASTRUCTURE ONLY: only tests/ load the library it builds
 * (oracle/_ref/librefside_gpu.so, linked with the reference's compiled
 * sources and with fwi3d_b200/libfwi3d_b200.so).
 *
 * One shot: the operator is the unmodified nl_we_op_{e,vti,a} (gpu = 0) or
 * its GPU subclass (gpu = 1), built with the reference's (domain, allsrc, s,
 * par) constructor after analyzeGeometry / analyzeWavelet as
 * src/main/we_modeling.cpp:35-90 does; then nl_we_op::forward and
 * nl_we_op::jacobianT (we_op.hpp:37-44) on vecReg vectors, as the reference's
 * callers use them (optimization.cpp:50, 181).
 */
#include <cstdio>
#include <exception>
#include <memory>
#include <omp.h>

#include "driver_common.hpp"
#include "fwi3d_we_op_gpu.hpp"

using namespace oracle_common;

extern "C" {

/* Forward traces [nrcomp][nr][nt_data] and, with adj non-null, the gradient
 * jacobianT(add=false, grad, model, adj) [nmodels][nxyz]. */
int refside_run(const oracle_param *p, int gpu, const float *model, const float *wavelet, int wavelet_ncomp,
                const float *sxyz, int nr, const float *rxyz, const float *adj, double *syn, double *grad)
{
    try {
        if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
        param par;
        fill_param(p, nr, sxyz, rxyz, par);
        hypercube<data_t> hyp = model_hyper(p);
        analyzeGeometry(hyp, par, false);
        std::shared_ptr<vecReg<data_t> > src = make_wavelet(p, wavelet, wavelet_ncomp);
        std::shared_ptr<vecReg<data_t> > allsrc = analyzeWavelet(src, par, false);
        std::unique_ptr<nl_we_op> op;
        if (par.nmodels == 2) op.reset(gpu ? (nl_we_op *)new nl_we_op_a_gpu(hyp, allsrc, 0, par) : new nl_we_op_a(hyp, allsrc, 0, par));
        else if (par.nmodels == 3) op.reset(gpu ? (nl_we_op *)new nl_we_op_e_gpu(hyp, allsrc, 0, par) : new nl_we_op_e(hyp, allsrc, 0, par));
        else op.reset(gpu ? (nl_we_op *)new nl_we_op_vti_gpu(hyp, allsrc, 0, par) : new nl_we_op_vti(hyp, allsrc, 0, par));
        std::shared_ptr<vecReg<data_t> > mod = std::make_shared<vecReg<data_t> >(hyp);
        for (long i = 0; i < hyp.getN123(); i++) mod->getVals()[i] = (data_t)model[i];
        std::shared_ptr<vecReg<data_t> > dat = std::make_shared<vecReg<data_t> >(*op->getRange());
        dat->zero();
        op->forward(false, mod, dat);
        for (long i = 0; i < dat->getN123(); i++) syn[i] = (double)dat->getCVals()[i];
        if (adj) {
            std::shared_ptr<vecReg<data_t> > a = std::make_shared<vecReg<data_t> >(*op->getRange());
            for (long i = 0; i < a->getN123(); i++) a->getVals()[i] = (data_t)adj[i];
            std::shared_ptr<vecReg<data_t> > g = std::make_shared<vecReg<data_t> >(hyp);
            g->zero();
            op->jacobianT(false, g, mod, a);
            for (long i = 0; i < hyp.getN123(); i++) grad[i] = (double)g->getCVals()[i];
        }
        return 0;
    } catch (const std::exception &e) {
        fprintf(stderr, "refside_run: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
