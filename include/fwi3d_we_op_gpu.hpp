/*
 * fwi3d_we_op_gpu.hpp -- reference-side binding: GPU operators that drop in
 * beside nmbader/fwi3d's nl_we_op_e, nl_we_op_vti and nl_we_op_a
 * (src/include/we_op.hpp:50-167).
 *
 * Each class derives from the reference operator it replaces, keeps its
 * constructor (domain, allsrc, s, par), its public members (_par, _src,
 * _allsrc) and its range, and overrides the two virtual seams the reference's
 * forward / jacobianT call (we_op.hpp:37-47):
 *   apply_forward(add, pmod, pdat)            -> fwi_op_forward
 *   apply_jacobianT(add, pmod, pmod0, pdat)   -> fwi_op_jacobianT
 * so that model analysis, conversion, propagation, imaging, quadrature and
 * the chain rule to (vp, vs, rho[, delta, epsilon, gamma]) run in
 * libfwi3d_b200 on the GPU, with the reference's `add` semantics.  A failing
 * call stops through the reference's successCheck (misc.hpp:4-12) with the
 * library's message.
 *
 * Use: construct nl_we_op_e_gpu where the reference constructs nl_we_op_e
 * (src/main/we_modeling.cpp:77-86, src/cpp/optimization.cpp:41-50,
 * src/main/fwi3d.cpp:251-255); build the reference with data_t = float and
 * link -lfwi3d_b200 (include/fwi3d_gpu.h).
 */
#pragma once

#include <vector>

#include "fwi3d_gpu.h"
#include "we_op.hpp"

static_assert(sizeof(data_t) == sizeof(float), "the GPU operators take the reference's FP32 build (data_t = float)");

namespace fwi3d_binding {

/* The propagation knobs of the reference's param (param.hpp:8-71) as the C ABI's fwi_param. */
inline fwi_param to_c(const param &p)
{
    fwi_param c;
    fwi_param_default(&c);
    c.courant = p.courant;
    c.dt = p.dt;
    c.sub = p.sub;
    c.resampling_linear = p.resampling == "linear";
    c.sinc_half_length = p.sinc_half_length;
    c.mt = p.mt;
    c.fangle = p.fangle;
    c.fazimuth = p.fazimuth;
    c.mxx = p.mxx; c.myy = p.myy; c.mzz = p.mzz; c.mxy = p.mxy; c.mxz = p.mxz; c.myz = p.myz;
    c.seismotype = p.seismotype;
    c.gl = p.gl;
    const int bc[6] = {p.bc_top, p.bc_bottom, p.bc_left, p.bc_right, p.bc_front, p.bc_back};
    const int tp[6] = {p.taper_top, p.taper_bottom, p.taper_left, p.taper_right, p.taper_front, p.taper_back};
    for (int f = 0; f < 6; f++) {
        c.bc[f] = bc[f];
        c.taper[f] = tp[f];
    }
    c.free_surface_stiffness = p.free_surface_stiffness;
    c.taper_strength = p.taper_strength;
    c.vpmin = p.vpmin; c.vpmax = p.vpmax; c.vsmin = p.vsmin; c.vsmax = p.vsmax;
    c.rhomin = p.rhomin; c.rhomax = p.rhomax;
    c.deltamin = p.deltamin; c.deltamax = p.deltamax;
    c.epsilonmin = p.epsilonmin; c.epsilonmax = p.epsilonmax;
    c.gammamin = p.gammamin; c.gammamax = p.gammamax;
    c.soft_clip = p.soft_clip;
    c.verbose = p.verbose;
    return c;
}

/* One GPU operator (one shot) built from a reference operator's members. */
class gpu_op {
    fwi_op *_op = nullptr;

public:
    gpu_op() = default;
    gpu_op(const gpu_op &) = delete;
    gpu_op &operator=(const gpu_op &) = delete;
    ~gpu_op()
    {
        if (_op) fwi_op_destroy(_op);
    }
    void create(const hypercube<data_t> &domain, const std::shared_ptr<vecReg<data_t> > &src, const param &par,
                int nmodels, int device)
    {
        const axis<data_t> Z = domain.getAxis(1), X = domain.getAxis(2), Y = domain.getAxis(3);
        fwi_grid g{X.n, Y.n, Z.n, X.o, Y.o, Z.o, X.d, Y.d, Z.d};
        const fwi_param c = to_c(par);
        const axis<data_t> T = src->getHyper()->getAxis(1);
        const int ncomp = (int)(src->getN123() / T.n);
        std::vector<float> sxyz(par.sxyz[0].begin(), par.sxyz[0].begin() + 3), rxyz;
        for (const auto &r : par.rxyz[0]) rxyz.insert(rxyz.end(), r.begin(), r.begin() + 5);
        const int rc = fwi_op_create(&_op, device, &g, nmodels, &c, src->getCVals(), ncomp, T.n, T.d, sxyz.data(),
                                     (int)par.rxyz[0].size(), rxyz.data());
        successCheck(rc == FWI_OK, std::string("fwi_op_create: ") + fwi_last_error() + "\n");
    }
    /* the time axis the GPU path chose, written back as the reference's
     * apply_forward does to its _par (we_op.cpp:876) */
    void sync_par(param &par) const
    {
        fwi_op_info info;
        if (fwi_op_get_info(_op, &info) == FWI_OK) {
            par.dt = info.dt;
            par.nt = info.nt;
            par.sub = info.sub;
        }
    }
    void forward(bool add, const data_t *pmod, data_t *pdat, param &par)
    {
        successCheck(fwi_op_forward(_op, add, pmod, pdat) == FWI_OK,
                     std::string("fwi_op_forward: ") + fwi_last_error() + "\n");
        sync_par(par);
    }
    void jacobianT(bool add, data_t *pmod, const data_t *pmod0, const data_t *pdat, param &par)
    {
        successCheck(fwi_op_jacobianT(_op, add, pmod, pmod0, pdat) == FWI_OK,
                     std::string("fwi_op_jacobianT: ") + fwi_last_error() + "\n");
        sync_par(par);
    }
};

}  // namespace fwi3d_binding

/* Elastic isotropic operator on the GPU (replaces nl_we_op_e). */
class nl_we_op_e_gpu : public nl_we_op_e {
    fwi3d_binding::gpu_op _gpu;
    int _device;

public:
    nl_we_op_e_gpu(const hypercube<data_t> &domain, const std::shared_ptr<vecReg<data_t> > allsrc, int s, param &par,
                   int device = 0)
        : nl_we_op_e(domain, allsrc, s, par), _device(device)
    {
        _gpu.create(domain, _src, _par, 3, device);
    }
    nl_we_op_e_gpu *clone() const
    {
        param par = _par;
        return new nl_we_op_e_gpu(_domain, _src, 0, par, _device);
    }
    void apply_forward(bool add, const data_t *pmod, data_t *pdat) { _gpu.forward(add, pmod, pdat, _par); }
    void apply_jacobianT(bool add, data_t *pmod, const data_t *pmod0, const data_t *pdat)
    {
        _gpu.jacobianT(add, pmod, pmod0, pdat, _par);
    }
};

/* Elastic VTI operator on the GPU (replaces nl_we_op_vti). */
class nl_we_op_vti_gpu : public nl_we_op_vti {
    fwi3d_binding::gpu_op _gpu;
    int _device;

public:
    nl_we_op_vti_gpu(const hypercube<data_t> &domain, const std::shared_ptr<vecReg<data_t> > allsrc, int s,
                     param &par, int device = 0)
        : nl_we_op_e(domain, allsrc, s, par), nl_we_op_vti(domain, allsrc, s, par), _device(device)
    {
        _gpu.create(domain, _src, _par, 6, device);
    }
    nl_we_op_vti_gpu *clone() const
    {
        param par = _par;
        return new nl_we_op_vti_gpu(_domain, _src, 0, par, _device);
    }
    void apply_forward(bool add, const data_t *pmod, data_t *pdat) { _gpu.forward(add, pmod, pdat, _par); }
    void apply_jacobianT(bool add, data_t *pmod, const data_t *pmod0, const data_t *pdat)
    {
        _gpu.jacobianT(add, pmod, pmod0, pdat, _par);
    }
};

/* Acoustic variable-density operator on the GPU (replaces nl_we_op_a). */
class nl_we_op_a_gpu : public nl_we_op_a {
    fwi3d_binding::gpu_op _gpu;
    int _device;

public:
    nl_we_op_a_gpu(const hypercube<data_t> &domain, const std::shared_ptr<vecReg<data_t> > allsrc, int s, param &par,
                   int device = 0)
        : nl_we_op_a(domain, allsrc, s, par), _device(device)
    {
        _gpu.create(domain, _src, _par, 2, device);
    }
    nl_we_op_a_gpu *clone() const
    {
        param par = _par;
        return new nl_we_op_a_gpu(_domain, _src, 0, par, _device);
    }
    void apply_forward(bool add, const data_t *pmod, data_t *pdat) { _gpu.forward(add, pmod, pdat, _par); }
    void apply_jacobianT(bool add, data_t *pmod, const data_t *pmod0, const data_t *pdat)
    {
        _gpu.jacobianT(add, pmod, pmod0, pdat, _par);
    }
};
