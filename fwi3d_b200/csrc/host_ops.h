// Host-side preparation and post-processing around the propagator, with the
// semantics of the reference's apply_forward / apply_jacobianT
// (nmbader/fwi3d src/cpp/we_op.cpp:872-1078).  All O(nt*ntr) and O(nxyz)-once
// work lives here; the time loop runs on the GPU (engine.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fwi3d_gpu.h"

namespace fwi {

// Time axis after model analysis (we_op.cpp:405-446).
struct TimeAxis {
    float dt;      // propagation step
    int nt;        // propagation samples
    int sub;       // imaging / snapshot sub-sampling (0: none)
    float courant;
    float vmax, vmin;
};

// Clip the model to the bounds, derive dt/nt/sub (analyzeModel, we_op.cpp:234-446).
// `model` is [nmodels][ny][nx][nz] (vp, [vs], rho, [delta, eps, gamma]); modified in place.
TimeAxis analyze_model(std::vector<float> &model, int nmodels, int nx, int ny, int nz, float dx, float dy, float dz,
                       int nt_data, float dt_data, const fwi_param &p);

// vp,vs,rho(,delta,eps,gamma) -> lambda,mu,rho(,c13,eps,c66) or vp,rho -> K,1/rho
// (we_op.cpp:448-466, 1083-1106, 1535-1553).
void convert_model(std::vector<float> &model, int nmodels, int64_t n);

// Wavelet duplication (analyzeWavelet, we_op.cpp:138-232) for one shot:
// 1-D input -> [nscomp][nt]; already multi-component input is returned as is.
std::vector<float> expand_wavelet(const float *w, int ncomp_in, int nt, int nmodels, const fwi_param &p);

// Time resampling along the fast axis (operator.cpp:424-520); ntr traces.
void resample_forward(bool sinc, int hl, const float *in, int nt_in, float dt_in, float *out, int nt_out, float dt_out,
                      int ntr);
void resample_adjoint(bool sinc, int hl, float *in, int nt_in, float dt_in, const float *out, int nt_out, float dt_out,
                      int ntr);

// Windowed-sinc taps of the resampler from an (nt_in, dt_in) axis to an
// (nt_out, dt_out) axis: output sample t uses input samples first[t] ..
// first[t] + count[t] - 1 with factors s (float) and window win (double),
// concatenated in output order (the weights resample_forward/adjoint apply).
void sinc_resample_taps(int hl, int nt_in, float dt_in, int nt_out, float dt_out, std::vector<int> &first,
                        std::vector<int> &count, std::vector<float> &s, std::vector<double> &win);

// Trapezoid quadrature Ht and time derivative Dt (misc.cpp:44-94).
void apply_ht(bool inv, const float *in, float *out, int ntr, int nt, float dt);
void apply_dt(bool adj, const float *in, float *out, int ntr, int nt, float dt);

// 27-point H-weighted point injector / extractor (injector.cpp:3-311).
struct PointOp {
    int npts = 0;
    bool derivative = false;        // ddelta_m3 (moment tensor)
    std::vector<int> xind, yind, zind;  // [npts][3]
    std::vector<float> xw, yw, zw;      // [npts][2][3] (delta) or [npts][2][6] (derivative)
    int nw() const { return derivative ? 6 : 3; }
};
struct Loc {
    float x, y, z;
};
PointOp make_delta(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                   const std::vector<Loc> &loc, bool derivative);

// Device tables of an injector.  Injection entries: field component c receives
// weight * src[trace][it] at grid point gidx.  Extraction: receiver r of
// component c is sum_k w[k] u_c[gidx[k]].
struct InjTable {
    std::vector<int64_t> gidx[3];
    std::vector<int> trace[3];
    std::vector<float> w[3];
};
InjTable injection_table(const PointOp &op, int nx, int ny, int nz, int ncomp_field);
struct ExtTable {
    int nrec = 0;
    int ntap = 27;              // 27 (point receiver) or 54 (dipole: both ends)
    std::vector<int64_t> gidx;  // [nrec][ntap]
    std::vector<float> w;       // [nrec][ntap]
};
ExtTable extraction_table(const PointOp &op, int nx, int ny, int nz);

// DAS receivers (dipole_m3, injector.cpp:313-493): two delta points half a
// gauge length `gl` before (a) and after (b) the receiver along the fibre
// direction (dip, azimuth); the recorded value is b - a.
struct Loc5 {
    float x, y, z, dip, az;
};
struct Dipole {
    PointOp a, b;
};
Dipole make_dipole(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                   const std::vector<Loc5> &loc, float gl);
ExtTable dipole_extraction_table(const Dipole &d, int nx, int ny, int nz);
InjTable dipole_injection_table(const Dipole &d, int nx, int ny, int nz, int ncomp_field);
// dipole_to_strain (misc.cpp:11-42) on [3][nr][nt]: forward projects the
// three components on the fibre (into component 0, zeroing 1 and 2) and
// divides by gl; adjoint spreads component 0 back.
void dipole_to_strain(bool adj, float *p, const float *dip, const float *az, int nr, int nt, float gl);
// Fibre endpoints inside the model (analyzeGeometry, we_op.cpp:105-125).
bool dipole_inside(const Loc5 &l, float gl, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy,
                   float oz);

// H quadrature on a 3-D array along x, y, z (spatial_operators.cpp:11-177).
void apply_h3(float *g, int nx, int ny, int nz, float dx, float dy, float dz);

// Chain rule from (lambda,mu,rho) or (K,1/rho) gradients to (vp,vs,rho) or (vp,rho)
// (we_op.cpp:1040-1067).  `m` is the converted model.
void gradient_to_velocity(float *g, const float *m, int nmodels, int64_t nxyz);

// Absorbing-boundary divisors (1 + scaler) on the owning face of every boundary
// point, per component (spatial_operators.cpp:624-1076 acoustic,
// spatial_operators.hpp:1873-2567 elastic/VTI).  Face array sizes: top/bottom
// ny*nx, left/right ny*nz, front/back nx*nz.  Value 1 where nothing is scaled.
struct ScaleTables {
    std::vector<float> f[6][3];
};
ScaleTables boundary_divisors(const float *m, int nmodels, int nx, int ny, int nz, float dx, float dy, float dz,
                              float dt, const int bc[6]);

// cos^2 taper factors per axis and side (spatial_operators.cpp:408-506): value
// multiplied into the field at each index, 1 outside the zone.
struct TaperTables {
    std::vector<float> t[6];  // z_lo[nz], z_hi[nz], x_lo[nx], x_hi[nx], y_lo[ny], y_hi[ny]
};
TaperTables taper_tables(int nx, int ny, int nz, const int taper[6], float strength);

}  // namespace fwi
