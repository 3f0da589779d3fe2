// Summation-by-parts (SBP) stencil primitives evaluated at one grid point.
//
// The discretisation is the reference's (nmbader/fwi3d): 4th-order SBP first
// derivative D1 (interior (2/3, -1/12), 4 boundary rows x 6 weights;
// spatial_operators.cpp:179-290), variable-coefficient second derivative
// D2var (interior 5-point stencil with 10 weights, 6 boundary rows each an
// 8x8 block; spatial_operators.hpp:34-232), the one-sided boundary derivative
// S = (11/6, -3, 3/2, -1/3) used by the SAT penalties, and the diagonal H
// quadrature (17/48, 59/48, 43/48, 49/48).
//
// Everything here is a pure function of a point index and accessors, so the
// same code runs in the CUDA kernels and, compiled as host code, in unit
// harnesses.  Grid layout: [ny][nx][nz], z fastest; idx = (iy*nx + ix)*nz + iz.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define FWI_HD __host__ __device__ __forceinline__
#else
#define FWI_HD inline
#endif

namespace fwi {

struct SbpTables {
    float d2in[10];       // interior D2var weights
    float d2b[6][8][8];   // D2var boundary closure: row, field sample, material sample
    float d1b[4][6];      // D1 boundary closure
    float d1c0, d1c1;     // D1 interior: 2/3, -1/12
    float sb[4];          // one-sided boundary derivative S
    float hq[4];          // H quadrature closure weights
};

// Filled once by init_sbp_tables() (sbp_tables.cpp).  Each CUDA translation
// unit that includes this header gets its own constant-memory copy, uploaded
// from g_sbp_host with cudaMemcpyToSymbol before its first launch.
extern SbpTables g_sbp_host;
void init_sbp_tables();

#ifdef __CUDACC__
static __constant__ SbpTables c_sbp;
#endif

FWI_HD const SbpTables &sbp()
{
#if defined(__CUDA_ARCH__)
    return c_sbp;
#else
    return g_sbp_host;
#endif
}

// Strided 1-D view along one axis of a 3-D array: a(k) = p[base + k*stride].
struct Line {
    const float *p;
    int64_t base;
    int64_t stride;
    FWI_HD float operator()(int k) const { return p[base + (int64_t)k * stride]; }
};

// Closure-row coefficients, read where a kernel keeps them.  ConstRows: the
// constant-memory tables (a warp whose lanes sit on different closure rows
// reads them one row at a time).  SmemRows: a shared-memory copy whose rows
// are padded so that such lanes read different banks in one access
// (fill_smem_rows writes it).
struct ConstRows {
    FWI_HD float d1(int r, int k) const { return sbp().d1b[r][k]; }
    FWI_HD float d2(int r, int j, int k) const { return sbp().d2b[r][j][k]; }
};
constexpr int SR_D2 = 65, SR_D1 = 7;              // padded row strides (floats)
constexpr int SR_FLOATS = 6 * SR_D2 + 4 * SR_D1;  // 418
struct SmemRows {
    const float *p;
    FWI_HD float d1(int r, int k) const { return p[6 * SR_D2 + r * SR_D1 + k]; }
    FWI_HD float d2(int r, int j, int k) const { return p[r * SR_D2 + j * 8 + k]; }
};
// Thread `tid` of `nt` writes its share of the padded copy.
FWI_HD void fill_smem_rows(float *p, int tid, int nt)
{
    const SbpTables &t = sbp();
    for (int e = tid; e < 6 * 64 + 4 * 6; e += nt) {
        if (e < 6 * 64) p[(e >> 6) * SR_D2 + (e & 63)] = (&t.d2b[0][0][0])[e];
        else p[6 * SR_D2 + ((e - 384) / 6) * SR_D1 + (e - 384) % 6] = t.d1b[(e - 384) / 6][(e - 384) % 6];
    }
}

// Unscaled D1 row at index i of an n-sample line (no 1/h).  Boundary rows use
// the closure (left) or its mirror with a sign flip (right).
template <class A, class R = ConstRows>
FWI_HD float d1_row(const A &a, int i, int n, const R &b = R())
{
    const SbpTables &t = sbp();
    if (i < 4) {
        const int r = i;
        return b.d1(r, 0) * a(0) + b.d1(r, 1) * a(1) + b.d1(r, 2) * a(2) + b.d1(r, 3) * a(3) + b.d1(r, 4) * a(4) +
               b.d1(r, 5) * a(5);
    }
    if (i >= n - 4) {
        const int r = n - 1 - i;
        return -(b.d1(r, 0) * a(n - 1) + b.d1(r, 1) * a(n - 2) + b.d1(r, 2) * a(n - 3) + b.d1(r, 3) * a(n - 4) +
                 b.d1(r, 4) * a(n - 5) + b.d1(r, 5) * a(n - 6));
    }
    return t.d1c0 * (a(i + 1) - a(i - 1)) + t.d1c1 * (a(i + 2) - a(i - 2));
}

// D1 row of the product a*m (the reference's mult_D: derivative of par*in).
template <class A, class M, class R = ConstRows>
FWI_HD float d1_prod_row(const A &a, const M &m, int i, int n, const R &b = R())
{
    const SbpTables &t = sbp();
    if (i < 4) {
        const int r = i;
        return b.d1(r, 0) * a(0) * m(0) + b.d1(r, 1) * a(1) * m(1) + b.d1(r, 2) * a(2) * m(2) +
               b.d1(r, 3) * a(3) * m(3) + b.d1(r, 4) * a(4) * m(4) + b.d1(r, 5) * a(5) * m(5);
    }
    if (i >= n - 4) {
        const int r = n - 1 - i;
        return -(b.d1(r, 0) * a(n - 1) * m(n - 1) + b.d1(r, 1) * a(n - 2) * m(n - 2) +
                 b.d1(r, 2) * a(n - 3) * m(n - 3) + b.d1(r, 3) * a(n - 4) * m(n - 4) +
                 b.d1(r, 4) * a(n - 5) * m(n - 5) + b.d1(r, 5) * a(n - 6) * m(n - 6));
    }
    return t.d1c0 * (a(i + 1) * m(i + 1) - a(i - 1) * m(i - 1)) + t.d1c1 * (a(i + 2) * m(i + 2) - a(i - 2) * m(i - 2));
}

// Variable-coefficient second derivative (d/dx f d/dx) at index i, times ad2 = a/h^2.
// u: field line, f: material line (the coefficient function sampled on the same line).
template <class U, class F, class R = ConstRows>
FWI_HD float d2var_row(const U &u, const F &f, int i, int n, float ad2, const R &b = R())
{
    const SbpTables &t = sbp();
    if (i < 6 || i >= n - 6) {
        const bool hi = i >= n - 6;
        const int r = hi ? n - 1 - i : i;
        float fk[8];
#pragma unroll
        for (int k = 0; k < 8; k++) fk[k] = f(hi ? n - 1 - k : k);
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            float v = 0.f;
#pragma unroll
            for (int k = 0; k < 8; k++) v += b.d2(r, j, k) * fk[k];
            acc += ad2 * v * u(hi ? n - 1 - j : j);
        }
        return acc;
    }
    const float *c = t.d2in;
    const float fm2 = f(i - 2), fm1 = f(i - 1), f0 = f(i), fp1 = f(i + 1), fp2 = f(i + 2);
    return ad2 * ((c[0] * f0 + c[1] * (fm1 + fp1) + c[2] * (fm2 + fp2)) * u(i) +
                  (c[3] * fm2 + c[4] * fm1 + c[5] * f0 + c[6] * fp1) * u(i - 1) +
                  (c[3] * fp2 + c[4] * fp1 + c[5] * f0 + c[6] * fm1) * u(i + 1) +
                  (c[7] * fm2 + c[8] * fm1 + c[9] * f0) * u(i - 2) +
                  (c[7] * fp2 + c[8] * fp1 + c[9] * f0) * u(i + 2));
}

// Outward one-sided boundary derivative S at the wall (unscaled), lo or hi side.
template <class A>
FWI_HD float sbound(const A &a, int n, bool hi)
{
    const SbpTables &t = sbp();
    if (!hi) return t.sb[0] * a(0) + t.sb[1] * a(1) + t.sb[2] * a(2) + t.sb[3] * a(3);
    return t.sb[0] * a(n - 1) + t.sb[1] * a(n - 2) + t.sb[2] * a(n - 3) + t.sb[3] * a(n - 4);
}

// Boundary D1 row 0 at the wall (unscaled), with the sign of the closure on each side.
template <class A>
FWI_HD float d1_wall(const A &a, int n, bool hi)
{
    const float *b = sbp().d1b[0];
    if (!hi) return b[0] * a(0) + b[1] * a(1) + b[2] * a(2) + b[3] * a(3) + b[4] * a(4) + b[5] * a(5);
    return -(b[0] * a(n - 1) + b[1] * a(n - 2) + b[2] * a(n - 3) + b[3] * a(n - 4) + b[4] * a(n - 5) +
             b[5] * a(n - 6));
}

// Grid helper.
struct Dims {
    int nx, ny, nz;
    FWI_HD int64_t idx(int ix, int iy, int iz) const { return ((int64_t)iy * nx + ix) * nz + iz; }
    FWI_HD int64_t nxyz() const { return (int64_t)nx * ny * nz; }
    // Lines through (ix,iy,iz) along each axis.
    FWI_HD Line lx(const float *p, int iy, int iz) const { return Line{p, (int64_t)iy * nx * nz + iz, nz}; }
    FWI_HD Line ly(const float *p, int ix, int iz) const { return Line{p, (int64_t)ix * nz + iz, (int64_t)nx * nz}; }
    FWI_HD Line lz(const float *p, int ix, int iy) const { return Line{p, ((int64_t)iy * nx + ix) * nz, 1}; }
};

}  // namespace fwi
