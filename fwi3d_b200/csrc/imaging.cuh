// Imaging conditions of the adjoint-state gradient at one grid point.
//
// Reference: compute_gradients of nl_we_op_e (we_op.cpp:488-565),
// nl_we_op_vti (:1108-1216) and nl_we_op_a (:1555-1605).  `itl` is the snapshot
// index (time / sub); the first (itl == 0) and last (itl >= nt/sub) samples use
// one-sided time differences and the half trapezoid weight, as in the reference.
// Increments are formed in the reference's precision (float, with the 1/dt and
// 0.5 dt factors evaluated in double) and accumulated in double.
#pragma once

#include "physics.cuh"

namespace fwi {

struct ImageArgs {
    Dims g;
    float dx, dy, dz;
    float rdx, rdy, rdz;  // 1/dx, 1/dy, 1/dz (interior taps multiply, as the step kernels do)
    float dtimg;  // sub * dt
    int itl;      // snapshot index of this imaging step
    int last;     // nt / sub (integer division)
    const float *m[6];
    const float *fwd[3][3];   // forward snapshots [itl-1, itl, itl+1][component]
    const float *adj[3];      // adjoint wavefield (curr)
    const float *lag[3];      // adjoint wavefield one step earlier (elastic derivatives lag one step)
    double *grad[3];
};

// D1 of a component field (with the 1/h).
FWI_HD float dx1(const Dims &g, const float *p, int ix, int iy, int iz, float d) { return d1_row(g.lx(p, iy, iz), ix, g.nx) / d; }
FWI_HD float dy1(const Dims &g, const float *p, int ix, int iy, int iz, float d) { return d1_row(g.ly(p, ix, iz), iy, g.ny) / d; }
FWI_HD float dz1(const Dims &g, const float *p, int ix, int iy, int iz, float d) { return d1_row(g.lz(p, ix, iy), iz, g.nz) / d; }

// Interior D1 at flat index i along a stride, times rd = 1/h: the interior
// branch of d1_row, term for term, with the reference's division by h
// replaced by the product with its reciprocal (as in the step kernels; at
// most one rounding apart, and 18 IEEE divisions per point and shot were a
// quarter of the adjoint's time).
FWI_HD float d1s(const float *p, int64_t i, int64_t st, float rd)
{
    const SbpTables &t = sbp();
    return (t.d1c0 * (p[i + st] - p[i - st]) + t.d1c1 * (p[i + 2 * st] - p[i - 2 * st])) * rd;
}

// Increments of the three gradients at one point for the shot whose fields
// start at offset `so` (batches: shot s at s * shot stride).
// IN: the point is at least 4 samples from every face, so every D1 is an
// interior row and is read at constant strides (no closure tests).
template <int PH, bool IN = false>
FWI_HD void elastic_image_inc(const ImageArgs &a, int64_t so, int ix, int iy, int iz, double &inc0, double &inc1,
                              double &inc2)
{
    const Dims &g = a.g;
    const int64_t i = g.idx(ix, iy, iz);
    const float *const fn[3] = {a.fwd[1][0] + so, a.fwd[1][1] + so, a.fwd[1][2] + so};
    const float *const lag[3] = {a.lag[0] + so, a.lag[1] + so, a.lag[2] + so};
    const int64_t SX = g.nz, SY = (int64_t)g.nx * g.nz;
    auto DX = [&](const float *p) { return IN ? d1s(p, i, SX, a.rdx) : dx1(g, p, ix, iy, iz, a.dx); };
    auto DY = [&](const float *p) { return IN ? d1s(p, i, SY, a.rdy) : dy1(g, p, ix, iy, iz, a.dy); };
    auto DZ = [&](const float *p) { return IN ? d1s(p, i, 1, a.rdz) : dz1(g, p, ix, iy, iz, a.dz); };
    // forward strains at the imaging time (we_op.cpp:510-518)
    const float t0 = DX(fn[0]), t1 = DY(fn[1]), t2 = DZ(fn[2]);
    const float t3 = DX(fn[2]), t4 = DZ(fn[0]);
    const float t5 = DX(fn[1]), t6 = DY(fn[0]);
    const float t7 = DY(fn[2]), t8 = DZ(fn[1]);
    // adjoint strains (of the previous adjoint step)
    const float ax0 = DX(lag[0]), ax1 = DX(lag[1]), ax2 = DX(lag[2]);
    const float ay0 = DY(lag[0]), ay1 = DY(lag[1]), ay2 = DY(lag[2]);
    const float az0 = DZ(lag[0]), az1 = DZ(lag[1]), az2 = DZ(lag[2]);
    const float dt = a.dtimg;
    const bool first = a.itl == 0;
    const bool mid = a.itl > 0 && a.itl < a.last;
    float glam, gmu;
    if (PH == ELASTIC) {
        // dt (div adj) (div fwd): the reference multiplies dt into the first factor
        const float A = ax0 + ay1 + az2, B = t0 + t1 + t2;
        inc0 = first ? 0.5 * dt * A * B : (double)(dt * A * B);
        gmu = (az0 + ax2) * (t3 + t4) + (ay0 + ax1) * (t5 + t6) + (az1 + ay2) * (t7 + t8) + 2 * ax0 * t0 +
              2 * ay1 * t1 + 2 * az2 * t2;
    } else {
        const float lam = a.m[0][i], mu = a.m[1][i], c13 = a.m[3][i], eps = a.m[4][i], c66 = a.m[5][i];
        const float del = ((c13 + mu) * (c13 + mu) - (lam + mu) * (lam + mu)) / (2 * (lam + mu) * (lam + 2 * mu));
        const float gam = (c66 - mu) / (2 * mu);
        const float v1 = (float)sqrt((double)(2 * (lam + 2 * mu) * (lam + mu) * del + (lam + mu) * (lam + mu)));
        const float v2 = ((1 + 2 * del) * lam + (1 + 3 * del) * mu) / v1;
        const float v3 = ((1 + 3 * del) * lam + (1 + 4 * del) * mu) / v1 - 1;
        const float v4 = (ax0 + ay1) * t2 + az2 * (t0 + t1);
        glam = (1 + 2 * eps) * (ax0 + ay1) * (t0 + t1) + az2 * t2 + v2 * v4;
        gmu = 2 * (1 + 2 * eps) * (ax0 * t0 + ay1 * t1) + 2 * az2 * t2 + 4 * (eps - gam) * (ax0 * t1 + ax0 * t0) +
              (ay2 + az1) * (t7 + t8) + (ax2 + az0) * (t3 + t4) + (1 + 2 * gam) * (ax1 + ay0) * (t5 + t6) + v3 * v4;
        inc0 = first ? 0.5 * dt * glam : (double)(dt * glam);
    }
    inc1 = first ? 0.5 * dt * gmu : (double)(dt * gmu);
    float s = 0.f;
    for (int c = 0; c < 3; c++) {
        const float fp = a.fwd[2][c][so + i], f0 = a.fwd[1][c][so + i];
        float tt;
        if (mid) tt = fp - 2 * f0 + a.fwd[0][c][so + i];
        else if (first) tt = fp - f0;
        else tt = -f0 + a.fwd[0][c][so + i];
        s = (c == 0) ? a.adj[c][so + i] * tt : s + a.adj[c][so + i] * tt;
    }
    inc2 = 1.0 / dt * s;
}

template <int PH>
FWI_HD void elastic_image_point(const ImageArgs &a, int ix, int iy, int iz)
{
    const int64_t i = a.g.idx(ix, iy, iz);
    double inc0, inc1, inc2;
    elastic_image_inc<PH>(a, 0, ix, iy, iz, inc0, inc1, inc2);
    a.grad[0][i] += inc0;
    a.grad[1][i] += inc1;
    a.grad[2][i] += inc2;
}

FWI_HD void acoustic_image_inc(const ImageArgs &a, int64_t so, int ix, int iy, int iz, double &inck, double &incb)
{
    const Dims &g = a.g;
    const int64_t i = g.idx(ix, iy, iz);
    const float *fn = a.fwd[1][0] + so;
    const float t0 = dx1(g, fn, ix, iy, iz, a.dx), t1 = dy1(g, fn, ix, iy, iz, a.dy), t2 = dz1(g, fn, ix, iy, iz, a.dz);
    const float *ad = a.adj[0] + so;
    const float t3 = dx1(g, ad, ix, iy, iz, a.dx), t4 = dy1(g, ad, ix, iy, iz, a.dy), t5 = dz1(g, ad, ix, iy, iz, a.dz);
    const float dt = a.dtimg;
    const float K = a.m[0][i];
    const bool first = a.itl == 0;
    const bool mid = a.itl > 0 && a.itl < a.last;
    const float fp = a.fwd[2][0][so + i], f0 = a.fwd[1][0][so + i];
    float tt;
    if (mid) tt = fp - 2 * f0 + a.fwd[0][0][so + i];
    else if (first) tt = fp - f0;
    else tt = -2 * f0 + a.fwd[0][0][so + i];  // the reference's last-sample form (we_op.cpp:1601)
    const float q = t3 * t0 + t4 * t1 + t5 * t2;
    inck = 1.0 / (double)(dt * K * K) * (double)ad[i] * (double)tt;
    incb = first ? 0.5 * dt * q : (double)(dt * q);
}

FWI_HD void acoustic_image_point(const ImageArgs &a, int ix, int iy, int iz)
{
    const int64_t i = a.g.idx(ix, iy, iz);
    double inck, incb;
    acoustic_image_inc(a, 0, ix, iy, iz, inck, incb);
    a.grad[0][i] -= inck;
    a.grad[1][i] += incb;
}

}  // namespace fwi
