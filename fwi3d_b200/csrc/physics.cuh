// Per-point right-hand sides of the three wave equations, their SAT boundary
// penalties, the leapfrog update, the absorbing-boundary scaling and the taper.
//
// Reference semantics (nmbader/fwi3d src/cpp/we_op.cpp):
//   acoustic VD  propagate :1607-1826  (p_tt = K div(b grad p), b = 1/rho)
//   elastic iso  propagate :567-870    (rho u_tt = div sigma, displacement form)
//   elastic VTI  propagate :1218-1531
// Each time step computes, per output point, the same sum of operator terms in
// the same order as the reference's sequence of full-grid passes (D2var x3,
// D1(tmp), mult_D x2, SAT faces top..back), then
//   next = dt^2 acc / rho + 2 curr - prev      (elastic, :806-813)
//   next = dt^2 acc K     + 2 curr - prev      (acoustic, :1768-1773)
// then divides absorbing-boundary points by (1 + scaler) and applies the
// cos^2 taper.  The reference tapers `curr` in place after each step, so the
// value it later reads as `prev` carries the taper twice; here `curr` is left
// as written and the second taper is applied when it is read back as `prev`
// (flag taper_prev, off for the first step whose `prev` is the initial
// source injection).
#pragma once

#include "sbp.cuh"

namespace fwi {

enum Physics { ACOUSTIC = 2, ELASTIC = 3, VTI = 6 };
enum Face { TOP = 0, BOTTOM = 1, LEFT = 2, RIGHT = 3, FRONT = 4, BACK = 5 };
enum Bc { BC_NONE = 0, BC_FREE = 1, BC_ABSORB = 2, BC_RIGID = 3 };

// Elastic auxiliary first-derivative fields written by the derivative pass.
// Slot: 0..2 the divergence-like combination differentiated by Dx (comp 0),
// Dy (comp 1), Dz (comp 2) -- one shared array for isotropic media;
// 3 u_x[1], 4 u_x[2], 5 u_y[0], 6 u_y[2], 7 u_z[0], 8 u_z[1].
enum Aux { AUX_T0 = 0, AUX_T1 = 1, AUX_T2 = 2, AUX_X1 = 3, AUX_X2 = 4, AUX_Y0 = 5, AUX_Y2 = 6, AUX_Z0 = 7, AUX_Z1 = 8 };

struct StepArgs {
    Dims g;
    float dx, dy, dz, dt;
    float idx, idy, idz;       // 1/h per axis
    float ad1[3], ad2[3];      // a/(h*h) per axis (x, y, z) for a = 1 and a = 2, as the reference forms them
    // converted model: acoustic {K, 1/rho}; elastic {lambda, mu, rho}; VTI {lambda, mu, rho, c13, eps, c66}
    const float *m[6];
    const float *curr[3];
    const float *prev[3];
    float *next[3];
    const float *aux[9];
    int bc[6];
    float alpha_fs;            // acoustic free-surface Dirichlet penalty 0.2508560249/free_surface_stiffness
    const float *sdiv[6][3];   // absorbing-boundary divisors (1+scaler) on the owning face, per component
    int scale;                 // any face absorbing
    const float *tap[6];       // taper factors tz_lo[nz], tz_hi[nz], tx_lo[nx], tx_hi[nx], ty_lo[ny], ty_hi[ny]
    int tw[6];                 // taper widths top, bottom, left, right, front, back
    int taper_prev;
    // batch layout: shot s of a field component c lives at curr[c] + s*sst
    int nyb;                   // y blocks per shot in the launch grid
    int y0, y1;                // planes [y0, y1) covered by the launch
    int64_t sst;               // wavefield shot stride (floats)
    int64_t ast;               // derivative-scratch shot stride (floats)
    // D2var closure weights precomputed per model for the 12 closure rows of
    // every line along x, y, z (w2c[axis][f], null: formed in place), of the
    // coefficient f = 0 mu, 1 c66, 2 c11b = 2 (1 + 2 eps) mu (VTI); line index
    // y*nz + z (x lines), x*nz + z (y lines), y*nx + x (z lines)
    const float *w2c[3][3];
    // shot slots: active[s] == 0 marks an idle slot, whose fields no kernel
    // advances (null: every shot active)
    const int *active;
};

// An idle shot slot: its CTAs or threads return at once.
FWI_HD bool shot_idle(const StepArgs &a, int s) { return a.active && !a.active[s]; }

// Pointers of shot s.
FWI_HD StepArgs shot_args(const StepArgs &a, int s)
{
    StepArgs b = a;
    for (int c = 0; c < 3; c++) {
        if (b.curr[c]) b.curr[c] += s * a.sst;
        if (b.prev[c]) b.prev[c] += s * a.sst;
        if (b.next[c]) b.next[c] += s * a.sst;
    }
    for (int k = 0; k < 9; k++)
        if (b.aux[k]) b.aux[k] += s * a.ast;
    return b;
}

// ---------------------------------------------------------------------------
// Taper and absorbing-boundary scaling
// ---------------------------------------------------------------------------
// True where any taper factor differs from one (the reference tapers the
// first taper_top rows from the top, the last taper_bottom rows, etc.).
FWI_HD bool in_taper(const StepArgs &a, int ix, int iy, int iz)
{
    return iz < a.tw[0] || iz >= a.g.nz - a.tw[1] || ix < a.tw[2] || ix >= a.g.nx - a.tw[3] || iy < a.tw[4] ||
           iy >= a.g.ny - a.tw[5];
}

FWI_HD float taper(const StepArgs &a, float v, int ix, int iy, int iz)
{
    v = v * a.tap[0][iz];
    v = v * a.tap[1][iz];
    v = v * a.tap[2][ix];
    v = v * a.tap[3][ix];
    v = v * a.tap[4][iy];
    v = v * a.tap[5][iy];
    return v;
}

// Owning face of a boundary point for the scaling tables, and its 2-D offset.
FWI_HD int owner_face(const Dims &g, int ix, int iy, int iz, int64_t &off)
{
    if (iz == 0) { off = (int64_t)iy * g.nx + ix; return TOP; }
    if (iz == g.nz - 1) { off = (int64_t)iy * g.nx + ix; return BOTTOM; }
    if (ix == 0) { off = (int64_t)iy * g.nz + iz; return LEFT; }
    if (ix == g.nx - 1) { off = (int64_t)iy * g.nz + iz; return RIGHT; }
    if (iy == 0) { off = (int64_t)ix * g.nz + iz; return FRONT; }
    if (iy == g.ny - 1) { off = (int64_t)ix * g.nz + iz; return BACK; }
    return -1;
}

FWI_HD float boundary_scale(const StepArgs &a, float v, int c, int ix, int iy, int iz)
{
    if (!a.scale) return v;
    int64_t off;
    const int f = owner_face(a.g, ix, iy, iz, off);
    if (f < 0) return v;
    return v / a.sdiv[f][c][off];
}

FWI_HD float prev_eff(const StepArgs &a, int c, int64_t i, int ix, int iy, int iz, int64_t so = 0)
{
    const float p = a.prev[c][so + i];
    return a.taper_prev ? taper(a, p, ix, iy, iz) : p;
}

// ---------------------------------------------------------------------------
// Acoustic variable density
// ---------------------------------------------------------------------------
struct Mat {
    Line l;
    FWI_HD float operator()(int k) const { return l(k); }
};

FWI_HD float acoustic_acc(const StepArgs &a, int ix, int iy, int iz)
{
    const Dims &g = a.g;
    const float *u = a.curr[0];
    const float *b = a.m[1];
    // D2var along x, y, z with coefficient 1/rho (we_op.cpp:1664-1666)
    float acc = d2var_row(g.lx(u, iy, iz), g.lx(b, iy, iz), ix, g.nx, 1.0f / (a.dx * a.dx));
    acc += d2var_row(g.ly(u, ix, iz), g.ly(b, ix, iz), iy, g.ny, 1.0f / (a.dy * a.dy));
    acc += d2var_row(g.lz(u, ix, iy), g.lz(b, ix, iy), iz, g.nz, 1.0f / (a.dz * a.dz));
    return acc;
}

// Dirichlet (free-surface) SAT contribution at row `r` (0..3) from the wall
// point w (spatial_operators.cpp:508-622): the reference evaluates
// 1.0/(h_r d^2) s_r b_w p_w in double precision before rounding.
FWI_HD float asat_dirichlet(float acc, int r, float bw, float pw, float d, float alpha)
{
    const SbpTables &t = sbp();
    const float d2 = d * d;
    double v = 1.0 / (double)(t.hq[r] * d2) * (double)t.sb[r] * (double)bw * (double)pw;
    acc = (float)((double)acc + v);
    if (r == 0) acc -= bw * pw / (alpha * t.hq[0] * d2);
    return acc;
}

// Neumann SAT at a wall point (spatial_operators.hpp:2580-2716): f1 = 1/rho,
// f2 = 1/(2 sqrt(rho K)) (absorbing) or 0 (rigid).
FWI_HD float asat_neumann(float acc, float S, float bw, float Kw, float pw, float d, float dt, bool absorbing)
{
    const float h0 = sbp().hq[0];
    const float adh = (float)(1.0 / (double)(h0 * d));
    float f2 = 0.f;
    if (absorbing) f2 = (float)(0.5 / sqrt((double)(Kw / bw)));
    return acc - adh * (bw * S / d - f2 * pw / dt);
}

FWI_HD float acoustic_sat(const StepArgs &a, float acc, int ix, int iy, int iz)
{
    const Dims &g = a.g;
    const float *u = a.curr[0];
    const float *K = a.m[0];
    const float *b = a.m[1];
    // top / bottom (normal z)
    for (int side = 0; side < 2; side++) {
        const int bc = a.bc[TOP + side];
        const int wz = side ? g.nz - 1 : 0;
        const int r = side ? g.nz - 1 - iz : iz;
        if (bc == BC_FREE && r < 4) {
            const int64_t w = g.idx(ix, iy, wz);
            acc = asat_dirichlet(acc, r, b[w], u[w], a.dz, a.alpha_fs);
        } else if ((bc == BC_ABSORB || bc == BC_RIGID) && r == 0) {
            const int64_t w = g.idx(ix, iy, wz);
            const float S = sbound(g.lz(u, ix, iy), g.nz, side);
            acc = asat_neumann(acc, S, b[w], K[w], prev_eff(a, 0, w, ix, iy, wz), a.dz, a.dt, bc == BC_ABSORB);
        }
    }
    // left / right (normal x)
    for (int side = 0; side < 2; side++) {
        const int bc = a.bc[LEFT + side];
        const int wx = side ? g.nx - 1 : 0;
        const int r = side ? g.nx - 1 - ix : ix;
        if (bc == BC_FREE && r < 4) {
            const int64_t w = g.idx(wx, iy, iz);
            acc = asat_dirichlet(acc, r, b[w], u[w], a.dx, a.alpha_fs);
        } else if ((bc == BC_ABSORB || bc == BC_RIGID) && r == 0) {
            const int64_t w = g.idx(wx, iy, iz);
            const float S = sbound(g.lx(u, iy, iz), g.nx, side);
            acc = asat_neumann(acc, S, b[w], K[w], prev_eff(a, 0, w, wx, iy, iz), a.dx, a.dt, bc == BC_ABSORB);
        }
    }
    // front / back (normal y)
    for (int side = 0; side < 2; side++) {
        const int bc = a.bc[FRONT + side];
        const int wy = side ? g.ny - 1 : 0;
        const int r = side ? g.ny - 1 - iy : iy;
        if (bc == BC_FREE && r < 4) {
            const int64_t w = g.idx(ix, wy, iz);
            acc = asat_dirichlet(acc, r, b[w], u[w], a.dy, a.alpha_fs);
        } else if ((bc == BC_ABSORB || bc == BC_RIGID) && r == 0) {
            const int64_t w = g.idx(ix, wy, iz);
            const float S = sbound(g.ly(u, ix, iz), g.ny, side);
            acc = asat_neumann(acc, S, b[w], K[w], prev_eff(a, 0, w, ix, wy, iz), a.dy, a.dt, bc == BC_ABSORB);
        }
    }
    return acc;
}

FWI_HD float acoustic_point(const StepArgs &a, int ix, int iy, int iz)
{
    const int64_t i = a.g.idx(ix, iy, iz);
    float acc = acoustic_acc(a, ix, iy, iz);
    acc = acoustic_sat(a, acc, ix, iy, iz);
    const float dt2 = a.dt * a.dt;
    float v = dt2 * acc * a.m[0][i] + 2.f * a.curr[0][i] - prev_eff(a, 0, i, ix, iy, iz);
    v = boundary_scale(a, v, 0, ix, iy, iz);
    return taper(a, v, ix, iy, iz);
}

// ---------------------------------------------------------------------------
// Elastic (isotropic and VTI): material functions of the reference
// (we_op.cpp:468-486): c11b = 2(1+2eps)mu, c11c = (1+2eps)lambda,
// c12 = (1+2eps)(lambda+2mu) - 2 c66, simp = sqrt(rho mu)/2,
// pimp = sqrt(rho(lambda+2mu))/2, pimp2 = sqrt(rho(1+2eps)(lambda+2mu))/2.
// ---------------------------------------------------------------------------
struct C11bLine {
    Line eps, mu;
    FWI_HD float operator()(int k) const { return 2.f * (1.f + 2.f * eps(k)) * mu(k); }
};

FWI_HD float f_simp(float mu, float rho) { return (float)(0.5 * sqrt((double)(mu * rho))); }
FWI_HD float f_pimp(float lam, float mu, float rho) { return (float)(0.5 * sqrt((double)((lam + 2.f * mu) * rho))); }
FWI_HD float f_pimp2(float lam, float mu, float rho, float eps)
{
    return (float)(0.5 * sqrt((double)((1.f + 2.f * eps) * (lam + 2.f * mu) * rho)));
}

// Sum of the interior operator terms for component c (before SAT).
template <int PH>
FWI_HD float elastic_acc(const StepArgs &a, int c, int ix, int iy, int iz)
{
    const Dims &g = a.g;
    const float *mu = a.m[1];
    const float *u = a.curr[c];
    const float idx2 = 1.0f / (a.dx * a.dx), idy2 = 1.0f / (a.dy * a.dy), idz2 = 1.0f / (a.dz * a.dz);
    float acc;
    if (PH == ELASTIC) {
        // we_op.cpp:647-657: on-axis term doubled
        acc = d2var_row(g.lx(u, iy, iz), g.lx(mu, iy, iz), ix, g.nx, (c == 0 ? 2.0f : 1.0f) / (a.dx * a.dx));
        acc += d2var_row(g.ly(u, ix, iz), g.ly(mu, ix, iz), iy, g.ny, (c == 1 ? 2.0f : 1.0f) / (a.dy * a.dy));
        acc += d2var_row(g.lz(u, ix, iy), g.lz(mu, ix, iy), iz, g.nz, (c == 2 ? 2.0f : 1.0f) / (a.dz * a.dz));
    } else {
        // we_op.cpp:1298-1308: c11b on the in-plane axis of u_x/u_y, c66 across, mu along z
        const float *eps = a.m[4], *c66 = a.m[5];
        if (c == 0) {
            acc = d2var_row(g.lx(u, iy, iz), C11bLine{g.lx(eps, iy, iz), g.lx(mu, iy, iz)}, ix, g.nx, idx2);
            acc += d2var_row(g.ly(u, ix, iz), g.ly(c66, ix, iz), iy, g.ny, idy2);
            acc += d2var_row(g.lz(u, ix, iy), g.lz(mu, ix, iy), iz, g.nz, idz2);
        } else if (c == 1) {
            acc = d2var_row(g.lx(u, iy, iz), g.lx(c66, iy, iz), ix, g.nx, idx2);
            acc += d2var_row(g.ly(u, ix, iz), C11bLine{g.ly(eps, ix, iz), g.ly(mu, ix, iz)}, iy, g.ny, idy2);
            acc += d2var_row(g.lz(u, ix, iy), g.lz(mu, ix, iy), iz, g.nz, idz2);
        } else {
            acc = d2var_row(g.lx(u, iy, iz), g.lx(mu, iy, iz), ix, g.nx, idx2);
            acc += d2var_row(g.ly(u, ix, iz), g.ly(mu, ix, iz), iy, g.ny, idy2);
            acc += d2var_row(g.lz(u, ix, iy), g.lz(mu, ix, iy), iz, g.nz, 2.0f / (a.dz * a.dz));
        }
    }
    // Derivative of the normal-stress combination (we_op.cpp:669-671 / 1320-1332)
    // and the mixed terms mult_D (we_op.cpp:675-688 / 1336-1349).
    const float *P = (PH == VTI) ? a.m[5] : mu;  // c66 in VTI for the xy coupling
    if (c == 0) {
        acc += d1_row(g.lx(a.aux[AUX_T0], iy, iz), ix, g.nx) / a.dx;
        acc += d1_prod_row(g.ly(a.aux[AUX_X1], ix, iz), g.ly(P, ix, iz), iy, g.ny) / a.dy;
        // mult_Dz is passed dy here in the reference (we_op.cpp:678, 1339); kept for parity.
        acc += d1_prod_row(g.lz(a.aux[AUX_X2], ix, iy), g.lz(mu, ix, iy), iz, g.nz) / a.dy;
    } else if (c == 1) {
        acc += d1_row(g.ly(a.aux[AUX_T1], ix, iz), iy, g.ny) / a.dy;
        acc += d1_prod_row(g.lx(a.aux[AUX_Y0], iy, iz), g.lx(P, iy, iz), ix, g.nx) / a.dx;
        acc += d1_prod_row(g.lz(a.aux[AUX_Y2], ix, iy), g.lz(mu, ix, iy), iz, g.nz) / a.dz;
    } else {
        acc += d1_row(g.lz(a.aux[AUX_T2], ix, iy), iz, g.nz) / a.dz;
        acc += d1_prod_row(g.lx(a.aux[AUX_Z0], iy, iz), g.lx(mu, iy, iz), ix, g.nx) / a.dx;
        acc += d1_prod_row(g.ly(a.aux[AUX_Z1], ix, iz), g.ly(mu, ix, iz), iy, g.ny) / a.dy;
    }
    return acc;
}

// Coefficients of one elastic SAT face term (spatial_operators.hpp:236-1870):
//   lo face:  acc -= adh ( -f1 T1/d1 - f2 T2/d2 - f3 N0/dn + f4 S/dn - f5 P/dt )
//   hi face:  acc -= adh (  f1 T1/d1 + f2 T2/d2 + f3 N0/dn + f4 S/dn - f5 P/dt )
// T1, T2: tangential D1 rows of in1, in2; N0: wall D1 row of in3; S: one-sided
// derivative of in3; P: prev of the output component.
struct SatTerm {
    float f1, f2, f3, f4, f5;
};

// Material coefficients of the face terms for component c on a face with
// normal axis n (0 x, 1 y, 2 z) at point i (we_op.cpp:697-804, 1358-1465).
template <int PH>
FWI_HD SatTerm sat_coefs(const StepArgs &a, int n, int c, int64_t i, bool absorbing)
{
    const float lam = a.m[0][i], mu = a.m[1][i], rho = a.m[2][i];
    SatTerm s{0.f, 0.f, 0.f, 0.f, 0.f};
    if (c != n) {
        // tangential component: f(in1 or in2) = P, f4 = P, f5 = simp
        float P = mu;
        if (PH == VTI && n != 2 && c != 2) P = a.m[5][i];  // c66 couples x and y on x/y faces
        // which tangential slot carries the normal displacement derivative
        const bool first = (n == 2) ? (c == 0) : (n == 0 ? (c == 1) : (c == 0));
        if (first) s.f1 = P; else s.f2 = P;
        s.f4 = P;
        if (absorbing) s.f5 = f_simp(mu, rho);
    } else {
        if (PH == VTI && n != 2) {
            const float eps = a.m[4][i], c13 = a.m[3][i], c66 = a.m[5][i];
            s.f1 = (1.f + 2.f * eps) * (lam + 2.f * mu) - 2.f * c66;  // c12
            s.f2 = c13;
            s.f3 = (1.f + 2.f * eps) * lam;                              // c11c
            s.f4 = 2.f * (1.f + 2.f * eps) * mu;                         // c11b
            if (absorbing) s.f5 = f_pimp2(lam, mu, rho, eps);
        } else {
            const float lat = (PH == VTI) ? a.m[3][i] : lam;  // c13 on the top/bottom faces of VTI
            s.f1 = lat;
            s.f2 = lat;
            s.f3 = lam;
            s.f4 = 2.f * mu;
            if (absorbing) s.f5 = f_pimp(lam, mu, rho);
        }
    }
    return s;
}

template <int PH>
FWI_HD float elastic_face(const StepArgs &a, float acc, int c, int n, bool hi, int ix, int iy, int iz, int64_t so = 0)
{
    const float *cu[3] = {a.curr[0] + so, a.curr[1] + so, a.curr[2] + so};
    const Dims &g = a.g;
    const int64_t i = g.idx(ix, iy, iz);
    const bool absorbing = a.bc[2 * (n == 0 ? 1 : (n == 1 ? 2 : 0)) + (hi ? 1 : 0)] == BC_ABSORB;
    const SatTerm s = sat_coefs<PH>(a, n, c, i, absorbing);
    const float h0 = sbp().hq[0];
    float d1, d2, dn;
    // in1/in2 tangential axes and the fields they carry:
    //   n = z: in1 along x, in2 along y ; n = x: in1 along y, in2 along z ; n = y: in1 along x, in2 along z
    // tangential comp c: in(c-slot) = u_n ; normal comp: in1 = u_t1, in2 = u_t2, in3 = u_n
    // all samples are read unconditionally (valid addresses on every face),
    // so that their loads issue together; the coefficients select the terms
    float T1, T2, N0, S;
    if (n == 2) {
        d1 = a.dx; d2 = a.dy; dn = a.dz;
        const float *in1 = (c == 2) ? cu[0] : cu[2];
        const float *in2 = (c == 2) ? cu[1] : cu[2];
        T1 = d1_row(g.lx(in1, iy, iz), ix, g.nx);
        T2 = d1_row(g.ly(in2, ix, iz), iy, g.ny);
        const Line l3 = g.lz(cu[c], ix, iy);
        N0 = d1_wall(l3, g.nz, hi);
        S = sbound(l3, g.nz, hi);
    } else if (n == 0) {
        d1 = a.dy; d2 = a.dz; dn = a.dx;
        const float *in1 = (c == 0) ? cu[1] : cu[0];
        const float *in2 = (c == 0) ? cu[2] : cu[0];
        T1 = d1_row(g.ly(in1, ix, iz), iy, g.ny);
        T2 = d1_row(g.lz(in2, ix, iy), iz, g.nz);
        const Line l3 = g.lx(cu[c], iy, iz);
        N0 = d1_wall(l3, g.nx, hi);
        S = sbound(l3, g.nx, hi);
    } else {
        d1 = a.dx; d2 = a.dz; dn = a.dy;
        const float *in1 = (c == 1) ? cu[0] : cu[1];
        const float *in2 = (c == 1) ? cu[2] : cu[1];
        T1 = d1_row(g.lx(in1, iy, iz), ix, g.nx);
        T2 = d1_row(g.lz(in2, ix, iy), iz, g.nz);
        const Line l3 = g.ly(cu[c], ix, iz);
        N0 = d1_wall(l3, g.ny, hi);
        S = sbound(l3, g.ny, hi);
    }
    const float adh = (float)(1.0 / (double)(dn * h0));
    float v;
    if (!hi) {
        v = 0.f;
        if (s.f1 != 0.f) v = -s.f1 * T1 / d1;
        if (s.f2 != 0.f) v = v - s.f2 * T2 / d2;
        if (s.f3 != 0.f) v = v - s.f3 * N0 / dn;
    } else {
        v = 0.f;
        if (s.f1 != 0.f) v = s.f1 * T1 / d1;
        if (s.f2 != 0.f) v = v + s.f2 * T2 / d2;
        if (s.f3 != 0.f) v = v + s.f3 * N0 / dn;
    }
    v = v + s.f4 * S / dn;
    if (s.f5 != 0.f) v = v - s.f5 * prev_eff(a, c, i, ix, iy, iz, so) / a.dt;
    return acc - adh * v;
}

template <int PH>
FWI_HD float elastic_sat(const StepArgs &a, float acc, int c, int ix, int iy, int iz, int64_t so = 0)
{
    const Dims &g = a.g;
    // order of the reference: top, bottom, left, right, front, back
    if (iz == 0 && (a.bc[TOP] == BC_FREE || a.bc[TOP] == BC_ABSORB)) acc = elastic_face<PH>(a, acc, c, 2, false, ix, iy, iz, so);
    if (iz == g.nz - 1 && (a.bc[BOTTOM] == BC_FREE || a.bc[BOTTOM] == BC_ABSORB))
        acc = elastic_face<PH>(a, acc, c, 2, true, ix, iy, iz, so);
    if (ix == 0 && (a.bc[LEFT] == BC_FREE || a.bc[LEFT] == BC_ABSORB)) acc = elastic_face<PH>(a, acc, c, 0, false, ix, iy, iz, so);
    if (ix == g.nx - 1 && (a.bc[RIGHT] == BC_FREE || a.bc[RIGHT] == BC_ABSORB))
        acc = elastic_face<PH>(a, acc, c, 0, true, ix, iy, iz, so);
    if (iy == 0 && (a.bc[FRONT] == BC_FREE || a.bc[FRONT] == BC_ABSORB)) acc = elastic_face<PH>(a, acc, c, 1, false, ix, iy, iz, so);
    if (iy == g.ny - 1 && (a.bc[BACK] == BC_FREE || a.bc[BACK] == BC_ABSORB))
        acc = elastic_face<PH>(a, acc, c, 1, true, ix, iy, iz, so);
    return acc;
}

template <int PH>
FWI_HD float elastic_point(const StepArgs &a, int c, int ix, int iy, int iz)
{
    const int64_t i = a.g.idx(ix, iy, iz);
    float acc = elastic_acc<PH>(a, c, ix, iy, iz);
    acc = elastic_sat<PH>(a, acc, c, ix, iy, iz);
    const float dt2 = a.dt * a.dt;
    float v = dt2 * acc / a.m[2][i] + 2.f * a.curr[c][i] - prev_eff(a, c, i, ix, iy, iz);
    v = boundary_scale(a, v, c, ix, iy, iz);
    return taper(a, v, ix, iy, iz);
}

// Derivative pass (we_op.cpp:661-688 / 1312-1349): first derivatives of curr and
// the stress-like combinations whose derivatives the main pass takes.
struct AuxArgs {
    Dims g;
    float dx, dy, dz;
    const float *m[6];
    const float *curr[3];
    float *aux[9];
    float *dlag[3];  // optional: u_x[0], u_y[1], u_z[2] (kept for imaging), may be null
    int nyb;
    int y0, y1;
    int64_t sst, ast;
};

FWI_HD AuxArgs shot_args(const AuxArgs &a, int s)
{
    AuxArgs b = a;
    for (int c = 0; c < 3; c++)
        if (b.curr[c]) b.curr[c] += s * a.sst;
    for (int k = 0; k < 9; k++)
        if (b.aux[k]) b.aux[k] += s * a.ast;
    return b;
}

template <int PH>
FWI_HD void elastic_aux_point(const AuxArgs &a, int ix, int iy, int iz)
{
    const Dims &g = a.g;
    const int64_t i = g.idx(ix, iy, iz);
    const float ux0 = d1_row(g.lx(a.curr[0], iy, iz), ix, g.nx) / a.dx;
    const float uy1 = d1_row(g.ly(a.curr[1], ix, iz), iy, g.ny) / a.dy;
    const float uz2 = d1_row(g.lz(a.curr[2], ix, iy), iz, g.nz) / a.dz;
    const float lam = a.m[0][i];
    if (PH == ELASTIC) {
        a.aux[AUX_T0][i] = lam * (ux0 + uy1 + uz2);
    } else {
        const float mu = a.m[1][i], c13 = a.m[3][i], eps = a.m[4][i], c66 = a.m[5][i];
        const float c11c = (1.f + 2.f * eps) * lam;
        const float c12 = (1.f + 2.f * eps) * (lam + 2.f * mu) - 2.f * c66;
        a.aux[AUX_T0][i] = c11c * ux0 + c12 * uy1 + c13 * uz2;
        a.aux[AUX_T1][i] = c11c * uy1 + c12 * ux0 + c13 * uz2;
        a.aux[AUX_T2][i] = c13 * (ux0 + uy1) + lam * uz2;
    }
    a.aux[AUX_X1][i] = d1_row(g.lx(a.curr[1], iy, iz), ix, g.nx) / a.dx;
    a.aux[AUX_X2][i] = d1_row(g.lx(a.curr[2], iy, iz), ix, g.nx) / a.dx;
    a.aux[AUX_Y0][i] = d1_row(g.ly(a.curr[0], ix, iz), iy, g.ny) / a.dy;
    a.aux[AUX_Y2][i] = d1_row(g.ly(a.curr[2], ix, iz), iy, g.ny) / a.dy;
    a.aux[AUX_Z0][i] = d1_row(g.lz(a.curr[0], ix, iy), iz, g.nz) / a.dz;
    a.aux[AUX_Z1][i] = d1_row(g.lz(a.curr[1], ix, iy), iz, g.nz) / a.dz;
    if (a.dlag[0]) {
        a.dlag[0][i] = ux0;
        a.dlag[1][i] = uy1;
        a.dlag[2][i] = uz2;
    }
}

}  // namespace fwi
