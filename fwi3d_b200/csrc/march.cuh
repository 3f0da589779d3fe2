// Elastic time step (isotropic and VTI) as one marching kernel over every
// plane of the grid: for each output point it computes all operator terms of
// the reference's step (we_op.cpp:646-836, 1297-1497) -- D2var x9, D1 of the
// stress combinations, the six mixed mult_D terms -- then the leapfrog update,
// absorbing scaling and taper (the SAT of the faces is added by
// k_elastic_face_sat), reading each wavefield and model array from HBM once.
//
// Blocking: a CTA owns a TZ x TX tile of (z, x) columns (z = lanes, x = warps)
// and marches along y over a chunk of planes.  Shared memory holds
//   u   : an 8-plane ring of the displacement over the tile + 4-point halo,
//   yd  : a 6-plane ring of the own-column quantities differentiated along y
//         (stress combination, Dx u1, Dz u1) and the y coefficients,
//   dv  : the derived quantities of the output plane differentiated in x or z
//         (tile + 2-point halo), mp: the materials of that plane.
// Iteration q computes the own-column quantities of plane q and outputs plane
// q-2; the first four planes are output together at q = 5 and the last four
// at q = ny-1, when the 6-row SBP closures along y have all their samples.
// Tiles whose x (z) range keeps every stencil in the interior run the
// closure-free code (template flags XF, ZF); the first and last tiles of each
// axis (tile_range) hold the closure rows and use the general accessors.
//
// Every phase is a host/device function of (context, thread index), so a CPU
// harness can run the same code thread by thread between the barriers.
#pragma once

#include "fused.cuh"

namespace fwi {

namespace f3 {
constexpr int TZ = 32, TX = 16, NT = TZ * TX;
constexpr int HU = 4, ZU = TZ + 2 * HU, XU = TX + 2 * HU;  // displacement window
constexpr int HD = 2, ZD = TZ + 2 * HD, XD = TX + 2 * HD;  // derived window
constexpr int NR = 8;                                      // displacement ring (power of two)
constexpr int NY = 6;                                      // y-quantity ring
constexpr int USTR = 3 * XU * ZU;                          // floats between ring planes
}  // namespace f3

// y-ring fields: stress combination differentiated along y (T iso, T1 VTI),
// Dx u1, Dz u1, and the own-column coefficients mu, eps, c66.
enum { YD_T = 0, YD_X1 = 1, YD_Z1 = 2, YD_MU = 3, YD_EPS = 4, YD_C66 = 5, NYD = 6 };
// Derived fields of the output plane (iso stores T once, in T0).
enum { D3_T0 = 0, D3_T2 = 1, D3_Y0 = 2, D3_Z0 = 3, D3_X2 = 4, D3_Y2 = 5, ND3 = 6 };

namespace f3 {
constexpr int YF = TX * TZ;       // floats between y-ring fields
constexpr int YSTR = NYD * YF;    // floats between y-ring planes
}  // namespace f3

struct MarchSmem {
    float u[f3::NR][3][f3::XU][f3::ZU];
    float yd[f3::NY][NYD][f3::TX][f3::TZ];
    float dv[ND3][f3::XD][f3::ZD];
    float mp[2][NMP][f3::XD][f3::ZD];  // double-buffered: the next plane's arrive while this one is used
    float rows[SR_FLOATS];              // SBP closure rows, padded (SmemRows)
};

struct MarchCtx {
    const StepArgs *a;
    int64_t so;      // wavefield offset of this shot
    int x0, z0;      // tile origin
    int xend, zend;  // end of this tile's output rows
    int mb;          // materials buffer of the plane being output
    MarchSmem *sm;
    SmemRows rows{nullptr};  // closure rows in shared memory (MarchSmem::rows)
};

// Ring accessors along y (own column), indexed by global plane.
struct URing {
    const float *p;  // &u[0][k][xu][zu]
    FWI_HD float operator()(int k) const { return p[(k & (f3::NR - 1)) * f3::USTR]; }
};
struct YRing {
    const float *p;  // &yd[0][f][lx][lz]
    FWI_HD float operator()(int k) const { return p[(k % f3::NY) * f3::YSTR]; }
};

// ---------------------------------------------------------------------------
// Loads
// ---------------------------------------------------------------------------
template <bool INSIDE, bool ASYNC>
FWI_HD void m3_load_u(const MarchCtx &c, int tid, int q)
{
    const Dims &g = c.a->g;
    const int slot = q & (f3::NR - 1);
    for (int p = tid; p < f3::XU * f3::ZU; p += f3::NT) {
        const int xu = p / f3::ZU, zu = p - xu * f3::ZU;
        const int ix = c.x0 - f3::HU + xu, iz = c.z0 - f3::HU + zu;
        const bool in = INSIDE || (ix >= 0 && ix < g.nx && iz >= 0 && iz < g.nz);
        const int64_t i = c.so + (in ? g.idx(ix, q, iz) : 0);
#pragma unroll
        for (int k = 0; k < 3; k++) cpa4<ASYNC>(&c.sm->u[slot][k][xu][zu], c.a->curr[k] + i, in);
    }
}

template <int PH, bool INSIDE, bool ASYNC>
FWI_HD void m3_load_mat(const MarchCtx &c, int tid, int b, int y)
{
    const Dims &g = c.a->g;
    for (int p = tid; p < f3::XD * f3::ZD; p += f3::NT) {
        const int xd = p / f3::ZD, zd = p - xd * f3::ZD;
        const int ix = c.x0 - f3::HD + xd, iz = c.z0 - f3::HD + zd;
        const bool in = INSIDE || (ix >= 0 && ix < g.nx && iz >= 0 && iz < g.nz);
        const int64_t i = in ? g.idx(ix, y, iz) : 0;
        cpa4<ASYNC>(&c.sm->mp[b][MP_MU][xd][zd], c.a->m[1] + i, in);
        cpa4<ASYNC>(&c.sm->mp[b][MP_LAM][xd][zd], c.a->m[0] + i, in);
        if (PH == VTI) {
            cpa4<ASYNC>(&c.sm->mp[b][MP_C13][xd][zd], c.a->m[3] + i, in);
            cpa4<ASYNC>(&c.sm->mp[b][MP_EPS][xd][zd], c.a->m[4] + i, in);
            cpa4<ASYNC>(&c.sm->mp[b][MP_C66][xd][zd], c.a->m[5] + i, in);
        }
    }
}

// ---------------------------------------------------------------------------
// First derivatives of the displacement from the ring (with 1/h)
// ---------------------------------------------------------------------------
template <bool XF>
FWI_HD float m3_dx(const MarchCtx &c, int k, int slot, int xu, int zu)
{
    const float *p = &c.sm->u[slot][k][0][zu];
    const int ix = c.x0 - f3::HU + xu;
    if (XF || (ix >= 4 && ix < c.a->g.nx - 4)) {
        const SbpTables &t = sbp();
        return (t.d1c0 * (p[(xu + 1) * f3::ZU] - p[(xu - 1) * f3::ZU]) +
                t.d1c1 * (p[(xu + 2) * f3::ZU] - p[(xu - 2) * f3::ZU])) * c.a->idx;
    }
    return d1_row(SXc{p, c.x0 - f3::HU, f3::ZU, f3::XU}, ix, c.a->g.nx, c.rows) * c.a->idx;
}
template <bool ZF>
FWI_HD float m3_dz(const MarchCtx &c, int k, int slot, int xu, int zu)
{
    const float *p = &c.sm->u[slot][k][xu][0];
    const int iz = c.z0 - f3::HU + zu;
    if (ZF || (iz >= 4 && iz < c.a->g.nz - 4)) {
        const SbpTables &t = sbp();
        return (t.d1c0 * (p[zu + 1] - p[zu - 1]) + t.d1c1 * (p[zu + 2] - p[zu - 2])) * c.a->idz;
    }
    return d1_row(SZc{p, c.z0 - f3::HU, f3::ZU}, iz, c.a->g.nz, c.rows) * c.a->idz;
}
// Dy at plane q: interior taps from the ring, closure rows through the ring
// accessor (their samples 0..5 or ny-6..ny-1 are resident when used).
FWI_HD float m3_dy(const MarchCtx &c, int k, int q, int xu, int zu)
{
    const Dims &g = c.a->g;
    const float *p = &c.sm->u[0][k][xu][zu];
    if (q >= 4 && q < g.ny - 4) {
        const SbpTables &t = sbp();
        const int R = f3::NR - 1;
        return (t.d1c0 * (p[((q + 1) & R) * f3::USTR] - p[((q - 1) & R) * f3::USTR]) +
                t.d1c1 * (p[((q + 2) & R) * f3::USTR] - p[((q - 2) & R) * f3::USTR])) * c.a->idy;
    }
    return d1_row(URing{p}, q, g.ny, c.rows) * c.a->idy;
}

// ---------------------------------------------------------------------------
// Column phase: own-column y quantities of plane q into the y ring
// ---------------------------------------------------------------------------
template <int PH, bool XF, bool ZF>
FWI_HD void m3_column(const MarchCtx &c, int tid, int q)
{
    const Dims &g = c.a->g;
    const int lz = tid % f3::TZ, lx = tid / f3::TZ;
    const int ix = c.x0 + lx, iz = c.z0 + lz;
    const int xu = lx + f3::HU, zu = lz + f3::HU;
    const int s = q & (f3::NR - 1);
    float(*yd)[f3::TX][f3::TZ] = c.sm->yd[q % f3::NY];
    const int64_t i = g.idx(ix, q, iz);
    const float mu = c.a->m[1][i], lam = c.a->m[0][i];
    const float ux0 = m3_dx<XF>(c, 0, s, xu, zu);
    const float uy1 = m3_dy(c, 1, q, xu, zu);
    const float uz2 = m3_dz<ZF>(c, 2, s, xu, zu);
    const float ux1 = m3_dx<XF>(c, 1, s, xu, zu);
    const float uz1 = m3_dz<ZF>(c, 1, s, xu, zu);
    yd[YD_MU][lx][lz] = mu;
    if (PH == ELASTIC) {
        yd[YD_T][lx][lz] = lam * (ux0 + uy1 + uz2);
    } else {
        const float c13 = c.a->m[3][i], eps = c.a->m[4][i], c66 = c.a->m[5][i];
        yd[YD_EPS][lx][lz] = eps;
        yd[YD_C66][lx][lz] = c66;
        const float c11c = (1.f + 2.f * eps) * lam;
        const float c12 = (1.f + 2.f * eps) * (lam + 2.f * mu) - 2.f * c66;
        yd[YD_T][lx][lz] = c11c * uy1 + c12 * ux0 + c13 * uz2;
    }
    yd[YD_X1][lx][lz] = ux1;
    yd[YD_Z1][lx][lz] = uz1;
}

// ---------------------------------------------------------------------------
// Derived phase: quantities of plane y differentiated in x or z, over the
// tile and a 2-point halo
// ---------------------------------------------------------------------------
template <int PH, bool XF, bool ZF>
FWI_HD void m3_derived(const MarchCtx &c, int tid, int y)
{
    const Dims &g = c.a->g;
    const int s = y & (f3::NR - 1);
    constexpr int STR = f3::XD * f3::ZD;
    for (int p = tid; p < f3::XD * f3::ZD; p += f3::NT) {
        const int xd = p / f3::ZD, zd = p - xd * f3::ZD;
        const int ix = c.x0 - f3::HD + xd, iz = c.z0 - f3::HD + zd;
        float *dv0 = &c.sm->dv[0][xd][zd];
        if (!(XF && ZF) && (ix < 0 || ix >= g.nx || iz < 0 || iz >= g.nz)) {
#pragma unroll
            for (int k = 0; k < ND3; k++) dv0[k * STR] = 0.f;
            continue;
        }
        const int xu = xd + (f3::HU - f3::HD), zu = zd + (f3::HU - f3::HD);
        const float ux0 = m3_dx<XF>(c, 0, s, xu, zu);
        const float uy1 = m3_dy(c, 1, y, xu, zu);
        const float uz2 = m3_dz<ZF>(c, 2, s, xu, zu);
        const float lam = c.sm->mp[c.mb][MP_LAM][xd][zd];
        if (PH == ELASTIC) {
            dv0[D3_T0 * STR] = lam * (ux0 + uy1 + uz2);
        } else {
            const float mu = c.sm->mp[c.mb][MP_MU][xd][zd];
            const float c13 = c.sm->mp[c.mb][MP_C13][xd][zd], eps = c.sm->mp[c.mb][MP_EPS][xd][zd];
            const float c66 = c.sm->mp[c.mb][MP_C66][xd][zd];
            const float c11c = (1.f + 2.f * eps) * lam;
            const float c12 = (1.f + 2.f * eps) * (lam + 2.f * mu) - 2.f * c66;
            dv0[D3_T0 * STR] = c11c * ux0 + c12 * uy1 + c13 * uz2;
            dv0[D3_T2 * STR] = c13 * (ux0 + uy1) + lam * uz2;
        }
        dv0[D3_Y0 * STR] = m3_dy(c, 0, y, xu, zu);
        dv0[D3_Z0 * STR] = m3_dz<ZF>(c, 0, s, xu, zu);
        dv0[D3_X2 * STR] = m3_dx<XF>(c, 2, s, xu, zu);
        dv0[D3_Y2 * STR] = m3_dy(c, 2, y, xu, zu);
    }
}

// ---------------------------------------------------------------------------
// Output phase: all operator terms at the own point of plane y, update
// ---------------------------------------------------------------------------
// In-plane unscaled D1 of a derived line, and of a derived*coefficient line.
template <bool F, class L>
FWI_HD float m3_d1(const L &s, int i, int n, const SmemRows &rows)
{
    if (F) return d1i(s(i - 2), s(i - 1), s(i + 1), s(i + 2));
    return d1_row(s, i, n, rows);
}
template <bool F, class L, class M>
FWI_HD float m3_d1p(const L &s, const M &m, int i, int n, const SmemRows &rows)
{
    if (F) return d1m(s(i - 2), m(i - 2), s(i - 1), m(i - 1), s(i + 1), m(i + 1), s(i + 2), m(i + 2));
    return d1_prod_row(s, m, i, n, rows);
}

template <int PH, bool XF, bool ZF>
FWI_HD void m3_output(const MarchCtx &c, int tid, int y)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    const int lz = tid % f3::TZ, lx = tid / f3::TZ;
    const int ix = c.x0 + lx, iz = c.z0 + lz;
    if (ix >= c.xend || iz >= c.zend) return;
    const int64_t i = g.idx(ix, y, iz);
    const bool xin = XF || (ix >= 6 && ix < g.nx - 6);
    const bool zin = ZF || (iz >= 6 && iz < g.nz - 6);
    const bool yin = y >= 6 && y < g.ny - 6;
    const bool yd1 = y >= 4 && y < g.ny - 4;
    const int xu = lx + f3::HU, zu = lz + f3::HU;
    const int xd = lx + f3::HD, zd = lz + f3::HD;
    const MarchSmem &s = *c.sm;
    const int R = f3::NR - 1;
    const int s0 = y & R;
    const float idx2 = a.ad1[0], idy2 = a.ad1[1];
    // y-ring slots of planes y-2..y+2 (interior rows)
    const float *ydb = &s.yd[0][0][lx][lz];
    const int ysl[5] = {((y + f3::NY - 2) % f3::NY) * f3::YSTR, ((y + f3::NY - 1) % f3::NY) * f3::YSTR,
                        (y % f3::NY) * f3::YSTR, ((y + 1) % f3::NY) * f3::YSTR, ((y + 2) % f3::NY) * f3::YSTR};
    auto ydv = [&](int f, int k) { return ydb[ysl[k] + f * f3::YF]; };
    const int64_t col = g.idx(ix, 0, iz);
    const int64_t ystr = (int64_t)g.nx * g.nz;
    const float *pu0 = &s.u[0][0][xu][zu];
    auto uy = [&](int k, int p) { return pu0[(p & R) * f3::USTR + k * f3::XU * f3::ZU]; };

    const SX mux{&s.mp[c.mb][MP_MU][0][zd], c.x0 - f3::HD, f3::ZD};
    const SZ muz{&s.mp[c.mb][MP_MU][xd][0], c.z0 - f3::HD};
    float acc[3];
    if (PH == ELASTIC) {
        W5 wx{}, wz{}, wy{};
        W8 wxc{}, wzc{}, wyc{};
        if (xin) wx = d2w(mux(ix - 2), mux(ix - 1), mux(ix), mux(ix + 1), mux(ix + 2));
        else wxc = d2closure_w(a.w2c[0][0], (int64_t)y * g.nz + iz, mux, ix, g.nx, c.rows);
        if (zin) wz = d2w(muz(iz - 2), muz(iz - 1), muz(iz), muz(iz + 1), muz(iz + 2));
        else wzc = d2closure_w(a.w2c[2][0], (int64_t)y * g.nx + ix, muz, iz, g.nz, c.rows);
        if (yin) wy = d2w(ydv(YD_MU, 0), ydv(YD_MU, 1), ydv(YD_MU, 2), ydv(YD_MU, 3), ydv(YD_MU, 4));
        else wyc = d2closure_w(a.w2c[1][0], (int64_t)ix * g.nz + iz, Line{a.m[1], col, ystr}, y, g.ny, c.rows);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float adx = k == 0 ? a.ad2[0] : a.ad1[0];
            const float ady = k == 1 ? a.ad2[1] : a.ad1[1];
            const float adz = k == 2 ? a.ad2[2] : a.ad1[2];
            const SX ul{&s.u[s0][k][0][zu], c.x0 - f3::HU, f3::ZU};
            const SZ uzl{&s.u[s0][k][xu][0], c.z0 - f3::HU};
            float v = xin ? d2apply(wx, adx, ul(ix - 2), ul(ix - 1), ul(ix), ul(ix + 1), ul(ix + 2))
                          : d2closure_apply(wxc, ul, ix, g.nx, adx);
            if (yin) v += d2apply(wy, ady, uy(k, y - 2), uy(k, y - 1), uy(k, y), uy(k, y + 1), uy(k, y + 2));
            else v += d2closure_apply(wyc, Line{a.curr[k] + c.so, col, ystr}, y, g.ny, ady);
            v += zin ? d2apply(wz, adz, uzl(iz - 2), uzl(iz - 1), uzl(iz), uzl(iz + 1), uzl(iz + 2))
                     : d2closure_apply(wzc, uzl, iz, g.nz, adz);
            acc[k] = v;
        }
    } else {
        const C11bS<SX, SX> bx{SX{&s.mp[c.mb][MP_EPS][0][zd], c.x0 - f3::HD, f3::ZD}, mux};
        const SX c6x{&s.mp[c.mb][MP_C66][0][zd], c.x0 - f3::HD, f3::ZD};
        W5 wxb{}, wx6{}, wxm{}, wz{}, wyb{}, wy6{}, wym{};
        if (xin) {
            wxb = d2w(bx(ix - 2), bx(ix - 1), bx(ix), bx(ix + 1), bx(ix + 2));
            wx6 = d2w(c6x(ix - 2), c6x(ix - 1), c6x(ix), c6x(ix + 1), c6x(ix + 2));
            wxm = d2w(mux(ix - 2), mux(ix - 1), mux(ix), mux(ix + 1), mux(ix + 2));
        }
        if (zin) wz = d2w(muz(iz - 2), muz(iz - 1), muz(iz), muz(iz + 1), muz(iz + 2));
        if (yin) {
            float qb[5];
#pragma unroll
            for (int k = 0; k < 5; k++) qb[k] = 2.f * (1.f + 2.f * ydv(YD_EPS, k)) * ydv(YD_MU, k);
            wyb = d2w(qb[0], qb[1], qb[2], qb[3], qb[4]);
            wy6 = d2w(ydv(YD_C66, 0), ydv(YD_C66, 1), ydv(YD_C66, 2), ydv(YD_C66, 3), ydv(YD_C66, 4));
            wym = d2w(ydv(YD_MU, 0), ydv(YD_MU, 1), ydv(YD_MU, 2), ydv(YD_MU, 3), ydv(YD_MU, 4));
        }
        const Line muy{a.m[1], col, ystr}, epsy{a.m[4], col, ystr}, c6y{a.m[5], col, ystr};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const W5 &wx = k == 0 ? wxb : (k == 1 ? wx6 : wxm);
            const W5 &wy = k == 0 ? wy6 : (k == 1 ? wyb : wym);
            const float adz = k == 2 ? a.ad2[2] : a.ad1[2];
            const SX ul{&s.u[s0][k][0][zu], c.x0 - f3::HU, f3::ZU};
            const SZ uzl{&s.u[s0][k][xu][0], c.z0 - f3::HU};
            float v;
            if (xin) v = d2apply(wx, idx2, ul(ix - 2), ul(ix - 1), ul(ix), ul(ix + 1), ul(ix + 2));
            else if (k == 0) v = d2var_tab(a.w2c[0][2], (int64_t)y * g.nz + iz, ul, bx, ix, g.nx, idx2, c.rows);
            else if (k == 1) v = d2var_tab(a.w2c[0][1], (int64_t)y * g.nz + iz, ul, c6x, ix, g.nx, idx2, c.rows);
            else v = d2var_tab(a.w2c[0][0], (int64_t)y * g.nz + iz, ul, mux, ix, g.nx, idx2, c.rows);
            if (yin) {
                v += d2apply(wy, idy2, uy(k, y - 2), uy(k, y - 1), uy(k, y), uy(k, y + 1), uy(k, y + 2));
            } else {
                const Line ucol{a.curr[k] + c.so, col, ystr};
                if (k == 0) v += d2var_tab(a.w2c[1][1], (int64_t)ix * g.nz + iz, ucol, c6y, y, g.ny, idy2, c.rows);
                else if (k == 1) v += d2var_tab(a.w2c[1][2], (int64_t)ix * g.nz + iz, ucol, C11bLine{epsy, muy}, y, g.ny, idy2, c.rows);
                else v += d2var_tab(a.w2c[1][0], (int64_t)ix * g.nz + iz, ucol, muy, y, g.ny, idy2, c.rows);
            }
            v += zin ? d2apply(wz, adz, uzl(iz - 2), uzl(iz - 1), uzl(iz), uzl(iz + 1), uzl(iz + 2))
                     : d2var_tab(a.w2c[2][0], (int64_t)y * g.nx + ix, uzl, muz, iz, g.nz, adz, c.rows);
            acc[k] = v;
        }
    }

    // ---- D1 of the stress combinations and the mixed terms (we_op.cpp:661-688, 1312-1349) ----
    const SX Px = (PH == VTI) ? SX{&s.mp[c.mb][MP_C66][0][zd], c.x0 - f3::HD, f3::ZD} : mux;
    const int PY = (PH == VTI) ? YD_C66 : YD_MU;
    const SX dT0x{&s.dv[D3_T0][0][zd], c.x0 - f3::HD, f3::ZD};
    const SZ dT2z{&s.dv[PH == ELASTIC ? D3_T0 : D3_T2][xd][0], c.z0 - f3::HD};
    const SX dY0x{&s.dv[D3_Y0][0][zd], c.x0 - f3::HD, f3::ZD};
    const SX dZ0x{&s.dv[D3_Z0][0][zd], c.x0 - f3::HD, f3::ZD};
    const SZ dX2z{&s.dv[D3_X2][xd][0], c.z0 - f3::HD};
    const SZ dY2z{&s.dv[D3_Y2][xd][0], c.z0 - f3::HD};
    float dyX1, dyT, dyZ1;
    if (yd1) {
        dyX1 = d1m(ydv(YD_X1, 0), ydv(PY, 0), ydv(YD_X1, 1), ydv(PY, 1), ydv(YD_X1, 3), ydv(PY, 3), ydv(YD_X1, 4),
                   ydv(PY, 4));
        dyT = d1i(ydv(YD_T, 0), ydv(YD_T, 1), ydv(YD_T, 3), ydv(YD_T, 4));
        dyZ1 = d1m(ydv(YD_Z1, 0), ydv(YD_MU, 0), ydv(YD_Z1, 1), ydv(YD_MU, 1), ydv(YD_Z1, 3), ydv(YD_MU, 3),
                   ydv(YD_Z1, 4), ydv(YD_MU, 4));
    } else {
        dyX1 = d1_prod_row(YRing{ydb + YD_X1 * f3::YF}, YRing{ydb + PY * f3::YF}, y, g.ny, c.rows);
        dyT = d1_row(YRing{ydb + YD_T * f3::YF}, y, g.ny, c.rows);
        dyZ1 = d1_prod_row(YRing{ydb + YD_Z1 * f3::YF}, YRing{ydb + YD_MU * f3::YF}, y, g.ny, c.rows);
    }
    // comp 0: Dx(T0)/dx + Dy(P u_x1)/dy + Dz(mu u_x2)/dy (dy as in the reference, we_op.cpp:678)
    acc[0] += m3_d1<XF>(dT0x, ix, g.nx, c.rows) * a.idx;
    acc[0] += dyX1 * a.idy;
    acc[0] += m3_d1p<ZF>(dX2z, muz, iz, g.nz, c.rows) * a.idy;
    // comp 1: Dy(T1)/dy + Dx(P u_y0)/dx + Dz(mu u_y2)/dz
    acc[1] += dyT * a.idy;
    acc[1] += m3_d1p<XF>(dY0x, Px, ix, g.nx, c.rows) * a.idx;
    acc[1] += m3_d1p<ZF>(dY2z, muz, iz, g.nz, c.rows) * a.idz;
    // comp 2: Dz(T2)/dz + Dx(mu u_z0)/dx + Dy(mu u_z1)/dy
    acc[2] += m3_d1<ZF>(dT2z, iz, g.nz, c.rows) * a.idz;
    acc[2] += m3_d1p<XF>(dZ0x, mux, ix, g.nx, c.rows) * a.idx;
    acc[2] += dyZ1 * a.idy;

    // ---- update, scaling, taper (SAT is added by the face kernel) ----
    const float dt2 = a.dt * a.dt;
    const float irho = 1.0f / a.m[2][i];
    const bool face = ix == 0 || ix == g.nx - 1 || iz == 0 || iz == g.nz - 1 || y == 0 || y == g.ny - 1;
    const bool tz = in_taper(a, ix, y, iz);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float p = a.prev[k][c.so + i];
        const float pe = (a.taper_prev && tz) ? taper(a, p, ix, y, iz) : p;
        float v = dt2 * acc[k] * irho + 2.f * uy(k, y) - pe;
        if (face) v = boundary_scale(a, v, k, ix, y, iz);
        if (tz) v = taper(a, v, ix, y, iz);
        a.next[k][c.so + i] = v;
    }
}

// ---------------------------------------------------------------------------
// The march of one CTA over output planes [ya, yb)
// ---------------------------------------------------------------------------
// Output planes of iteration q: the first four at q = 5, the last four at
// q = ny-1, every other plane y at q = y+2.  Returns the count, planes in out[].
FWI_HD int m3_outputs(int q, int ny, int ya, int yb, int *out)
{
    int n = 0;
    if (q == 5) {
        for (int y = 0; y < 4; y++)
            if (y >= ya && y < yb) out[n++] = y;
    } else if (q == ny - 1) {
        for (int y = ny - 4; y < ny; y++)
            if (y >= ya && y < yb) out[n++] = y;
    }
    const int y = q - 2;
    if (y >= 4 && y < ny - 4 && y >= ya && y < yb) out[n++] = y;
    return n;
}
// Highest displacement plane iteration q reads.
FWI_HD int m3_need(int q, int ny)
{
    if (q < 4) return 5;
    if (q >= ny - 4) return ny - 1;
    return q + 2;
}
// Iterations of a chunk: chunk boundaries other than 0 and ny lie in [6, ny-6].
FWI_HD void m3_range(int ny, int ya, int yb, int &q0, int &q1)
{
    q0 = ya == 0 ? 0 : ya - 2;
    q1 = yb == ny ? ny - 1 : yb + 1;
}

// Lowest displacement plane iteration q reads (column phase and outputs).
FWI_HD int m3_lowest(int q, int ny, const int *out, int nout)
{
    auto lo = [&](int p) { return p < 4 ? 0 : (p >= ny - 4 ? ny - 6 : p - 2); };
    int low = lo(q);
    for (int k = 0; k < nout; k++) low = lo(out[k]) < low ? lo(out[k]) : low;
    return low;
}

// Runs the march with `par(phase)`: every thread of the block runs phase(tid),
// then the block synchronises.  While iteration q computes, the displacement
// planes and the materials that iteration q+1 needs are copied in
// asynchronously, into ring slots and a materials buffer q does not read.
template <int PH, bool XF, bool ZF, class Par>
FWI_HD void m3_march(MarchCtx c, int ya, int yb, Par &&par)
{
    constexpr bool IN = XF && ZF;
    const int ny = c.a->g.ny;
    int q0, q1;
    m3_range(ny, ya, yb, q0, q1);
    int loaded = (q0 == 0 ? 0 : q0 - 2) - 1;  // highest plane loaded or in flight
    int mb = 0;                                // materials buffer of the next output
    int mp_plane = -1;                         // plane whose materials are in flight into mb
    for (int q = q0; q <= q1; q++) {
        int out[5];
        const int nout = m3_outputs(q, ny, ya, yb, out);
        const int need = m3_need(q, ny);
        const int lo = loaded + 1;
        loaded = need > loaded ? need : loaded;
        const bool have_mp = nout && mp_plane == out[0];
        par([&](int tid) {
            cpa_wait();
            for (int p = lo; p <= need; p++) m3_load_u<IN, false>(c, tid, p);
            if (nout && !have_mp) m3_load_mat<PH, IN, false>(c, tid, mb, out[0]);
        });
        // copies for iteration q+1
        int pf_hi = loaded, nn = 0, nout1[5];
        if (q < q1) {
            const int need1 = m3_need(q + 1, ny), low = m3_lowest(q, ny, out, nout);
            while (pf_hi < need1 && pf_hi + 1 - f3::NR < low) pf_hi++;
            nn = m3_outputs(q + 1, ny, ya, yb, nout1);
        }
        const int pf_lo = loaded + 1;
        const int nmb = (mb + nout) & 1;
        const bool pf_mp = nn > 0 && nout <= 1;
        c.mb = mb;
        par([&](int tid) {
            for (int p = pf_lo; p <= pf_hi; p++) m3_load_u<IN, true>(c, tid, p);
            if (pf_mp) m3_load_mat<PH, IN, true>(c, tid, nmb, nout1[0]);
            cpa_commit();
            m3_column<PH, XF, ZF>(c, tid, q);
            if (nout) m3_derived<PH, XF, ZF>(c, tid, out[0]);
        });
        loaded = pf_hi;
        for (int k = 0; k < nout; k++) {
            c.mb = (mb + k) & 1;
            if (k > 0) {
                par([&](int tid) { m3_load_mat<PH, IN, false>(c, tid, c.mb, out[k]); });
                par([&](int tid) { m3_derived<PH, XF, ZF>(c, tid, out[k]); });
            }
            par([&](int tid) { m3_output<PH, XF, ZF>(c, tid, out[k]); });
        }
        mb = nmb;
        mp_plane = pf_mp ? nout1[0] : -1;
    }
    par([&](int) { cpa_wait(); });
}

// Chunk of planes [ya, yb) of chunk ch of nch along ny: interior boundaries
// are spread evenly over [6, ny-6].
FWI_HD void m3_chunk(int ny, int ch, int nch, int &ya, int &yb)
{
    auto bound = [&](int k) {
        if (k <= 0) return 0;
        if (k >= nch) return ny;
        return 6 + (int)((int64_t)(ny - 12) * k / nch);
    };
    ya = bound(ch);
    yb = bound(ch + 1);
}

// x (z) tile flag: every stencil of the tile's outputs and derived halo is interior.
FWI_HD bool m3_fast(int origin, int n, int T) { return origin >= 6 && origin + T <= n - 6; }

}  // namespace fwi
