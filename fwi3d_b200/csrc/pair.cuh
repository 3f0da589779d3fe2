// Isotropic elastic step on the interior tiles, two z-adjacent points per
// thread in packed FP32 pairs.
//
// Same tiling, ring and bulk-tensor plane copies as the fused kernel
// (fused.cuh): a CTA owns a TZ x TX = 32 x 16 tile of (z, x) columns whose
// outputs and derived halo hold no SBP closure row along x or z, and marches
// along y over planes of [6, ny-6).  Here a thread owns the pair (z, z+1) of
// one x row, so a CTA has 256 threads: lanes 0-15 of a warp cover row 2w,
// lanes 16-31 row 2w+1, and each half-warp reads 16 consecutive pairs (128
// contiguous bytes) per shared-memory access.
//
// Arithmetic on the pair uses the packed FP32 instructions of sm_100
// (fma/mul/add/sub .f32x2): one instruction advances both points, so the
// floating-point work costs half the issue slots of the scalar kernel.  Taps
// along x and y are whole 8-byte pairs; taps along z at odd offsets are
// re-paired from the two neighbouring pairs.
//
// Per plane y the work is organised to read each tap once:
//   column  (plane y+2, own pair): lambda div u, mu Dx u1, mu Dz u1 pushed into
//           register queues (their y derivatives at y);
//   phase B (plane y, own pair):   the nine D2var terms accumulated in
//           registers from the x, y and z taps of the three components, and
//           from the same taps the derived values lambda div u, mu Dy u0,
//           mu Dz u0, mu Dx u2, mu Dy u2 written to the derived planes;
//           96 threads also form the derived values of the tile's halo
//           (two rows on each x side, one pair on each z side);
//   phase C (plane y, own pair):   the nine first derivatives of the derived
//           planes and queues, then the leapfrog update and taper.
// The operator terms and their order follow the reference's step
// (we_op.cpp:646-688); products with mu are formed per tap as in mult_D
// (spatial_operators.cpp:300-406), first derivatives multiply by 1/h instead
// of dividing, and the a/h^2 factor of the D2var terms is folded into the
// weights (rounding differences of a few ulp per term).
#pragma once

#include <cmath>

#include "fused.cuh"

namespace fwi {

namespace pz {
constexpr int TZ = fz::TZ, TX = fz::TX;
constexpr int NPR = TZ / 2;   // pairs per x row
constexpr int NT = NPR * TX;  // 256 threads
}  // namespace pz

// ---------------------------------------------------------------------------
// Packed FP32 pairs.  On the GPU a pair lives in one 64-bit register pair and
// the arithmetic is one .f32x2 instruction; on the host it is two floats.
// ---------------------------------------------------------------------------
struct F2 {
#if defined(__CUDA_ARCH__)
    unsigned long long v;
#else
    float x, y;
#endif
};

FWI_HD F2 f2(float a, float b)
{
    F2 r;
#if defined(__CUDA_ARCH__)
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
#else
    r.x = a;
    r.y = b;
#endif
    return r;
}
FWI_HD F2 f2s(float a) { return f2(a, a); }
FWI_HD float f2lo(F2 p)
{
#if defined(__CUDA_ARCH__)
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(p.v));
    return a;
#else
    return p.x;
#endif
}
FWI_HD float f2hi(F2 p)
{
#if defined(__CUDA_ARCH__)
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(p.v));
    return b;
#else
    return p.y;
#endif
}
// (a.hi, b.lo): the pair one sample further than a, from a and the next pair b
FWI_HD F2 f2mid(F2 a, F2 b) { return f2(f2hi(a), f2lo(b)); }

FWI_HD F2 add2(F2 a, F2 b)
{
#if defined(__CUDA_ARCH__)
    F2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
#else
    return F2{a.x + b.x, a.y + b.y};
#endif
}
FWI_HD F2 sub2(F2 a, F2 b)
{
#if defined(__CUDA_ARCH__)
    F2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
#else
    return F2{a.x - b.x, a.y - b.y};
#endif
}
FWI_HD F2 mul2(F2 a, F2 b)
{
#if defined(__CUDA_ARCH__)
    F2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
#else
    return F2{a.x * b.x, a.y * b.y};
#endif
}
// a*b + c with one rounding per element
FWI_HD F2 fma2(F2 a, F2 b, F2 c)
{
#if defined(__CUDA_ARCH__)
    F2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
#else
    return F2{std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y)};
#endif
}
// correctly rounded reciprocal (1.0f / x)
FWI_HD float rcp_rn(float x)
{
#if defined(__CUDA_ARCH__)
    return __frcp_rn(x);
#else
    return 1.0f / x;
#endif
}
// 8-byte shared/global accesses of a pair (p 8-byte aligned)
FWI_HD F2 ld2(const float *p)
{
#if defined(__CUDA_ARCH__)
    F2 r;
    r.v = *reinterpret_cast<const unsigned long long *>(p);
    return r;
#else
    return F2{p[0], p[1]};
#endif
}
FWI_HD void st2(float *p, F2 v)
{
#if defined(__CUDA_ARCH__)
    *reinterpret_cast<unsigned long long *>(p) = v.v;
#else
    p[0] = v.x;
    p[1] = v.y;
#endif
}
// global pair: one 8-byte access when the pair is 8-byte aligned (EVEN), else two
template <bool EVEN>
FWI_HD F2 ldg2(const float *p)
{
    if (EVEN) return ld2(p);
    return f2(p[0], p[1]);
}
template <bool EVEN>
FWI_HD void stg2(float *p, F2 v)
{
    if (EVEN) {
        st2(p, v);
    } else {
        p[0] = f2lo(v);
        p[1] = f2hi(v);
    }
}

// Interior D2var weights of a pair from the coefficient taps f(i-2..i+2) of
// each point (the reference's grouping, spatial_operators.hpp:37, 200-229),
// scaled by s = a/h^2.
struct W5p {
    F2 w0, wm1, wp1, wm2, wp2;
};
FWI_HD W5p d2w_pair(F2 fm2, F2 fm1, F2 f0, F2 fp1, F2 fp2, F2 s)
{
    const float *c = sbp().d2in;
    W5p w;
    w.w0 = fma2(f2s(c[2]), add2(fm2, fp2), fma2(f2s(c[1]), add2(fm1, fp1), mul2(f2s(c[0]), f0)));
    w.wm1 = fma2(f2s(c[6]), fp1, fma2(f2s(c[5]), f0, fma2(f2s(c[4]), fm1, mul2(f2s(c[3]), fm2))));
    w.wp1 = fma2(f2s(c[6]), fm1, fma2(f2s(c[5]), f0, fma2(f2s(c[4]), fp1, mul2(f2s(c[3]), fp2))));
    w.wm2 = fma2(f2s(c[9]), f0, fma2(f2s(c[8]), fm1, mul2(f2s(c[7]), fm2)));
    w.wp2 = fma2(f2s(c[9]), f0, fma2(f2s(c[8]), fp1, mul2(f2s(c[7]), fp2)));
    w.w0 = mul2(w.w0, s);
    w.wm1 = mul2(w.wm1, s);
    w.wp1 = mul2(w.wp1, s);
    w.wm2 = mul2(w.wm2, s);
    w.wp2 = mul2(w.wp2, s);
    return w;
}
// sum of the five weighted taps, added to acc
FWI_HD F2 d2acc(const W5p &w, F2 um2, F2 um1, F2 u0, F2 up1, F2 up2, F2 acc)
{
    acc = fma2(w.w0, u0, acc);
    acc = fma2(w.wm1, um1, acc);
    acc = fma2(w.wp1, up1, acc);
    acc = fma2(w.wm2, um2, acc);
    return fma2(w.wp2, up2, acc);
}
// interior first derivative (coefficients pre-multiplied by 1/h: c0h, c1h)
FWI_HD F2 d1p(F2 am2, F2 am1, F2 ap1, F2 ap2, F2 c0h, F2 c1h)
{
    return fma2(c1h, sub2(ap2, am2), mul2(c0h, sub2(ap1, am1)));
}
// the same derivative added to acc
FWI_HD F2 d1acc(F2 am2, F2 am1, F2 ap1, F2 ap2, F2 c0h, F2 c1h, F2 acc)
{
    return fma2(c1h, sub2(ap2, am2), fma2(c0h, sub2(ap1, am1), acc));
}
// z taps of a pair at p (z, z+1): m = (z-2, z-1), a = (z, z+1), b = (z+2, z+3)
struct ZT {
    F2 m, a, b;
    FWI_HD F2 m1() const { return f2mid(m, a); }  // (z-1, z)
    FWI_HD F2 p1() const { return f2mid(a, b); }  // (z+1, z+2)
};
FWI_HD ZT ztaps(const float *p) { return ZT{ld2(p - 2), ld2(p), ld2(p + 2)}; }

// Per-thread queues along y (planes y-2 .. y+2 of the own pair).
struct PairThread {
    F2 qmu[5];  // mu
    F2 qT[5];   // lambda div u
    F2 qX1[5];  // mu Dx u1
    F2 qZ1[5];  // mu Dz u1
};

// Constants of a launch as pairs.
struct PairK {
    F2 cx0, cx1, cy0, cy1, cz0, cz1;  // D1 interior weights times 1/h per axis
    F2 sx1, sy1, sz1;                 // a/h^2 with a = 1 per axis
};
FWI_HD PairK pair_consts(const StepArgs &a)
{
    const SbpTables &t = sbp();
    PairK k;
    k.cx0 = f2s(t.d1c0 * a.idx);
    k.cx1 = f2s(t.d1c1 * a.idx);
    k.cy0 = f2s(t.d1c0 * a.idy);
    k.cy1 = f2s(t.d1c1 * a.idy);
    k.cz0 = f2s(t.d1c0 * a.idz);
    k.cz1 = f2s(t.d1c1 * a.idz);
    k.sx1 = f2s(a.ad1[0]);
    k.sy1 = f2s(a.ad1[1]);
    k.sz1 = f2s(a.ad1[2]);
    return k;
}

// Ring pointer of (slot, component) at window position (xw, zw).
FWI_HD const float *pz_u(const FusedCtx &c, int slot, int k, int xw, int zw)
{
    return &c.sm->u[slot][k][xw][zw];
}

// Phase A without bulk-tensor copies: plane q (tile + 4 halo) into its ring
// slot by per-thread 4-byte copies (asynchronous with ASYNC).
template <bool ASYNC>
FWI_HD void pz_load_u(FusedCtx &c, int tid, int q, int slot)
{
    const Dims &g = c.a->g;
    for (int p = tid; p < fz::XW * fz::ZW; p += pz::NT) {
        const int xw = p / fz::ZW, zw = p - xw * fz::ZW;
        const int ix = c.x0 - fz::HW + xw, iz = c.z0 - fz::HW + zw;
        const bool in = ix >= 0 && ix < g.nx && iz >= 0 && iz < g.nz;
        const int64_t i = c.so + (in ? g.idx(ix, q, iz) : 0);
        for (int k = 0; k < 3; k++) cpa4<ASYNC>(&c.sm->u[slot][k][xw][zw], c.a->curr[k] + i, in);
    }
}

// One 8-byte global->shared copy (both addresses 8-byte aligned):
// asynchronous on the GPU (cp.async), a plain copy on the host.
template <bool ASYNC>
FWI_HD void cpa8(float *dst, const float *src)
{
#if defined(__CUDA_ARCH__)
    if (ASYNC) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
        return;
    }
#endif
    dst[0] = src[0];
    dst[1] = src[1];
}

// Material planes mu, lambda at y over the derived region, as pairs; with
// ASYNC the copies are asynchronous (waited for with cpa_wait).
template <bool EVEN, bool ASYNC>
FWI_HD void pz_load_mat(FusedCtx &c, int tid, int y)
{
    const Dims &g = c.a->g;
    constexpr int NP = fz::ZH / 2;  // 18 pairs per row
    for (int p = tid; p < fz::XH * NP; p += pz::NT) {
        const int xh = p / NP, zh = 2 * (p - xh * NP);
        const int ix = c.x0 - fz::HD + xh, iz = c.z0 - fz::HD + zh;
        // interior tiles: every position of the derived region is inside the grid
        const int64_t i = g.idx(ix, y, iz);
        float *dm = &fz_mpp(c.sm, MP_MU)[xh][zh], *dl = &fz_mpp(c.sm, MP_LAM)[xh][zh];
        if (EVEN) {
            cpa8<ASYNC>(dm, c.a->m[1] + i);
            cpa8<ASYNC>(dl, c.a->m[0] + i);
        } else {
            cpa4<ASYNC>(dm, c.a->m[1] + i, true);
            cpa4<ASYNC>(dm + 1, c.a->m[1] + i + 1, true);
            cpa4<ASYNC>(dl, c.a->m[0] + i, true);
            cpa4<ASYNC>(dl + 1, c.a->m[0] + i + 1, true);
        }
    }
}

// Global inputs of the own pair, loaded one phase before they are used so
// that their latency overlaps shared-memory work: mu and lambda of the column
// plane, rho and the three prev components of the output plane.
struct ColIn {
    F2 mu, lam;
};
template <bool EVEN>
FWI_HD ColIn pz_col_in(const FusedCtx &c, int tid, int q)
{
    const int pzi = tid % pz::NPR, lx = tid / pz::NPR;
    const int64_t i = c.a->g.idx(c.x0 + lx, q, c.z0 + 2 * pzi);
    return ColIn{ldg2<EVEN>(c.a->m[1] + i), ldg2<EVEN>(c.a->m[0] + i)};
}
struct UpdIn {
    F2 rho, p[3];
};
template <bool EVEN>
FWI_HD UpdIn pz_upd_in(const FusedCtx &c, int tid, int y)
{
    const int pzi = tid % pz::NPR, lx = tid / pz::NPR;
    const int64_t i = c.a->g.idx(c.x0 + lx, y, c.z0 + 2 * pzi);
    UpdIn r;
    r.rho = ldg2<EVEN>(c.a->m[2] + i);
#pragma unroll
    for (int k = 0; k < 3; k++) r.p[k] = ldg2<EVEN>(c.a->prev[k] + c.so + i);
    return r;
}

// Column phase: plane q = y+2 of the own pair into the y queues.
FWI_HD void pz_column(const FusedCtx &c, const PairK &K, PairThread &th, int tid, const ColIn &in)
{
    const int pzi = tid % pz::NPR, lx = tid / pz::NPR;
    const int xw = lx + fz::HW, zw = 2 * pzi + fz::HW;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        th.qmu[k] = th.qmu[k + 1];
        th.qT[k] = th.qT[k + 1];
        th.qX1[k] = th.qX1[k + 1];
        th.qZ1[k] = th.qZ1[k + 1];
    }
    th.qmu[4] = in.mu;
    // plane q = y+2 sits in slot sl[4]; its neighbours q-2..q+2 in sl[2..6]
    const int s0 = c.sl[4];
    constexpr int X = fz::ZW;
    const float *u0 = pz_u(c, s0, 0, xw, zw), *u1 = pz_u(c, s0, 1, xw, zw), *u2 = pz_u(c, s0, 2, xw, zw);
    const F2 ux0 = d1p(ld2(u0 - 2 * X), ld2(u0 - X), ld2(u0 + X), ld2(u0 + 2 * X), K.cx0, K.cx1);
    const F2 ux1 = d1p(ld2(u1 - 2 * X), ld2(u1 - X), ld2(u1 + X), ld2(u1 + 2 * X), K.cx0, K.cx1);
    const F2 uy1 = d1p(ld2(pz_u(c, c.sl[2], 1, xw, zw)), ld2(pz_u(c, c.sl[3], 1, xw, zw)),
                       ld2(pz_u(c, c.sl[5], 1, xw, zw)), ld2(pz_u(c, c.sl[6], 1, xw, zw)), K.cy0, K.cy1);
    const ZT z2 = ztaps(u2), z1 = ztaps(u1);
    const F2 uz2 = d1p(z2.m, z2.m1(), z2.p1(), z2.b, K.cz0, K.cz1);
    const F2 uz1 = d1p(z1.m, z1.m1(), z1.p1(), z1.b, K.cz0, K.cz1);
    th.qT[4] = mul2(in.lam, add2(add2(ux0, uy1), uz2));
    th.qX1[4] = mul2(in.mu, ux1);
    th.qZ1[4] = mul2(in.mu, uz1);
}

// Derived values at one pair of the derived region (xh, zh): T always, and
// (Y0, Z0) on x-halo rows or (X2, Y2) on z-halo pairs.
template <bool XHALO>
FWI_HD void pz_derived_halo(const FusedCtx &c, const PairK &K, int xh, int zh)
{
    const int xw = xh + (fz::HW - fz::HD), zw = zh + (fz::HW - fz::HD);
    constexpr int X = fz::ZW;
    const int s0 = c.sl[2];
    const float *u0 = pz_u(c, s0, 0, xw, zw), *u2 = pz_u(c, s0, 2, xw, zw);
    const F2 mu = ld2(&fz_mpp(c.sm, MP_MU)[xh][zh]), lam = ld2(&fz_mpp(c.sm, MP_LAM)[xh][zh]);
    auto ydiff = [&](int k) {
        return d1p(ld2(pz_u(c, c.sl[0], k, xw, zw)), ld2(pz_u(c, c.sl[1], k, xw, zw)),
                   ld2(pz_u(c, c.sl[3], k, xw, zw)), ld2(pz_u(c, c.sl[4], k, xw, zw)), K.cy0, K.cy1);
    };
    const F2 ux0 = d1p(ld2(u0 - 2 * X), ld2(u0 - X), ld2(u0 + X), ld2(u0 + 2 * X), K.cx0, K.cx1);
    const F2 uy1 = ydiff(1);
    const ZT z2 = ztaps(u2);
    const F2 uz2 = d1p(z2.m, z2.m1(), z2.p1(), z2.b, K.cz0, K.cz1);
    st2(&fz_dvp(c.sm, DV_T0)[xh][zh], mul2(lam, add2(add2(ux0, uy1), uz2)));
    if (XHALO) {
        const ZT z0 = ztaps(u0);
        st2(&fz_dvp(c.sm, DV_Y0)[xh][zh], mul2(mu, ydiff(0)));
        st2(&fz_dvp(c.sm, DV_Z0)[xh][zh], mul2(mu, d1p(z0.m, z0.m1(), z0.p1(), z0.b, K.cz0, K.cz1)));
    } else {
        const F2 ux2 = d1p(ld2(u2 - 2 * X), ld2(u2 - X), ld2(u2 + X), ld2(u2 + 2 * X), K.cx0, K.cx1);
        st2(&fz_dvp(c.sm, DV_X2)[xh][zh], mul2(mu, ux2));
        st2(&fz_dvp(c.sm, DV_Y2)[xh][zh], mul2(mu, ydiff(2)));
    }
}

// Phase B: D2var terms of the own pair into acc, derived values of the own
// pair (and, for threads 0..95, of the halo) into the derived planes.
FWI_HD void pz_phase_b(const FusedCtx &c, const PairK &K, const PairThread &th, int tid, F2 acc[3])
{
    const int pzi = tid % pz::NPR, lx = tid / pz::NPR;
    const int xw = lx + fz::HW, zw = 2 * pzi + fz::HW;
    const int xh = lx + fz::HD, zh = 2 * pzi + fz::HD;
    constexpr int X = fz::ZW, XD = fz::ZH;
    const float *mp = &fz_mpp(c.sm, MP_MU)[xh][zh];
    const F2 mu0 = ld2(mp);
    const F2 lam = ld2(&fz_mpp(c.sm, MP_LAM)[xh][zh]);
    const W5p wx = d2w_pair(ld2(mp - 2 * XD), ld2(mp - XD), mu0, ld2(mp + XD), ld2(mp + 2 * XD), K.sx1);
    const ZT zm = ztaps(mp);
    const W5p wz = d2w_pair(zm.m, zm.m1(), mu0, zm.p1(), zm.b, K.sz1);
    const W5p wy = d2w_pair(th.qmu[0], th.qmu[1], th.qmu[2], th.qmu[3], th.qmu[4], K.sy1);
    F2 ux0, uy0, uz0, uy1, ux2, uy2, uz2;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float *u = pz_u(c, c.sl[2], k, xw, zw);
        const F2 xm2 = ld2(u - 2 * X), xm1 = ld2(u - X), u0 = ld2(u), xp1 = ld2(u + X), xp2 = ld2(u + 2 * X);
        const F2 ym2 = ld2(pz_u(c, c.sl[0], k, xw, zw)), ym1 = ld2(pz_u(c, c.sl[1], k, xw, zw));
        const F2 yp1 = ld2(pz_u(c, c.sl[3], k, xw, zw)), yp2 = ld2(pz_u(c, c.sl[4], k, xw, zw));
        const ZT z{ld2(u - 2), u0, ld2(u + 2)};
        const F2 zm1 = z.m1(), zp1 = z.p1();
        // own axis first, doubled (a = 2 for the component's own direction)
        F2 v;
        if (k == 0) {
            v = d2acc(wx, xm2, xm1, u0, xp1, xp2, f2s(0.f));
            v = add2(v, v);
            v = d2acc(wy, ym2, ym1, u0, yp1, yp2, v);
            v = d2acc(wz, z.m, zm1, u0, zp1, z.b, v);
            ux0 = d1p(xm2, xm1, xp1, xp2, K.cx0, K.cx1);
            uy0 = d1p(ym2, ym1, yp1, yp2, K.cy0, K.cy1);
            uz0 = d1p(z.m, zm1, zp1, z.b, K.cz0, K.cz1);
        } else if (k == 1) {
            v = d2acc(wy, ym2, ym1, u0, yp1, yp2, f2s(0.f));
            v = add2(v, v);
            v = d2acc(wx, xm2, xm1, u0, xp1, xp2, v);
            v = d2acc(wz, z.m, zm1, u0, zp1, z.b, v);
            uy1 = d1p(ym2, ym1, yp1, yp2, K.cy0, K.cy1);
        } else {
            v = d2acc(wz, z.m, zm1, u0, zp1, z.b, f2s(0.f));
            v = add2(v, v);
            v = d2acc(wx, xm2, xm1, u0, xp1, xp2, v);
            v = d2acc(wy, ym2, ym1, u0, yp1, yp2, v);
            ux2 = d1p(xm2, xm1, xp1, xp2, K.cx0, K.cx1);
            uy2 = d1p(ym2, ym1, yp1, yp2, K.cy0, K.cy1);
            uz2 = d1p(z.m, zm1, zp1, z.b, K.cz0, K.cz1);
        }
        acc[k] = v;
    }
    st2(&fz_dvp(c.sm, DV_T0)[xh][zh], mul2(lam, add2(add2(ux0, uy1), uz2)));
    st2(&fz_dvp(c.sm, DV_Y0)[xh][zh], mul2(mu0, uy0));
    st2(&fz_dvp(c.sm, DV_Z0)[xh][zh], mul2(mu0, uz0));
    st2(&fz_dvp(c.sm, DV_X2)[xh][zh], mul2(mu0, ux2));
    st2(&fz_dvp(c.sm, DV_Y2)[xh][zh], mul2(mu0, uy2));
    // halo of the derived planes: rows 0, 1, XH-2, XH-1 (T, Y0, Z0) by
    // threads 0..63, the first and last pair of rows 2..XH-3 (T, X2, Y2) by
    // threads 64..95 (warp-uniform split)
    if (tid < 4 * pz::NPR) {
        const int r = tid / pz::NPR;
        pz_derived_halo<true>(c, K, r < 2 ? r : fz::XH - 4 + r, fz::HD + 2 * (tid % pz::NPR));
    } else if (tid < 4 * pz::NPR + 2 * pz::TX) {
        const int u = tid - 4 * pz::NPR;
        pz_derived_halo<false>(c, K, fz::HD + (u >> 1), (u & 1) ? fz::ZH - 2 : 0);
    }
}

// Phase C: first derivatives of the derived planes and queues, update, taper.
template <bool EVEN>
FWI_HD void pz_phase_c(const FusedCtx &c, const PairK &K, const PairThread &th, int tid, int y, const F2 acc[3],
                       const UpdIn &in)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    const int pzi = tid % pz::NPR, lx = tid / pz::NPR;
    const int ix = c.x0 + lx, iz = c.z0 + 2 * pzi;
    const int xw = lx + fz::HW, zw = 2 * pzi + fz::HW;
    const int xh = lx + fz::HD, zh = 2 * pzi + fz::HD;
    constexpr int XD = fz::ZH;
    const float *t0 = &fz_dvp(c.sm, DV_T0)[xh][zh];
    const float *y0 = &fz_dvp(c.sm, DV_Y0)[xh][zh], *z0 = &fz_dvp(c.sm, DV_Z0)[xh][zh];
    const float *x2 = &fz_dvp(c.sm, DV_X2)[xh][zh], *y2 = &fz_dvp(c.sm, DV_Y2)[xh][zh];
    // comp 0: Dx(T) + Dy(mu u_x1) + Dz(mu u_x2) with 1/dy (we_op.cpp:678)
    F2 v0 = d1acc(ld2(t0 - 2 * XD), ld2(t0 - XD), ld2(t0 + XD), ld2(t0 + 2 * XD), K.cx0, K.cx1, acc[0]);
    v0 = d1acc(th.qX1[0], th.qX1[1], th.qX1[3], th.qX1[4], K.cy0, K.cy1, v0);
    const ZT zx2 = ztaps(x2);
    v0 = d1acc(zx2.m, zx2.m1(), zx2.p1(), zx2.b, K.cy0, K.cy1, v0);
    // comp 1: Dy(T) + Dx(mu u_y0) + Dz(mu u_y2)
    F2 v1 = d1acc(th.qT[0], th.qT[1], th.qT[3], th.qT[4], K.cy0, K.cy1, acc[1]);
    v1 = d1acc(ld2(y0 - 2 * XD), ld2(y0 - XD), ld2(y0 + XD), ld2(y0 + 2 * XD), K.cx0, K.cx1, v1);
    const ZT zy2 = ztaps(y2);
    v1 = d1acc(zy2.m, zy2.m1(), zy2.p1(), zy2.b, K.cz0, K.cz1, v1);
    // comp 2: Dz(T) + Dx(mu u_z0) + Dy(mu u_z1)
    const ZT zt = ztaps(t0);
    F2 v2 = d1acc(zt.m, zt.m1(), zt.p1(), zt.b, K.cz0, K.cz1, acc[2]);
    v2 = d1acc(ld2(z0 - 2 * XD), ld2(z0 - XD), ld2(z0 + XD), ld2(z0 + 2 * XD), K.cx0, K.cx1, v2);
    v2 = d1acc(th.qZ1[0], th.qZ1[1], th.qZ1[3], th.qZ1[4], K.cy0, K.cy1, v2);

    // update: next = dt^2 acc / rho + 2 curr - prev, then the taper
    const int64_t i = g.idx(ix, y, iz);
    const float dt2 = a.dt * a.dt;
    const F2 s = f2(dt2 * rcp_rn(f2lo(in.rho)), dt2 * rcp_rn(f2hi(in.rho)));
    const bool tz = in_taper(a, ix, y, iz) || in_taper(a, ix, y, iz + 1);
    F2 tf = f2s(1.f);
    if (tz) {
        // one factor per point, the product of the six in the reference's
        // order: z (top, bottom), x (left, right), y (front, back)
        tf = f2(a.tap[0][iz], a.tap[0][iz + 1]);
        tf = mul2(tf, f2(a.tap[1][iz], a.tap[1][iz + 1]));
        tf = mul2(tf, f2s(a.tap[2][ix]));
        tf = mul2(tf, f2s(a.tap[3][ix]));
        tf = mul2(tf, f2s(a.tap[4][y]));
        tf = mul2(tf, f2s(a.tap[5][y]));
    }
    const F2 v[3] = {v0, v1, v2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        F2 p = in.p[k];
        if (tz && a.taper_prev) p = mul2(p, tf);
        const F2 u0 = ld2(pz_u(c, c.sl[2], k, xw, zw));
        F2 r = sub2(fma2(v[k], s, add2(u0, u0)), p);
        if (tz) r = mul2(r, tf);
        stg2<EVEN>(a.next[k] + c.so + i, r);
    }
}

}  // namespace fwi
