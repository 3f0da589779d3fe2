// Isotropic elastic step of planes [6, ny-6), two z-adjacent points per
// thread in packed FP32 pairs.
//
// Same tiling, ring and bulk-tensor plane copies as the fused kernel
// (fused.cuh): a CTA owns a TZ x TX = 32 x 16 tile of (z, x) columns and
// marches along y over planes of [6, ny-6).  Interior tiles (outputs and
// derived halo free of SBP closure rows along x and z) run the pair form
// only; edge tiles add the closure rows (see pxd1/pzd1 and phase B).  Here a thread owns the pair (z, z+1) of
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

// Thread -> own pair: pair index pzi along z, x row lx of the tile.  The
// default layout gives each half-warp one x row (16 consecutive pairs), so the
// x closure rows are uniform per half-warp.  ZQ, for the tiles that touch a z
// face only: a warp holds 4 pairs of 8 x rows, so the closure pairs of a face
// (the first or last three of the tile) fall into two warps instead of all
// eight, warps 2b and 2b+1 for pair block b, which the SM issues from
// different sub-partitions (warp index mod 4); the x rows of a half-warp are
// interleaved so that its 16 eight-byte accesses hit distinct bank pairs at
// both row strides of the tile (ZW for the ring, ZH for the derived and
// material planes).
template <bool ZQ>
FWI_HD void pz_pos(int tid, int &pzi, int &lx)
{
    if (!ZQ) {
        pzi = tid % pz::NPR;
        lx = tid / pz::NPR;
        return;
    }
    const int w = tid >> 5, h = (tid >> 4) & 1, j = (tid >> 2) & 3, p = tid & 3;
    pzi = 4 * (w >> 1) + p;
    lx = 8 * (w & 1) + j + 4 * (h ^ ((p < 2 && j > 0) ? 1 : 0));
}
static_assert(pz::NPR == 16 && pz::TX == 16, "the ZQ layout covers 16 pairs x 16 rows");
static_assert(fz::ZW % 32 == 8 && fz::ZH % 32 == 4, "the ZQ layout is bank-conflict free at these row strides");

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
    float a;
    asm("{\n .reg .b32 t;\n mov.b64 {%0, t}, %1;\n}" : "=f"(a) : "l"(p.v));
    return a;
#else
    return p.x;
#endif
}
FWI_HD float f2hi(F2 p)
{
#if defined(__CUDA_ARCH__)
    float b;
    asm("{\n .reg .b32 t;\n mov.b64 {t, %0}, %1;\n}" : "=f"(b) : "l"(p.v));
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

// Taper of the own pair: the z and x factors do not change along the march,
// so they are read once; a plane adds its two y factors.
struct PairTaper {
    F2 zx;      // tz_lo * tz_hi * tx_lo * tx_hi per point (the reference's factor order)
    bool inzx;  // a point of the pair lies in a z or x taper zone
};
template <bool ZQ>
FWI_HD PairTaper pair_taper(const FusedCtx &c, int tid)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    int pzi, lx;
    pz_pos<ZQ>(tid, pzi, lx);
    // points past the grid's end (their stores are masked) take the last
    // row's factors, so that the tables are read in bounds
    const int ix = min(c.x0 + lx, g.nx - 1), iz = min(c.z0 + 2 * pzi, g.nz - 1), iz1 = min(iz + 1, g.nz - 1);
    auto zin = [&](int z) { return z < a.tw[0] || z >= g.nz - a.tw[1]; };
    PairTaper t;
    t.inzx = zin(iz) || zin(iz1) || ix < a.tw[2] || ix >= g.nx - a.tw[3];
    t.zx = f2s(1.f);
    if (t.inzx) {
        t.zx = f2(a.tap[0][iz], a.tap[0][iz1]);
        t.zx = mul2(t.zx, f2(a.tap[1][iz], a.tap[1][iz1]));
        t.zx = mul2(t.zx, f2s(a.tap[2][ix]));
        t.zx = mul2(t.zx, f2s(a.tap[3][ix]));
    }
    return t;
}

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
// asynchronous on the GPU (cp.async; zero fill when `valid` is false, `src`
// then only has to be a mapped address), a plain copy on the host.
template <bool ASYNC>
FWI_HD void cpa8(float *dst, const float *src, bool valid)
{
#if defined(__CUDA_ARCH__)
    if (ASYNC) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0)
                     : "memory");
        return;
    }
#endif
    dst[0] = valid ? src[0] : 0.f;
    dst[1] = valid ? src[1] : 0.f;
}

// Material planes mu, lambda at y over the derived region, as pairs (zeros
// outside the grid, where edge tiles' windows reach); with ASYNC the copies
// are asynchronous (waited for with cpa_wait).
template <bool EVEN, bool ASYNC>
FWI_HD void pz_load_mat(FusedCtx &c, int tid, int y)
{
    const Dims &g = c.a->g;
    constexpr int NP = fz::ZH / 2;  // 18 pairs per row
    for (int p = tid; p < fz::XH * NP; p += pz::NT) {
        const int xh = p / NP, zh = 2 * (p - xh * NP);
        const int ix = c.x0 - fz::HD + xh, iz = c.z0 - fz::HD + zh;
        const bool xin = ix >= 0 && ix < g.nx;
        const bool in0 = xin && iz >= 0 && iz < g.nz, in1 = xin && iz + 1 >= 0 && iz + 1 < g.nz;
        // positions outside the grid copy nothing (zero fill) from the array's start
        const int64_t i0 = in0 ? g.idx(ix, y, iz) : 0, i1 = in1 ? g.idx(ix, y, iz + 1) : 0;
        float *dm = &fz_mpp(c.sm, MP_MU)[xh][zh], *dl = &fz_mpp(c.sm, MP_LAM)[xh][zh];
        if (EVEN) {
            // nz, z0 and zh even: a pair is inside the grid or outside as a whole
            cpa8<ASYNC>(dm, c.a->m[1] + i0, in0);
            cpa8<ASYNC>(dl, c.a->m[0] + i0, in0);
        } else {
            cpa4<ASYNC>(dm, c.a->m[1] + i0, in0);
            cpa4<ASYNC>(dm + 1, c.a->m[1] + i1, in1);
            cpa4<ASYNC>(dl, c.a->m[0] + i0, in0);
            cpa4<ASYNC>(dl + 1, c.a->m[0] + i1, in1);
        }
    }
}

// L2 prefetch hint (no register result): the closure weights and face
// divisors of the next plane are requested a step ahead of their use.
FWI_HD void prefetch_l2(const void *p)
{
#if defined(__CUDA_ARCH__)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
#else
    (void)p;
#endif
}

// L2 prefetch of the next step's global inputs, so that their loads (issued
// a phase ahead of use) find them in L2 rather than in HBM.  By warp: the
// material plane y+2 (mu, lambda; tile and halo rows), the column's
// materials of plane y+3 (mu, lambda), rho and the three prev components of
// plane y+1.  A lane takes one x row and prefetches the first, middle and
// last word of its z span (at most three 128-byte lines).
FWI_HD void pz_prefetch_next(const FusedCtx &c, int tid, int y)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    const int w = tid >> 5, l = tid & 31;
    const bool mat = w < 2;
    const int q = mat ? y + 2 : w < 4 ? y + 3 : y + 1;
    const int ix = mat ? c.x0 - fz::HD + l : c.x0 + l;
    if (l >= (mat ? fz::XH : fz::TX) || ix < 0 || ix >= g.nx || q >= g.ny) return;
    const float *base = w == 0 || w == 2 ? a.m[1] : w == 1 || w == 3 ? a.m[0] : w == 4 ? a.m[2] : a.prev[w - 5] + c.so;
    const int za = max(mat ? c.z0 - fz::HD : c.z0, 0), zb = min((mat ? c.z0 + fz::TZ + fz::HD : c.z0 + fz::TZ) - 1, g.nz - 1);
    const float *row = base + g.idx(ix, q, 0);
    prefetch_l2(row + za);
    prefetch_l2(row + (za + zb) / 2);
    prefetch_l2(row + zb);
}

// Global inputs of the own pair, loaded one phase before they are used so
// that their latency overlaps shared-memory work: mu and lambda of the column
// plane, rho and the three prev components of the output plane.
struct ColIn {
    F2 mu, lam;
};
template <bool EVEN, bool ZQ>
FWI_HD ColIn pz_col_in(const FusedCtx &c, int tid, int q)
{
    int pzi, lx;
    pz_pos<ZQ>(tid, pzi, lx);
    const int64_t i = c.a->g.idx(c.x0 + lx, q, c.z0 + 2 * pzi);
    return ColIn{ldg2<EVEN>(c.a->m[1] + i), ldg2<EVEN>(c.a->m[0] + i)};
}
struct UpdIn {
    F2 rho, p[3];
};
template <bool EVEN, bool ZQ>
FWI_HD UpdIn pz_upd_in(const FusedCtx &c, int tid, int y)
{
    int pzi, lx;
    pz_pos<ZQ>(tid, pzi, lx);
    const int64_t i = c.a->g.idx(c.x0 + lx, y, c.z0 + 2 * pzi);
    UpdIn r;
    r.rho = ldg2<EVEN>(c.a->m[2] + i);
#pragma unroll
    for (int k = 0; k < 3; k++) r.p[k] = ldg2<EVEN>(c.a->prev[k] + c.so + i);
    return r;
}

// ---------------------------------------------------------------------------
// Derivatives at the own pair with the SBP closures of the edge tiles.
// XC: the tile touches an x face.  x rows are uniform per half-warp, so a row
// within 4 (D1) or 6 (D2var) of a face takes the reference's closure row for
// both points of the pair at once (pair taps along x, the row's coefficient in
// both halves) while the other half-warps take the interior form.
// ZC: the tile touches a z face.  Its closure pairs are (0,1), (2,3), (4,5)
// and their mirrors at the high face: both points of such a pair are closure
// rows that read the same wall samples, so a closure pair multiplies each
// wall sample (in both halves) by the pair of its two rows' coefficients.
// Only these pairs diverge from the rest of their warp.  Pairs of other
// alignments reach closure rows only in rows a tile does not store (the rows
// beyond the next tile's origin); they take the per-point rows.
// D2var closure weights come from the per-model tables (a.w2c, 8 weights per
// closure row and line), read once per plane for the three components.
// ---------------------------------------------------------------------------
// Closure coefficient pairs in shared memory (the rows region of FusedSmem):
//   [0, 48)    D1 along z, kinds 0..3 x 6 wall samples x (point 0, point 1):
//              rows (0,1), (2,3) of the low face, rows (1,0), (3,2) of the
//              high face negated (the reference's mirrored closure)
//   [48, 144)  D1 along x, kinds 0..7 x 6 wall samples x (c, c): row r of the
//              low face (kind r), row r of the high face negated (kind 4+r)
constexpr int PR_X = 48, PR_FLOATS = 144;
static_assert(PR_FLOATS <= SR_FLOATS, "closure pairs must fit the rows region");
FWI_HD void fill_pair_rows(float *p, int tid, int nt)
{
    const SbpTables &t = sbp();
    for (int e = tid; e < PR_FLOATS / 2; e += nt) {
        if (e < 24) {
            const int kind = e / 6, j = e % 6;
            const int r0 = kind == 0 ? 0 : kind == 1 ? 2 : kind == 2 ? 1 : 3;
            const int r1 = kind == 0 ? 1 : kind == 1 ? 3 : kind == 2 ? 0 : 2;
            const float sg = kind < 2 ? 1.f : -1.f;
            p[2 * e] = sg * t.d1b[r0][j];
            p[2 * e + 1] = sg * t.d1b[r1][j];
        } else {
            const int e2 = e - 24, kind = e2 / 6, j = e2 % 6;
            const float v = (kind < 4 ? 1.f : -1.f) * t.d1b[kind & 3][j];
            p[2 * e] = v;
            p[2 * e + 1] = v;
        }
    }
}

// D1 along x of a field at p (own pair, global row ix), row stride XS
template <bool XC>
FWI_HD F2 pxd1(const FusedCtx &c, const float *p, int XS, int ix, F2 c0h, F2 c1h, float ih)
{
    const int n = c.a->g.nx;
    if (XC && (ix < 4 || ix >= n - 4)) {
        const bool hi = ix >= n - 4;
        const float *w = c.sm->rows + PR_X + ((hi ? 4 : 0) + (hi ? n - 1 - ix : ix)) * 12;
        const float *b = p + ((hi ? n - 1 : 0) - ix) * XS;  // the own column at the wall
        const int st = hi ? -XS : XS;
        F2 acc = mul2(ld2(w), ld2(b));
#pragma unroll
        for (int j = 1; j < 6; j++) acc = fma2(ld2(w + 2 * j), ld2(b + j * st), acc);
        return mul2(acc, f2s(ih));
    }
    return d1p(ld2(p - 2 * XS), ld2(p - XS), ld2(p + XS), ld2(p + 2 * XS), c0h, c1h);
}
// D1 along z of a field at p (own pair at global z iz), window origin zoff (global z of index 0)
template <bool ZC>
FWI_HD F2 pzd1(const FusedCtx &c, const float *p, int iz, int zoff, F2 c0h, F2 c1h, float ih)
{
    const int n = c.a->g.nz;
    if (ZC && (iz < 4 || iz + 1 >= n - 4)) {
        const int kind = iz == 0 ? 0 : iz == 2 ? 1 : iz + 1 == n - 1 ? 2 : iz + 1 == n - 3 ? 3 : -1;
        if (kind >= 0) {
            const bool hi = kind >= 2;
            const float *w = c.sm->rows + kind * 12;
            const float *b = p + (hi ? n - 1 - iz : -iz);  // the wall sample
            const int st = hi ? -1 : 1;
            F2 acc = mul2(ld2(w), f2s(b[0]));
#pragma unroll
            for (int j = 1; j < 6; j++) acc = fma2(ld2(w + 2 * j), f2s(b[j * st]), acc);
            return mul2(acc, f2s(ih));
        }
        const SZ l{p - (iz - zoff), zoff};
        return f2(d1_row(l, iz, n, ConstRows()) * ih, d1_row(l, iz + 1, n, ConstRows()) * ih);
    }
    const ZT z = ztaps(p);
    return d1p(z.m, z.m1(), z.p1(), z.b, c0h, c1h);
}


// Absorbing-boundary scale of point (ix, y, iz) of component k (boundary_scale),
// with a prefetch of the same face's divisor at plane y+1.  Planes of the
// paired kernel lie in [6, ny-6), so only the x and z faces own its points.
FWI_HD float pz_face_scale(const StepArgs &a, float v, int k, int ix, int y, int iz)
{
    if (!a.scale) return v;
    int64_t off;
    const int f = owner_face(a.g, ix, y, iz, off);
    if (f < 0) return v;
    const float *d = a.sdiv[f][k] + off;
    prefetch_l2(d + (f == TOP || f == BOTTOM ? a.g.nx : a.g.nz));
    return v / d[0];
}

// D2var closure weights of a pair (8 per point, scaled by s) from a per-model table.
struct W8p {
    F2 w[8];
};
FWI_HD W8p w8_pair(const float *p0, const float *p1, F2 s)
{
    W8p r;
#if defined(__CUDA_ARCH__)
    const float4 a0 = *reinterpret_cast<const float4 *>(p0), a1 = *reinterpret_cast<const float4 *>(p0 + 4);
    const float4 b0 = *reinterpret_cast<const float4 *>(p1), b1 = *reinterpret_cast<const float4 *>(p1 + 4);
    r.w[0] = f2(a0.x, b0.x); r.w[1] = f2(a0.y, b0.y); r.w[2] = f2(a0.z, b0.z); r.w[3] = f2(a0.w, b0.w);
    r.w[4] = f2(a1.x, b1.x); r.w[5] = f2(a1.y, b1.y); r.w[6] = f2(a1.z, b1.z); r.w[7] = f2(a1.w, b1.w);
#else
    for (int j = 0; j < 8; j++) r.w[j] = f2(p0[j], p1[j]);
#endif
#pragma unroll
    for (int j = 0; j < 8; j++) r.w[j] = mul2(r.w[j], s);
    return r;
}

// The same derivatives added to acc (the pair form folds the sum into its FMAs).
template <bool XC>
FWI_HD F2 pxd1acc(const FusedCtx &c, const float *p, int XS, int ix, F2 c0h, F2 c1h, float ih, F2 acc)
{
    if (XC) return add2(acc, pxd1<XC>(c, p, XS, ix, c0h, c1h, ih));
    return d1acc(ld2(p - 2 * XS), ld2(p - XS), ld2(p + XS), ld2(p + 2 * XS), c0h, c1h, acc);
}
template <bool ZC>
FWI_HD F2 pzd1acc(const FusedCtx &c, const float *p, int iz, int zoff, F2 c0h, F2 c1h, float ih, F2 acc)
{
    if (ZC) return add2(acc, pzd1<ZC>(c, p, iz, zoff, c0h, c1h, ih));
    const ZT z = ztaps(p);
    return d1acc(z.m, z.m1(), z.p1(), z.b, c0h, c1h, acc);
}

// Column phase: plane q = y+2 of the own pair into the y queues.
template <bool XC, bool ZC>
FWI_HD void pz_column(const FusedCtx &c, const PairK &K, PairThread &th, int tid, const ColIn &in)
{
    const StepArgs &a = *c.a;
    int pzi, lx;
    pz_pos<ZC && !XC>(tid, pzi, lx);
    const int xw = lx + fz::HW, zw = 2 * pzi + fz::HW;
    const int ix = c.x0 + lx, iz = c.z0 + 2 * pzi;
    const int zo = c.z0 - fz::HW;
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
    const F2 ux0 = pxd1<XC>(c, u0, X, ix, K.cx0, K.cx1, a.idx);
    const F2 ux1 = pxd1<XC>(c, u1, X, ix, K.cx0, K.cx1, a.idx);
    const F2 uy1 = d1p(ld2(pz_u(c, c.sl[2], 1, xw, zw)), ld2(pz_u(c, c.sl[3], 1, xw, zw)),
                       ld2(pz_u(c, c.sl[5], 1, xw, zw)), ld2(pz_u(c, c.sl[6], 1, xw, zw)), K.cy0, K.cy1);
    const F2 uz2 = pzd1<ZC>(c, u2, iz, zo, K.cz0, K.cz1, a.idz);
    const F2 uz1 = pzd1<ZC>(c, u1, iz, zo, K.cz0, K.cz1, a.idz);
    th.qT[4] = mul2(in.lam, add2(add2(ux0, uy1), uz2));
    th.qX1[4] = mul2(in.mu, ux1);
    th.qZ1[4] = mul2(in.mu, uz1);
}

// Derived values at one pair of the derived region (xh, zh): T always, and
// (Y0, Z0) on x-halo rows or (X2, Y2) on z-halo pairs; zeros outside the grid
// (no closure row reads them).
template <bool XHALO, bool XC, bool ZC>
FWI_HD void pz_derived_halo(const FusedCtx &c, const PairK &K, int xh, int zh)
{
    const StepArgs &a = *c.a;
    const int ix = c.x0 - fz::HD + xh, iz = c.z0 - fz::HD + zh;
    if ((XC && (ix < 0 || ix >= a.g.nx)) || (ZC && (iz < 0 || iz >= a.g.nz))) {
        const F2 z = f2s(0.f);
        st2(&fz_dvp(c.sm, DV_T0)[xh][zh], z);
        st2(&fz_dvp(c.sm, XHALO ? DV_Y0 : DV_X2)[xh][zh], z);
        st2(&fz_dvp(c.sm, XHALO ? DV_Z0 : DV_Y2)[xh][zh], z);
        return;
    }
    const int xw = xh + (fz::HW - fz::HD), zw = zh + (fz::HW - fz::HD);
    const int zo = c.z0 - fz::HW;
    constexpr int X = fz::ZW;
    const int s0 = c.sl[2];
    const float *u0 = pz_u(c, s0, 0, xw, zw), *u2 = pz_u(c, s0, 2, xw, zw);
    const F2 mu = ld2(&fz_mpp(c.sm, MP_MU)[xh][zh]), lam = ld2(&fz_mpp(c.sm, MP_LAM)[xh][zh]);
    auto ydiff = [&](int k) {
        return d1p(ld2(pz_u(c, c.sl[0], k, xw, zw)), ld2(pz_u(c, c.sl[1], k, xw, zw)),
                   ld2(pz_u(c, c.sl[3], k, xw, zw)), ld2(pz_u(c, c.sl[4], k, xw, zw)), K.cy0, K.cy1);
    };
    const F2 ux0 = pxd1<XC>(c, u0, X, ix, K.cx0, K.cx1, a.idx);
    const F2 uy1 = ydiff(1);
    const F2 uz2 = pzd1<ZC>(c, u2, iz, zo, K.cz0, K.cz1, a.idz);
    st2(&fz_dvp(c.sm, DV_T0)[xh][zh], mul2(lam, add2(add2(ux0, uy1), uz2)));
    if (XHALO) {
        st2(&fz_dvp(c.sm, DV_Y0)[xh][zh], mul2(mu, ydiff(0)));
        st2(&fz_dvp(c.sm, DV_Z0)[xh][zh], mul2(mu, pzd1<ZC>(c, u0, iz, zo, K.cz0, K.cz1, a.idz)));
    } else {
        st2(&fz_dvp(c.sm, DV_X2)[xh][zh], mul2(mu, pxd1<XC>(c, u2, X, ix, K.cx0, K.cx1, a.idx)));
        st2(&fz_dvp(c.sm, DV_Y2)[xh][zh], mul2(mu, ydiff(2)));
    }
}

// Phase B: D2var terms of the own pair into acc, derived values of the own
// pair (and, for threads 0..95, of the halo) into the derived planes.
template <bool XC, bool ZC>
FWI_HD void pz_phase_b(const FusedCtx &c, const PairK &K, const PairThread &th, int tid, int y, F2 acc[3])
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    int pzi, lx;
    pz_pos<ZC && !XC>(tid, pzi, lx);
    const int xw = lx + fz::HW, zw = 2 * pzi + fz::HW;
    const int xh = lx + fz::HD, zh = 2 * pzi + fz::HD;
    const int ix = c.x0 + lx, iz = c.z0 + 2 * pzi;
    const int xo = c.x0 - fz::HW, zo = c.z0 - fz::HW;
    constexpr int X = fz::ZW, XD = fz::ZH;
    // closure rows of D2var (rows within 6 of a face) on this pair
    const bool xcl = XC && (ix < 6 || ix >= g.nx - 6);
    const bool zcl = ZC && (iz < 6 || iz + 1 >= g.nz - 6);
    const float *mp = &fz_mpp(c.sm, MP_MU)[xh][zh];
    const F2 mu0 = ld2(mp);
    W5p wx{}, wz{};
    if (!xcl) wx = d2w_pair(ld2(mp - 2 * XD), ld2(mp - XD), mu0, ld2(mp + XD), ld2(mp + 2 * XD), K.sx1);
    if (!zcl) {
        const ZT zm = ztaps(mp);
        wz = d2w_pair(zm.m, zm.m1(), mu0, zm.p1(), zm.b, K.sz1);
    }
    const W5p wy = d2w_pair(th.qmu[0], th.qmu[1], th.qmu[2], th.qmu[3], th.qmu[4], K.sy1);
    // D2var closure terms of the three components (scaled by a/h^2, a = 1):
    // weights read once per plane, wall samples of each component's ring line
    F2 d2xc[3], d2zc[3];
    if (XC && xcl) {
        const bool hi = ix >= g.nx - 6;
        const int r = hi ? g.nx - 1 - ix : ix, slot = hi ? 6 + r : r;
        const float *tab = a.w2c[0][0];
        const int64_t ln = (int64_t)y * g.nz + iz;
        const int st = hi ? -X : X;
        if (tab) {
            const W8p W = w8_pair(tab + (ln * 12 + slot) * 8, tab + ((ln + 1) * 12 + slot) * 8, K.sx1);
            // the same rows of plane y+1 (line ln + nz; y+1 < ny-5, so in the table)
            prefetch_l2(tab + ((ln + g.nz) * 12 + slot) * 8);
            prefetch_l2(tab + ((ln + g.nz + 1) * 12 + slot) * 8);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float *b = pz_u(c, c.sl[2], k, xw, zw) + ((hi ? g.nx - 1 : 0) - ix) * X;
                F2 v = mul2(W.w[0], ld2(b));
#pragma unroll
                for (int j = 1; j < 8; j++) v = fma2(W.w[j], ld2(b + j * st), v);
                d2xc[k] = v;
            }
        } else {
            for (int k = 0; k < 3; k++) {
                const float *l = pz_u(c, c.sl[2], k, xw, zw) - (ix - xo) * X;
                d2xc[k] = f2(d2var_row(SX{l, xo, X}, mx_line(c, MP_MU, zh), ix, g.nx, a.ad1[0], ConstRows()),
                             d2var_row(SX{l + 1, xo, X}, mx_line(c, MP_MU, zh + 1), ix, g.nx, a.ad1[0], ConstRows()));
            }
        }
    }
    if (ZC && zcl) {
        const int n = g.nz;
        const bool lo = iz == 0 || iz == 2 || iz == 4, hi = n - 1 - iz == 1 || n - 1 - iz == 3 || n - 1 - iz == 5;
        const float *tab = a.w2c[2][0];
        const int64_t ln = (int64_t)y * g.nx + ix;
        if (tab && (lo || hi)) {
            // rows (iz, iz+1) at the low face, (n-1-iz, n-2-iz) at the high face
            const int s0 = lo ? iz : 6 + (n - 1 - iz), s1 = lo ? iz + 1 : 5 + (n - 1 - iz);
            const W8p W = w8_pair(tab + (ln * 12 + s0) * 8, tab + (ln * 12 + s1) * 8, K.sz1);
            prefetch_l2(tab + ((ln + g.nx) * 12 + s0) * 8);  // plane y+1
            prefetch_l2(tab + ((ln + g.nx) * 12 + s1) * 8);
            const int st = hi ? -1 : 1;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float *b = pz_u(c, c.sl[2], k, xw, zw) + (hi ? n - 1 - iz : -iz);
                F2 v = mul2(W.w[0], f2s(b[0]));
#pragma unroll
                for (int j = 1; j < 8; j++) v = fma2(W.w[j], f2s(b[j * st]), v);
                d2zc[k] = v;
            }
        } else {
            const SZ f = mz_line(c, MP_MU, xh);
            for (int k = 0; k < 3; k++) {
                const SZ l{pz_u(c, c.sl[2], k, xw, zw) - (iz - zo), zo};
                d2zc[k] = f2(d2var_tab(tab, ln, l, f, iz, n, a.ad1[2], ConstRows()),
                             d2var_tab(tab, ln, l, f, iz + 1, n, a.ad1[2], ConstRows()));
            }
        }
    }
    // D2var along x / z of component k added to v
    auto d2x = [&](int k, F2 xm2, F2 xm1, F2 u0, F2 xp1, F2 xp2, F2 v) -> F2 {
        if (XC && xcl) return add2(v, d2xc[k]);
        return d2acc(wx, xm2, xm1, u0, xp1, xp2, v);
    };
    auto d2z = [&](int k, const ZT &z, F2 zm1, F2 zp1, F2 v) -> F2 {
        if (ZC && zcl) return add2(v, d2zc[k]);
        return d2acc(wz, z.m, zm1, z.a, zp1, z.b, v);
    };
    F2 uy0, uz0, ux2, uy2;
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
            v = d2x(k, xm2, xm1, u0, xp1, xp2, f2s(0.f));
            v = add2(v, v);
            v = d2acc(wy, ym2, ym1, u0, yp1, yp2, v);
            v = d2z(k, z, zm1, zp1, v);
            uy0 = d1p(ym2, ym1, yp1, yp2, K.cy0, K.cy1);
            uz0 = ZC ? pzd1<ZC>(c, u, iz, zo, K.cz0, K.cz1, a.idz) : d1p(z.m, zm1, zp1, z.b, K.cz0, K.cz1);
        } else if (k == 1) {
            v = d2acc(wy, ym2, ym1, u0, yp1, yp2, f2s(0.f));
            v = add2(v, v);
            v = d2x(k, xm2, xm1, u0, xp1, xp2, v);
            v = d2z(k, z, zm1, zp1, v);
        } else {
            v = d2z(k, z, zm1, zp1, f2s(0.f));
            v = add2(v, v);
            v = d2x(k, xm2, xm1, u0, xp1, xp2, v);
            v = d2acc(wy, ym2, ym1, u0, yp1, yp2, v);
            ux2 = XC ? pxd1<XC>(c, u, X, ix, K.cx0, K.cx1, a.idx) : d1p(xm2, xm1, xp1, xp2, K.cx0, K.cx1);
            uy2 = d1p(ym2, ym1, yp1, yp2, K.cy0, K.cy1);
        }
        acc[k] = v;
    }
    // lambda div u of the own pair is the column phase's value of this plane
    st2(&fz_dvp(c.sm, DV_T0)[xh][zh], th.qT[2]);
    st2(&fz_dvp(c.sm, DV_Y0)[xh][zh], mul2(mu0, uy0));
    st2(&fz_dvp(c.sm, DV_Z0)[xh][zh], mul2(mu0, uz0));
    st2(&fz_dvp(c.sm, DV_X2)[xh][zh], mul2(mu0, ux2));
    st2(&fz_dvp(c.sm, DV_Y2)[xh][zh], mul2(mu0, uy2));
    // halo of the derived planes: rows 0, 1, XH-2, XH-1 (T, Y0, Z0) by the
    // first two of three warps from warp hw, the first and last pair of rows
    // 2..XH-3 (T, X2, Y2) by the third (warp-uniform split).  hw keeps this
    // work off the warps that hold closure rows: warps 0..2 in a tile whose
    // first x rows are closure rows, warps 0, 1 or 6, 7 (the z faces' pair
    // blocks) in the z-face layout.
    const int hw = (ZC && !XC) ? 2 : (XC && (c.x0 < 6 || c.x0 >= g.nx - 6)) ? 5 : 0;
    const int ht = (tid - 32 * hw) & (pz::NT - 1);
    if (ht < 4 * pz::NPR) {
        const int r = ht / pz::NPR;
        pz_derived_halo<true, XC, ZC>(c, K, r < 2 ? r : fz::XH - 4 + r, fz::HD + 2 * (ht % pz::NPR));
    } else if (ht < 4 * pz::NPR + 2 * pz::TX) {
        const int u = ht - 4 * pz::NPR;
        pz_derived_halo<false, XC, ZC>(c, K, fz::HD + (u >> 1), (u & 1) ? fz::ZH - 2 : 0);
    }
}

// Phase C: first derivatives of the derived planes and queues, update,
// absorbing-boundary scaling of face points (edge tiles), taper; points
// beyond the tile's output rows (xend, zend: rows the next tile owns) are
// not stored.
template <bool EVEN, bool XC, bool ZC>
FWI_HD void pz_phase_c(const FusedCtx &c, const PairK &K, const PairThread &th, int tid, int y, const F2 acc[3],
                       const UpdIn &in, const PairTaper &tp)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    int pzi, lx;
    pz_pos<ZC && !XC>(tid, pzi, lx);
    const int ix = c.x0 + lx, iz = c.z0 + 2 * pzi;
    const int xw = lx + fz::HW, zw = 2 * pzi + fz::HW;
    const int xh = lx + fz::HD, zh = 2 * pzi + fz::HD;
    const int zo = c.z0 - fz::HD;
    constexpr int XD = fz::ZH;
    const float *t0 = &fz_dvp(c.sm, DV_T0)[xh][zh];
    const float *y0 = &fz_dvp(c.sm, DV_Y0)[xh][zh], *z0 = &fz_dvp(c.sm, DV_Z0)[xh][zh];
    const float *x2 = &fz_dvp(c.sm, DV_X2)[xh][zh], *y2 = &fz_dvp(c.sm, DV_Y2)[xh][zh];
    // comp 0: Dx(T) + Dy(mu u_x1) + Dz(mu u_x2) with 1/dy (we_op.cpp:678)
    F2 v0 = pxd1acc<XC>(c, t0, XD, ix, K.cx0, K.cx1, a.idx, acc[0]);
    v0 = d1acc(th.qX1[0], th.qX1[1], th.qX1[3], th.qX1[4], K.cy0, K.cy1, v0);
    v0 = pzd1acc<ZC>(c, x2, iz, zo, K.cy0, K.cy1, a.idy, v0);
    // comp 1: Dy(T) + Dx(mu u_y0) + Dz(mu u_y2)
    F2 v1 = d1acc(th.qT[0], th.qT[1], th.qT[3], th.qT[4], K.cy0, K.cy1, acc[1]);
    v1 = pxd1acc<XC>(c, y0, XD, ix, K.cx0, K.cx1, a.idx, v1);
    v1 = pzd1acc<ZC>(c, y2, iz, zo, K.cz0, K.cz1, a.idz, v1);
    // comp 2: Dz(T) + Dx(mu u_z0) + Dy(mu u_z1)
    F2 v2 = pzd1acc<ZC>(c, t0, iz, zo, K.cz0, K.cz1, a.idz, acc[2]);
    v2 = pxd1acc<XC>(c, z0, XD, ix, K.cx0, K.cx1, a.idx, v2);
    v2 = d1acc(th.qZ1[0], th.qZ1[1], th.qZ1[3], th.qZ1[4], K.cy0, K.cy1, v2);

    // update: next = dt^2 acc / rho + 2 curr - prev, then the taper
    if (ix >= c.xend) return;
    const int64_t i = g.idx(ix, y, iz);
    const float dt2 = a.dt * a.dt;
    const F2 s = f2(dt2 * rcp_rn(f2lo(in.rho)), dt2 * rcp_rn(f2hi(in.rho)));
    const bool tz = tp.inzx || y < a.tw[4] || y >= g.ny - a.tw[5];
    const bool face = (XC && (ix == 0 || ix == g.nx - 1)) || (ZC && (iz == 0 || iz >= g.nz - 2));
    F2 tf = f2s(1.f);
    if (tz) {
        // one factor per point, the product of the six in the reference's
        // order: z (top, bottom), x (left, right), y (front, back)
        tf = mul2(tp.zx, f2s(a.tap[4][y]));
        tf = mul2(tf, f2s(a.tap[5][y]));
    }
    const F2 v[3] = {v0, v1, v2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        F2 p = in.p[k];
        if (tz && a.taper_prev) p = mul2(p, tf);
        const F2 u0 = ld2(pz_u(c, c.sl[2], k, xw, zw));
        F2 r = sub2(fma2(v[k], s, add2(u0, u0)), p);
        if (face) r = f2(pz_face_scale(a, f2lo(r), k, ix, y, iz), pz_face_scale(a, f2hi(r), k, ix, y, iz + 1));
        if (tz) r = mul2(r, tf);
        float *dst = a.next[k] + c.so + i;
        if (iz + 1 < c.zend) {
            stg2<EVEN>(dst, r);
        } else if (iz < c.zend) {
            dst[0] = f2lo(r);
        }
    }
}

}  // namespace fwi
