// Fused elastic time step (isotropic and VTI): one kernel computes, for every
// output point, all operator terms of the reference's step (we_op.cpp:646-836,
// 1297-1497) -- D2var x9, D1 of the stress combination, the six mixed mult_D
// terms -- plus SAT, leapfrog update, absorbing scaling and taper, reading each
// wavefield and model array from HBM once.
//
// Blocking: a CTA owns a TZ x TX tile of (z, x) columns (z = lanes, x = warps)
// and marches along y.  Shared memory holds a ring of the last 7 planes of the
// three displacement components over the tile plus a 4-point halo, and, for the
// output plane, the first-derivative combinations whose x/z derivatives are
// taken (tile plus 2-point halo).  Quantities differentiated along y are kept
// per thread in 5-deep register queues.  The x/z tiling (tile_range) gives the
// rows of the SBP boundary closures to the first and last tiles, whose windows
// hold every sample those rows read; first derivatives at closure rows of the
// halo are taken from global memory.  The 6 planes next to each y wall (the
// y closure rows) are left to the marching kernel (or the per-point kernels);
// the launch covers y in [6, ny-6), where every first derivative along y of
// the planes it reads, y-2 .. y+2 of each output plane y, is an interior row.
//
// Every helper is a host/device function of (context, thread index) so a CPU
// harness can run the same phases thread by thread.
#pragma once

#include "physics.cuh"

namespace fwi {

namespace fz {
constexpr int TZ = 32, TX = 16, NT = TZ * TX;
constexpr int HW = 4;                          // halo of the displacement ring
constexpr int ZW = TZ + 2 * HW, XW = TX + 2 * HW;
constexpr int HD = 2;                          // halo of the derived planes
constexpr int ZH = TZ + 2 * HD, XH = TX + 2 * HD;
constexpr int YPAD = 6;                        // y planes per side left to the closure-capable kernels
}  // namespace fz

// Derived-plane slots: T0, Y0, Z0, X2, Y2 in dv; T2 (VTI only; the isotropic
// T2 equals T0) in the overlay below.
enum { DV_T0 = 0, DV_Y0 = 1, DV_Z0 = 2, DV_X2 = 3, DV_Y2 = 4, NDVC = 5, DV_T2 = 5, NDV = 6 };
// Material planes over the derived region: mu, lambda in mp; (VTI) c13, eps,
// c66 in the overlay.
enum { MP_MU = 0, MP_LAM = 1, NMPC = 2, MP_C13 = 2, MP_EPS = 3, MP_C66 = 4, NMP = 5 };

// Ring slot 7: the elastic kernel's eighth displacement plane (the one
// copied in while the others are in use); the VTI kernel keeps a 7-slot ring
// and stores its four extra planes (T2, c13, eps, c66) there instead.
struct FusedSmem {
    float u[8][3][fz::XW][fz::ZW];
    float dv[NDVC][fz::XH][fz::ZH];
    float mp[NMPC][fz::XH][fz::ZH];
    unsigned long long bar[8];  // completion barriers of the ring slots' bulk-tensor copies
    float rows[SR_FLOATS];      // SBP closure rows, padded (SmemRows)
};
// bytes of one displacement plane window (three components) in a ring slot
constexpr unsigned FZ_PLANE_BYTES = 3u * fz::XW * fz::ZW * sizeof(float);
static_assert(FZ_PLANE_BYTES % 128 == 0, "ring slots must stay 128-byte aligned for bulk-tensor copies");
static_assert(4 * fz::XH * fz::ZH <= 3 * fz::XW * fz::ZW, "VTI overlay must fit one ring slot");
using ZRow = float[fz::ZH];
FWI_HD ZRow *fz_dvp(const FusedSmem *s, int d)
{
    if (d < NDVC) return const_cast<ZRow *>(s->dv[d]);
    return reinterpret_cast<ZRow *>(const_cast<float *>(&s->u[7][0][0][0]));
}
FWI_HD ZRow *fz_mpp(const FusedSmem *s, int m)
{
    if (m < NMPC) return const_cast<ZRow *>(s->mp[m]);
    return reinterpret_cast<ZRow *>(const_cast<float *>(&s->u[7][0][0][0]) + (m - NMPC + 1) * fz::XH * fz::ZH);
}

// One 4-byte global->shared copy: asynchronous on the GPU (cp.async; zero
// fill when `valid` is false, `src` then only has to be a mapped address),
// a plain copy on the host.
template <bool ASYNC>
FWI_HD void cpa4(float *dst, const float *src, bool valid)
{
#if defined(__CUDA_ARCH__)
    if (ASYNC) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0)
                     : "memory");
        return;
    }
#endif
    *dst = valid ? *src : 0.f;
}
FWI_HD void cpa_commit()
{
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}
FWI_HD void cpa_wait()
{
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
}

// Per-thread state carried along the march (registers on the GPU).
struct FusedThread {
    float qmu[5];   // mu at y-2..y+2 (own column)
    float qeps[5];  // eps (VTI)
    float q66[5];   // c66 (VTI)
    float qT[5];    // stress combination differentiated along y (T iso, T1 VTI)
    float qX1[5];   // P * Dx u1
    float qZ1[5];   // mu * Dz u1
};

struct FusedCtx {
    const StepArgs *a; // launch arguments (pointers of shot 0)
    int shot;
    int64_t so;        // wavefield offset of this shot (shot * sst)
    int x0, z0;        // tile (window) origin
    int xend, zend;    // end of this tile's output rows
    int sl[7];         // ring slots of planes y-2 .. y+4 for the current march step
    FusedSmem *sm;
    // bulk-tensor plane copies (GPU only): tensor map of the current level,
    // error flag, per-slot barrier phases of this thread, copies on / given up
    SmemRows rows{nullptr};  // closure rows in shared memory (FusedSmem::rows)
    const void *tmap = nullptr;
    int *err = nullptr;
    unsigned ph = 0;
    bool tma = false, dead = false;
};


// Smem line accessors (global index -> smem slot).
struct SZ {  // along z at fixed (slot, comp, xw)
    const float *p;  // &u[slot][c][xw][0]
    int off;         // global z of smem position 0
    FWI_HD float operator()(int k) const { return p[k - off]; }
};
struct SX {  // along x at fixed zw
    const float *p;  // &arr[0][zw]
    int off;         // global x of smem position 0
    int stride;
    FWI_HD float operator()(int k) const { return p[(k - off) * stride]; }
};
// Window-clamped variants (closure rows of halo positions).
struct SZc {
    const float *p;
    int off, len;
    FWI_HD float operator()(int k) const
    {
        const int j = k - off;
        return p[j < 0 ? 0 : (j >= len ? len - 1 : j)];
    }
};
struct SXc {
    const float *p;
    int off, stride, len;
    FWI_HD float operator()(int k) const
    {
        const int j = k - off;
        return p[(j < 0 ? 0 : (j >= len ? len - 1 : j)) * stride];
    }
};

// Ring depth: 8 slots for the elastic kernel (one plane in flight), 7 for VTI.
template <int PH>
FWI_HD constexpr int fz_nring() { return PH == ELASTIC ? 8 : 7; }
template <int PH>
FWI_HD int ring(int q) { return ((q % fz_nring<PH>()) + fz_nring<PH>()) % fz_nring<PH>(); }

// Ring slots of planes y-2 .. y+4.
template <int PH>
FWI_HD void fz_slots(FusedCtx &c, int y)
{
    int s = ring<PH>(y - 2);
    for (int k = 0; k < 7; k++) {
        c.sl[k] = s;
        s = s + 1 == fz_nring<PH>() ? 0 : s + 1;
    }
}

// ---------------------------------------------------------------------------
// Phase A: load displacement plane q (tile + 4 halo) into its ring slot.
// ---------------------------------------------------------------------------
template <bool ASYNC = false>
FWI_HD void fz_load_u(FusedCtx &c, int tid, int q, int slot)
{
    const Dims &g = c.a->g;
    for (int p = tid; p < fz::XW * fz::ZW; p += fz::NT) {
        const int xw = p / fz::ZW, zw = p - xw * fz::ZW;
        const int ix = c.x0 - fz::HW + xw, iz = c.z0 - fz::HW + zw;
        const bool in = ix >= 0 && ix < g.nx && iz >= 0 && iz < g.nz;
        const int64_t i = c.so + (in ? g.idx(ix, q, iz) : 0);
        for (int k = 0; k < 3; k++) cpa4<ASYNC>(&c.sm->u[slot][k][xw][zw], c.a->curr[k] + i, in);
    }
}

// Position p of the derived region (XH x ZH = 20 x 36): the 32 columns
// zh = 2..33 row by row first, so that a warp covers one row of the tile
// (no shared-memory bank conflicts), then the four halo columns.
FWI_HD void fz_dpos(int p, int &xh, int &zh)
{
    constexpr int MAIN = fz::XH * fz::TZ;  // 640
    static_assert(fz::TZ == 32 && fz::ZH == fz::TZ + 4, "warp-row mapping assumes 32 + 2 x 2 columns");
    if (p < MAIN) {
        xh = p >> 5;
        zh = fz::HD + (p & 31);
    } else {
        const int h = p - MAIN;
        xh = h >> 2;
        const int zc = h & 3;
        zh = zc < 2 ? zc : fz::TZ + zc;
    }
}

// Material planes at y over the derived region.
template <int PH>
FWI_HD void fz_load_mat(FusedCtx &c, int tid, int y)
{
    const Dims &g = c.a->g;
    for (int p = tid; p < fz::XH * fz::ZH; p += fz::NT) {
        int xh, zh;
        fz_dpos(p, xh, zh);
        const int ix = c.x0 - fz::HD + xh, iz = c.z0 - fz::HD + zh;
        const bool in = ix >= 0 && ix < g.nx && iz >= 0 && iz < g.nz;
        const int64_t i = in ? g.idx(ix, y, iz) : 0;
        fz_mpp(c.sm, MP_MU)[xh][zh] = in ? c.a->m[1][i] : 0.f;
        fz_mpp(c.sm, MP_LAM)[xh][zh] = in ? c.a->m[0][i] : 0.f;
        if (PH == VTI) {
            fz_mpp(c.sm, MP_C13)[xh][zh] = in ? c.a->m[3][i] : 0.f;
            fz_mpp(c.sm, MP_EPS)[xh][zh] = in ? c.a->m[4][i] : 0.f;
            fz_mpp(c.sm, MP_C66)[xh][zh] = in ? c.a->m[5][i] : 0.f;
        }
    }
}

// First derivatives of displacement component k at (ix, q, iz) along x, y, z
// from the ring (with the 1/h).  ixw/izw: smem coordinates in the ring window.
template <bool F = false>
FWI_HD float fz_dx(const FusedCtx &c, int k, int slot, int ix, int izw)
{
    const float *p = &c.sm->u[slot][k][0][izw];
    const int j = ix - (c.x0 - fz::HW);
    if (F || (ix >= 4 && ix < c.a->g.nx - 4)) {
        const SbpTables &t = sbp();
        return (t.d1c0 * (p[(j + 1) * fz::ZW] - p[(j - 1) * fz::ZW]) + t.d1c1 * (p[(j + 2) * fz::ZW] - p[(j - 2) * fz::ZW])) *
               c.a->idx;
    }
    const SXc s{p, c.x0 - fz::HW, fz::ZW, fz::XW};
    return d1_row(s, ix, c.a->g.nx, c.rows) * c.a->idx;
}
template <bool F = false>
FWI_HD float fz_dz(const FusedCtx &c, int k, int slot, int ixw, int iz)
{
    const float *p = &c.sm->u[slot][k][ixw][0];
    const int j = iz - (c.z0 - fz::HW);
    if (F || (iz >= 4 && iz < c.a->g.nz - 4)) {
        const SbpTables &t = sbp();
        return (t.d1c0 * (p[j + 1] - p[j - 1]) + t.d1c1 * (p[j + 2] - p[j - 2])) * c.a->idz;
    }
    const SZc s{p, c.z0 - fz::HW, fz::ZW};
    return d1_row(s, iz, c.a->g.nz, c.rows) * c.a->idz;
}
// Dy at a plane from the ring slots of its four neighbours: interior rows only
// (the fused launch differentiates planes 4 .. ny-5 only, interior D1 rows).
FWI_HD float fz_dy(const FusedCtx &c, int k, const int *sn, int ixw, int izw)
{
    const SbpTables &t = sbp();
    const float um2 = c.sm->u[sn[0]][k][ixw][izw], um1 = c.sm->u[sn[1]][k][ixw][izw];
    const float up1 = c.sm->u[sn[2]][k][ixw][izw], up2 = c.sm->u[sn[3]][k][ixw][izw];
    return (t.d1c0 * (up1 - um1) + t.d1c1 * (up2 - um2)) * c.a->idy;
}

// ---------------------------------------------------------------------------
// Phase B1: derived quantities of plane y over the derived region.
// ---------------------------------------------------------------------------
template <int PH, bool XF = false, bool ZF = false>
FWI_HD void fz_derived(FusedCtx &c, int tid, int y)
{
    const Dims &g = c.a->g;
    for (int p = tid; p < fz::XH * fz::ZH; p += fz::NT) {
        int xh, zh;
        fz_dpos(p, xh, zh);
        const int ix = c.x0 - fz::HD + xh, iz = c.z0 - fz::HD + zh;
        auto dv = [&](int d) -> float & { return fz_dvp(c.sm, d)[xh][zh]; };
        if (!(XF && ZF) && (ix < 0 || ix >= g.nx || iz < 0 || iz >= g.nz)) {
            for (int k = 0; k < (PH == ELASTIC ? NDVC : NDV); k++) dv(k) = 0.f;
            continue;
        }
        const int ixw = xh + (fz::HW - fz::HD), izw = zh + (fz::HW - fz::HD);
        const int s0 = c.sl[2];
        const int sn[4] = {c.sl[0], c.sl[1], c.sl[3], c.sl[4]};
        const float ux0 = fz_dx<XF>(c, 0, s0, ix, izw);
        const float uy1 = fz_dy(c, 1, sn, ixw, izw);
        const float uz2 = fz_dz<ZF>(c, 2, s0, ixw, iz);
        const float mu = fz_mpp(c.sm, MP_MU)[xh][zh], lam = fz_mpp(c.sm, MP_LAM)[xh][zh];
        const float uy0 = fz_dy(c, 0, sn, ixw, izw);
        const float uz0 = fz_dz<ZF>(c, 0, s0, ixw, iz);
        const float ux2 = fz_dx<XF>(c, 2, s0, ix, izw);
        const float uy2 = fz_dy(c, 2, sn, ixw, izw);
        if (PH == ELASTIC) {
            dv(DV_T0) = lam * (ux0 + uy1 + uz2);  // also the z-differentiated T2
            dv(DV_Y0) = uy0;  // multiplied by the coefficient at the tap (mult_D)
        } else {
            const float c13 = fz_mpp(c.sm, MP_C13)[xh][zh], eps = fz_mpp(c.sm, MP_EPS)[xh][zh];
            const float c66 = fz_mpp(c.sm, MP_C66)[xh][zh];
            const float c11c = (1.f + 2.f * eps) * lam;
            const float c12 = (1.f + 2.f * eps) * (lam + 2.f * mu) - 2.f * c66;
            dv(DV_T0) = c11c * ux0 + c12 * uy1 + c13 * uz2;
            dv(DV_T2) = c13 * (ux0 + uy1) + lam * uz2;
            dv(DV_Y0) = uy0;
        }
        dv(DV_Z0) = uz0;
        dv(DV_X2) = ux2;
        dv(DV_Y2) = uy2;
    }
}

// Phase B2: own-column quantities of plane q = y+2 pushed into the y queues.
template <int PH, bool XF = false, bool ZF = false>
FWI_HD void fz_column(FusedCtx &c, FusedThread &th, int tid, int q)
{
    const Dims &g = c.a->g;
    const int lz = tid % fz::TZ, lx = tid / fz::TZ;
    const int ix = c.x0 + lx, iz = c.z0 + lz;
    for (int k = 0; k < 4; k++) {
        th.qmu[k] = th.qmu[k + 1];
        th.qeps[k] = th.qeps[k + 1];
        th.q66[k] = th.q66[k + 1];
        th.qT[k] = th.qT[k + 1];
        th.qX1[k] = th.qX1[k + 1];
        th.qZ1[k] = th.qZ1[k + 1];
    }
    if (ix >= g.nx || iz >= g.nz) {
        th.qmu[4] = th.qeps[4] = th.q66[4] = th.qT[4] = th.qX1[4] = th.qZ1[4] = 0.f;
        return;
    }
    const int ixw = lx + fz::HW, izw = lz + fz::HW;
    const int64_t i = g.idx(ix, q, iz);
    const float mu = c.a->m[1][i], lam = c.a->m[0][i];
    th.qmu[4] = mu;
    // plane q = y+2 sits in slot sl[4]; its neighbours q-2..q+2 in sl[2..6]
    const int s0 = c.sl[4];
    const int sn[4] = {c.sl[2], c.sl[3], c.sl[5], c.sl[6]};
    const float ux0 = fz_dx<XF>(c, 0, s0, ix, izw);
    const float uy1 = fz_dy(c, 1, sn, ixw, izw);
    const float uz2 = fz_dz<ZF>(c, 2, s0, ixw, iz);
    const float ux1 = fz_dx<XF>(c, 1, s0, ix, izw);
    const float uz1 = fz_dz<ZF>(c, 1, s0, ixw, iz);
    if (PH == ELASTIC) {
        th.qT[4] = lam * (ux0 + uy1 + uz2);
        th.qX1[4] = ux1;
    } else {
        const float c13 = c.a->m[3][i], eps = c.a->m[4][i], c66 = c.a->m[5][i];
        th.qeps[4] = eps;
        th.q66[4] = c66;
        const float c11c = (1.f + 2.f * eps) * lam;
        const float c12 = (1.f + 2.f * eps) * (lam + 2.f * mu) - 2.f * c66;
        th.qT[4] = c11c * uy1 + c12 * ux0 + c13 * uz2;
        th.qX1[4] = ux1;
    }
    th.qZ1[4] = uz1;
}

// ---------------------------------------------------------------------------
// Phase C: output point (own column) of plane y.
// ---------------------------------------------------------------------------
// Interior D2var weights for the five taps (the reference's grouping).
struct W5 {
    float w0, wm1, wp1, wm2, wp2;
};
FWI_HD W5 d2w(float fm2, float fm1, float f0, float fp1, float fp2)
{
    const float *cc = sbp().d2in;
    W5 w;
    w.w0 = cc[0] * f0 + cc[1] * (fm1 + fp1) + cc[2] * (fm2 + fp2);
    w.wm1 = cc[3] * fm2 + cc[4] * fm1 + cc[5] * f0 + cc[6] * fp1;
    w.wp1 = cc[3] * fp2 + cc[4] * fp1 + cc[5] * f0 + cc[6] * fm1;
    w.wm2 = cc[7] * fm2 + cc[8] * fm1 + cc[9] * f0;
    w.wp2 = cc[7] * fp2 + cc[8] * fp1 + cc[9] * f0;
    return w;
}
FWI_HD float d2apply(const W5 &w, float ad2, float um2, float um1, float u0, float up1, float up2)
{
    return ad2 * (w.w0 * u0 + w.wm1 * um1 + w.wp1 * up1 + w.wm2 * um2 + w.wp2 * up2);
}
// Interior D1 (unscaled) from five taps.
FWI_HD float d1i(float am2, float am1, float ap1, float ap2)
{
    const SbpTables &t = sbp();
    return t.d1c0 * (ap1 - am1) + t.d1c1 * (ap2 - am2);
}
// Interior mult_D (unscaled): D1 of a*m with per-tap products.
FWI_HD float d1m(float am2, float mm2, float am1, float mm1, float ap1, float mp1, float ap2, float mp2)
{
    const SbpTables &t = sbp();
    return t.d1c0 * (ap1 * mp1 - am1 * mm1) + t.d1c1 * (ap2 * mp2 - am2 * mm2);
}

// D2var closure row: the 8 weights sum_k B[r][j][k] f(k) of the row, then
// applied to the field (spatial_operators.hpp:58-81).
struct W8 {
    float w[8];
};
template <class F, class R>
FWI_HD W8 d2closure_weights(const F &f, int i, int n, const R &b)
{
    const bool hi = i >= n - 6;
    const int r = hi ? n - 1 - i : i;
    float fk[8];
    for (int k = 0; k < 8; k++) fk[k] = f(hi ? n - 1 - k : k);
    W8 w;
    for (int j = 0; j < 8; j++) {
        float v = 0.f;
        for (int k = 0; k < 8; k++) v += b.d2(r, j, k) * fk[k];
        w.w[j] = v;
    }
    return w;
}
// Closure weights of row i (of n) on line `line` of a precomputed table
// (12 rows x 8 weights per line, the low rows first, then the high rows from
// the face inwards), or formed from the material line when there is none.
template <class F, class R>
FWI_HD W8 d2closure_w(const float *tab, int64_t line, const F &f, int i, int n, const R &b)
{
    if (!tab) return d2closure_weights(f, i, n, b);
    const int slot = i < 6 ? i : 6 + (n - 1 - i);
    const float *p = tab + (line * 12 + slot) * 8;
    W8 w;
#if defined(__CUDA_ARCH__)
    const float4 lo = *reinterpret_cast<const float4 *>(p), hi = *reinterpret_cast<const float4 *>(p + 4);
    w.w[0] = lo.x; w.w[1] = lo.y; w.w[2] = lo.z; w.w[3] = lo.w;
    w.w[4] = hi.x; w.w[5] = hi.y; w.w[6] = hi.z; w.w[7] = hi.w;
#else
    for (int j = 0; j < 8; j++) w.w[j] = p[j];
#endif
    return w;
}
template <class U>
FWI_HD float d2closure_apply(const W8 &w, const U &u, int i, int n, float ad2)
{
    const bool hi = i >= n - 6;
    float acc = 0.f;
    for (int j = 0; j < 8; j++) acc += ad2 * w.w[j] * u(hi ? n - 1 - j : j);
    return acc;
}
// d2var_row with the closure weights of a precomputed table (when present).
template <class U, class F, class R>
FWI_HD float d2var_tab(const float *tab, int64_t line, const U &u, const F &f, int i, int n, float ad2, const R &b)
{
    if (tab && (i < 6 || i >= n - 6)) return d2closure_apply(d2closure_w(tab, line, f, i, n, b), u, i, n, ad2);
    return d2var_row(u, f, i, n, ad2, b);
}

// Smem accessors of the output phase.
FWI_HD SX ux_line(const FusedCtx &c, int slot, int k, int izw) { return SX{&c.sm->u[slot][k][0][izw], c.x0 - fz::HW, fz::ZW}; }
FWI_HD SZ uz_line(const FusedCtx &c, int slot, int k, int ixw) { return SZ{&c.sm->u[slot][k][ixw][0], c.z0 - fz::HW}; }
FWI_HD SX mx_line(const FusedCtx &c, int m, int zh) { return SX{&fz_mpp(c.sm, m)[0][zh], c.x0 - fz::HD, fz::ZH}; }
FWI_HD SZ mz_line(const FusedCtx &c, int m, int xh) { return SZ{&fz_mpp(c.sm, m)[xh][0], c.z0 - fz::HD}; }
FWI_HD SX dx_line(const FusedCtx &c, int d, int zh) { return SX{&fz_dvp(c.sm, d)[0][zh], c.x0 - fz::HD, fz::ZH}; }
FWI_HD SZ dz_line(const FusedCtx &c, int d, int xh) { return SZ{&fz_dvp(c.sm, d)[xh][0], c.z0 - fz::HD}; }
template <class E, class M>
struct C11bS {
    E eps;
    M mu;
    FWI_HD float operator()(int k) const { return 2.f * (1.f + 2.f * eps(k)) * mu(k); }
};

template <int PH>
FWI_HD void fz_output(FusedCtx &c, const FusedThread &th, int tid, int y)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    const int lz = tid % fz::TZ, lx = tid / fz::TZ;
    const int ix = c.x0 + lx, iz = c.z0 + lz;
    if (ix >= c.xend || iz >= c.zend) return;
    const int64_t i = g.idx(ix, y, iz);
    const bool xin = ix >= 6 && ix < g.nx - 6;
    const bool zin = iz >= 6 && iz < g.nz - 6;
    const int ixw = lx + fz::HW, izw = lz + fz::HW;
    const int xh = lx + fz::HD, zh = lz + fz::HD;
    const FusedSmem &s = *c.sm;
    const int r0 = c.sl[2], rm1 = c.sl[1], rm2 = c.sl[0], rp1 = c.sl[3], rp2 = c.sl[4];
    const float idx2 = a.ad1[0], idy2 = a.ad1[1];

    float acc[3];
    // ---- D2var terms (we_op.cpp:647-657, 1298-1308) ----
    const SX mux = mx_line(c, MP_MU, zh);
    const SZ muz = mz_line(c, MP_MU, xh);
    if (PH == ELASTIC) {
        // one set of weights per axis serves the three components (all use mu)
        W5 wx{}, wz{};
        W8 wxc{}, wzc{};
        if (xin) wx = d2w(mux(ix - 2), mux(ix - 1), mux(ix), mux(ix + 1), mux(ix + 2));
        else wxc = d2closure_w(a.w2c[0][0], (int64_t)y * g.nz + iz, mux, ix, g.nx, c.rows);
        if (zin) wz = d2w(muz(iz - 2), muz(iz - 1), muz(iz), muz(iz + 1), muz(iz + 2));
        else wzc = d2closure_w(a.w2c[2][0], (int64_t)y * g.nx + ix, muz, iz, g.nz, c.rows);
        const W5 wy = d2w(th.qmu[0], th.qmu[1], th.qmu[2], th.qmu[3], th.qmu[4]);
        for (int k = 0; k < 3; k++) {
            const float adx = k == 0 ? a.ad2[0] : a.ad1[0];
            const float ady = k == 1 ? a.ad2[1] : a.ad1[1];
            const float adz = k == 2 ? a.ad2[2] : a.ad1[2];
            const SX ul = ux_line(c, r0, k, izw);
            const SZ uzl = uz_line(c, r0, k, ixw);
            float v = xin ? d2apply(wx, adx, ul(ix - 2), ul(ix - 1), ul(ix), ul(ix + 1), ul(ix + 2))
                          : d2closure_apply(wxc, ul, ix, g.nx, adx);
            v += d2apply(wy, ady, s.u[rm2][k][ixw][izw], s.u[rm1][k][ixw][izw], s.u[r0][k][ixw][izw],
                         s.u[rp1][k][ixw][izw], s.u[rp2][k][ixw][izw]);
            v += zin ? d2apply(wz, adz, uzl(iz - 2), uzl(iz - 1), uzl(iz), uzl(iz + 1), uzl(iz + 2))
                     : d2closure_apply(wzc, uzl, iz, g.nz, adz);
            acc[k] = v;
        }
    } else {
        // VTI: comp0 x:c11b y:c66 z:mu ; comp1 x:c66 y:c11b z:mu ; comp2 mu, mu, 2mu
        const C11bS<SX, SX> bx{mx_line(c, MP_EPS, zh), mux};
        const SX c6x = mx_line(c, MP_C66, zh);
        W5 wxb{}, wx6{}, wxm{}, wz{};
        if (xin) {
            wxb = d2w(bx(ix - 2), bx(ix - 1), bx(ix), bx(ix + 1), bx(ix + 2));
            wx6 = d2w(c6x(ix - 2), c6x(ix - 1), c6x(ix), c6x(ix + 1), c6x(ix + 2));
            wxm = d2w(mux(ix - 2), mux(ix - 1), mux(ix), mux(ix + 1), mux(ix + 2));
        }
        if (zin) wz = d2w(muz(iz - 2), muz(iz - 1), muz(iz), muz(iz + 1), muz(iz + 2));
        float qb[5];
        for (int k = 0; k < 5; k++) qb[k] = 2.f * (1.f + 2.f * th.qeps[k]) * th.qmu[k];
        const W5 wyb = d2w(qb[0], qb[1], qb[2], qb[3], qb[4]);
        const W5 wy6 = d2w(th.q66[0], th.q66[1], th.q66[2], th.q66[3], th.q66[4]);
        const W5 wym = d2w(th.qmu[0], th.qmu[1], th.qmu[2], th.qmu[3], th.qmu[4]);
        for (int k = 0; k < 3; k++) {
            const W5 &wx = k == 0 ? wxb : (k == 1 ? wx6 : wxm);
            const W5 &wy = k == 0 ? wy6 : (k == 1 ? wyb : wym);
            const float adz = k == 2 ? a.ad2[2] : a.ad1[2];
            const SX ul = ux_line(c, r0, k, izw);
            const SZ uzl = uz_line(c, r0, k, ixw);
            float v;
            if (xin) v = d2apply(wx, idx2, ul(ix - 2), ul(ix - 1), ul(ix), ul(ix + 1), ul(ix + 2));
            else if (k == 0) v = d2var_tab(a.w2c[0][2], (int64_t)y * g.nz + iz, ul, bx, ix, g.nx, idx2, c.rows);
            else if (k == 1) v = d2var_tab(a.w2c[0][1], (int64_t)y * g.nz + iz, ul, c6x, ix, g.nx, idx2, c.rows);
            else v = d2var_tab(a.w2c[0][0], (int64_t)y * g.nz + iz, ul, mux, ix, g.nx, idx2, c.rows);
            v += d2apply(wy, idy2, s.u[rm2][k][ixw][izw], s.u[rm1][k][ixw][izw], s.u[r0][k][ixw][izw],
                         s.u[rp1][k][ixw][izw], s.u[rp2][k][ixw][izw]);
            v += zin ? d2apply(wz, adz, uzl(iz - 2), uzl(iz - 1), uzl(iz), uzl(iz + 1), uzl(iz + 2))
                     : d2var_tab(a.w2c[2][0], (int64_t)y * g.nx + ix, uzl, muz, iz, g.nz, adz, c.rows);
            acc[k] = v;
        }
    }

    // ---- D1 of the stress combinations and the mixed terms (we_op.cpp:661-688, 1312-1349) ----
    const SX Px = (PH == VTI) ? mx_line(c, MP_C66, zh) : mux;
    const float *qP = (PH == VTI) ? th.q66 : th.qmu;
    // comp 0: Dx(T0)/dx + Dy(P u_x1)/dy + Dz(mu u_x2)/dy (dy as in the reference, we_op.cpp:678)
    acc[0] += d1_row(dx_line(c, DV_T0, zh), ix, g.nx, c.rows) * a.idx;
    acc[0] += d1m(th.qX1[0], qP[0], th.qX1[1], qP[1], th.qX1[3], qP[3], th.qX1[4], qP[4]) * a.idy;
    acc[0] += d1_prod_row(dz_line(c, DV_X2, xh), muz, iz, g.nz, c.rows) * a.idy;
    // comp 1: Dy(T1)/dy + Dx(P u_y0)/dx + Dz(mu u_y2)/dz
    acc[1] += d1i(th.qT[0], th.qT[1], th.qT[3], th.qT[4]) * a.idy;
    acc[1] += d1_prod_row(dx_line(c, DV_Y0, zh), Px, ix, g.nx, c.rows) * a.idx;
    acc[1] += d1_prod_row(dz_line(c, DV_Y2, xh), muz, iz, g.nz, c.rows) * a.idz;
    // comp 2: Dz(T2)/dz + Dx(mu u_z0)/dx + Dy(mu u_z1)/dy
    acc[2] += d1_row(dz_line(c, PH == ELASTIC ? DV_T0 : DV_T2, xh), iz, g.nz, c.rows) * a.idz;
    acc[2] += d1_prod_row(dx_line(c, DV_Z0, zh), mux, ix, g.nx, c.rows) * a.idx;
    acc[2] += d1m(th.qZ1[0], th.qmu[0], th.qZ1[1], th.qmu[1], th.qZ1[3], th.qmu[3], th.qZ1[4], th.qmu[4]) * a.idy;

    // ---- update, scaling, taper (SAT is added by the face kernel) ----
    const float dt2 = a.dt * a.dt;
    const float rho = a.m[2][i];
    const bool face = ix == 0 || ix == g.nx - 1 || iz == 0 || iz == g.nz - 1;
    const bool tz = in_taper(a, ix, y, iz);
    const float irho = 1.0f / rho;
    for (int k = 0; k < 3; k++) {
        float v = acc[k];
        const float p = a.prev[k][c.so + i];
        const float pe = (a.taper_prev && tz) ? taper(a, p, ix, y, iz) : p;
        v = dt2 * v * irho + 2.f * s.u[r0][k][ixw][izw] - pe;
        if (face) v = boundary_scale(a, v, k, ix, y, iz);
        if (tz) v = taper(a, v, ix, y, iz);
        a.next[k][c.so + i] = v;
    }
}

// Output phase with the taps read at constant offsets from per-point base
// pointers.  XF (ZF): every output and derived-halo point of the tile is
// interior along x (z); otherwise the rows of the SBP closures along that
// axis take the closure code, the other points the interior code.
template <int PH, bool XF, bool ZF>
FWI_HD void fz_output_t(FusedCtx &c, const FusedThread &th, int tid, int y)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    const int lz = tid % fz::TZ, lx = tid / fz::TZ;
    const int ix = c.x0 + lx, iz = c.z0 + lz;
    if (ix >= c.xend || iz >= c.zend) return;
    const int64_t i = g.idx(ix, y, iz);
    const int ixw = lx + fz::HW, izw = lz + fz::HW;
    const int xh = lx + fz::HD, zh = lz + fz::HD;
    const bool xin = XF || (ix >= 6 && ix < g.nx - 6);
    const bool zin = ZF || (iz >= 6 && iz < g.nz - 6);
    FusedSmem &s = *c.sm;
    constexpr int UX = fz::ZW, UC = fz::XW * fz::ZW, US = 3 * fz::XW * fz::ZW, DX = fz::ZH;
    const float *ub = &s.u[0][0][ixw][izw];
    const int r0 = c.sl[2] * US, rm1 = c.sl[1] * US, rm2 = c.sl[0] * US, rp1 = c.sl[3] * US, rp2 = c.sl[4] * US;
    const float *mu = &fz_mpp(&s, MP_MU)[xh][zh];
    const float idx2 = a.ad1[0], idy2 = a.ad1[1];
    const SX mux = mx_line(c, MP_MU, zh);
    const SZ muz = mz_line(c, MP_MU, xh);
    float acc[3];
    const W5 wym = d2w(th.qmu[0], th.qmu[1], th.qmu[2], th.qmu[3], th.qmu[4]);
    if (PH == ELASTIC) {
        W5 wx{}, wz{};
        W8 wxc{}, wzc{};
        if (xin) wx = d2w(mu[-2 * DX], mu[-DX], mu[0], mu[DX], mu[2 * DX]);
        else wxc = d2closure_w(a.w2c[0][0], (int64_t)y * g.nz + iz, mux, ix, g.nx, c.rows);
        if (zin) wz = d2w(mu[-2], mu[-1], mu[0], mu[1], mu[2]);
        else wzc = d2closure_w(a.w2c[2][0], (int64_t)y * g.nx + ix, muz, iz, g.nz, c.rows);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float adx = k == 0 ? a.ad2[0] : a.ad1[0];
            const float ady = k == 1 ? a.ad2[1] : a.ad1[1];
            const float adz = k == 2 ? a.ad2[2] : a.ad1[2];
            const float *u = ub + k * UC + r0;
            const float *uc = ub + k * UC;
            float v = xin ? d2apply(wx, adx, u[-2 * UX], u[-UX], u[0], u[UX], u[2 * UX])
                          : d2closure_apply(wxc, ux_line(c, c.sl[2], k, izw), ix, g.nx, adx);
            v += d2apply(wym, ady, uc[rm2], uc[rm1], u[0], uc[rp1], uc[rp2]);
            v += zin ? d2apply(wz, adz, u[-2], u[-1], u[0], u[1], u[2])
                     : d2closure_apply(wzc, uz_line(c, c.sl[2], k, ixw), iz, g.nz, adz);
            acc[k] = v;
        }
    } else {
        const float *ep = &fz_mpp(&s, MP_EPS)[xh][zh], *c6 = &fz_mpp(&s, MP_C66)[xh][zh];
        const C11bS<SX, SX> bx{mx_line(c, MP_EPS, zh), mux};
        const SX c6x = mx_line(c, MP_C66, zh);
        auto c11b = [&](int o) { return 2.f * (1.f + 2.f * ep[o]) * mu[o]; };
        W5 wxb{}, wx6{}, wxm{}, wz{};
        if (xin) {
            wxb = d2w(c11b(-2 * DX), c11b(-DX), c11b(0), c11b(DX), c11b(2 * DX));
            wx6 = d2w(c6[-2 * DX], c6[-DX], c6[0], c6[DX], c6[2 * DX]);
            wxm = d2w(mu[-2 * DX], mu[-DX], mu[0], mu[DX], mu[2 * DX]);
        }
        if (zin) wz = d2w(mu[-2], mu[-1], mu[0], mu[1], mu[2]);
        float qb[5];
#pragma unroll
        for (int k = 0; k < 5; k++) qb[k] = 2.f * (1.f + 2.f * th.qeps[k]) * th.qmu[k];
        const W5 wyb = d2w(qb[0], qb[1], qb[2], qb[3], qb[4]);
        const W5 wy6 = d2w(th.q66[0], th.q66[1], th.q66[2], th.q66[3], th.q66[4]);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const W5 &wx = k == 0 ? wxb : (k == 1 ? wx6 : wxm);
            const W5 &wy = k == 0 ? wy6 : (k == 1 ? wyb : wym);
            const float adz = k == 2 ? a.ad2[2] : a.ad1[2];
            const float *u = ub + k * UC + r0;
            const float *uc = ub + k * UC;
            float v;
            if (xin) {
                v = d2apply(wx, idx2, u[-2 * UX], u[-UX], u[0], u[UX], u[2 * UX]);
            } else {
                const SX ul = ux_line(c, c.sl[2], k, izw);
                const int64_t xl = (int64_t)y * g.nz + iz;
                v = k == 0 ? d2var_tab(a.w2c[0][2], xl, ul, bx, ix, g.nx, idx2, c.rows)
                           : (k == 1 ? d2var_tab(a.w2c[0][1], xl, ul, c6x, ix, g.nx, idx2, c.rows)
                                     : d2var_tab(a.w2c[0][0], xl, ul, mux, ix, g.nx, idx2, c.rows));
            }
            v += d2apply(wy, idy2, uc[rm2], uc[rm1], u[0], uc[rp1], uc[rp2]);
            v += zin ? d2apply(wz, adz, u[-2], u[-1], u[0], u[1], u[2])
                     : d2var_tab(a.w2c[2][0], (int64_t)y * g.nx + ix, uz_line(c, c.sl[2], k, ixw), muz, iz, g.nz, adz,
                                 c.rows);
            acc[k] = v;
        }
    }
    // D1 of the stress combinations and the mixed terms (we_op.cpp:661-688, 1312-1349)
    const float *P = (PH == VTI) ? &fz_mpp(&s, MP_C66)[xh][zh] : mu;
    const SX Px = (PH == VTI) ? mx_line(c, MP_C66, zh) : mux;
    const float *qP = (PH == VTI) ? th.q66 : th.qmu;
    const int DT2 = PH == ELASTIC ? DV_T0 : DV_T2;
    const float *t0 = &fz_dvp(&s, DV_T0)[xh][zh], *t2 = &fz_dvp(&s, DT2)[xh][zh];
    const float *x2 = &fz_dvp(&s, DV_X2)[xh][zh], *y0 = &fz_dvp(&s, DV_Y0)[xh][zh];
    const float *y2 = &fz_dvp(&s, DV_Y2)[xh][zh], *z0 = &fz_dvp(&s, DV_Z0)[xh][zh];
    // each term is added where it is formed, so that few values are live at once
    // comp 0: Dx(T0)/dx + Dy(P u_x1)/dy + Dz(mu u_x2)/dy (dy as in the reference, we_op.cpp:678)
    acc[0] += (xin ? d1i(t0[-2 * DX], t0[-DX], t0[DX], t0[2 * DX]) : d1_row(dx_line(c, DV_T0, zh), ix, g.nx, c.rows)) * a.idx;
    acc[0] += d1m(th.qX1[0], qP[0], th.qX1[1], qP[1], th.qX1[3], qP[3], th.qX1[4], qP[4]) * a.idy;
    acc[0] += (zin ? d1m(x2[-2], mu[-2], x2[-1], mu[-1], x2[1], mu[1], x2[2], mu[2])
                   : d1_prod_row(dz_line(c, DV_X2, xh), muz, iz, g.nz, c.rows)) * a.idy;
    // comp 1: Dy(T1)/dy + Dx(P u_y0)/dx + Dz(mu u_y2)/dz
    acc[1] += d1i(th.qT[0], th.qT[1], th.qT[3], th.qT[4]) * a.idy;
    acc[1] += (xin ? d1m(y0[-2 * DX], P[-2 * DX], y0[-DX], P[-DX], y0[DX], P[DX], y0[2 * DX], P[2 * DX])
                   : d1_prod_row(dx_line(c, DV_Y0, zh), Px, ix, g.nx, c.rows)) * a.idx;
    acc[1] += (zin ? d1m(y2[-2], mu[-2], y2[-1], mu[-1], y2[1], mu[1], y2[2], mu[2])
                   : d1_prod_row(dz_line(c, DV_Y2, xh), muz, iz, g.nz, c.rows)) * a.idz;
    // comp 2: Dz(T2)/dz + Dx(mu u_z0)/dx + Dy(mu u_z1)/dy
    acc[2] += (zin ? d1i(t2[-2], t2[-1], t2[1], t2[2]) : d1_row(dz_line(c, DT2, xh), iz, g.nz, c.rows)) * a.idz;
    acc[2] += (xin ? d1m(z0[-2 * DX], mu[-2 * DX], z0[-DX], mu[-DX], z0[DX], mu[DX], z0[2 * DX], mu[2 * DX])
                   : d1_prod_row(dx_line(c, DV_Z0, zh), mux, ix, g.nx, c.rows)) * a.idx;
    acc[2] += d1m(th.qZ1[0], th.qmu[0], th.qZ1[1], th.qmu[1], th.qZ1[3], th.qmu[3], th.qZ1[4], th.qmu[4]) * a.idy;

    // update, scaling (x/z faces), taper; SAT is added by the face kernel
    const float dt2 = a.dt * a.dt;
    const float irho = 1.0f / a.m[2][i];
    const bool face = !(XF && ZF) && (ix == 0 || ix == g.nx - 1 || iz == 0 || iz == g.nz - 1);
    const bool tz = in_taper(a, ix, y, iz);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float p = a.prev[k][c.so + i];
        const float pe = (a.taper_prev && tz) ? taper(a, p, ix, y, iz) : p;
        float v = dt2 * acc[k] * irho + 2.f * ub[k * UC + r0] - pe;
        if (face) v = boundary_scale(a, v, k, ix, y, iz);
        if (tz) v = taper(a, v, ix, y, iz);
        a.next[k][c.so + i] = v;
    }
}

// Tile origin and end of the output rows of tile k along an axis of n points
// tiled by T: regular tiles start at k*T, the last one is shifted to end at n
// and the one before it stops where the last begins, so that every row of the
// SBP closures belongs to the first or the last tile, whose windows hold all
// samples those rows read.
FWI_HD void tile_range(int k, int n, int T, int &origin, int &end)
{
    const int K = (n + T - 1) / T;
    if (k == K - 1) {
        origin = n - T;
        end = n;
    } else {
        origin = k * T;
        end = k * T + T < n - T ? k * T + T : n - T;
    }
}

// A tile (window origin x0, T points) whose outputs and derived halo all lie
// at least 6 points inside the grid along its axis: no SBP closure row.
FWI_HD bool fz_interior_tile(int x0, int T, int n) { return x0 >= 6 && x0 + T <= n - 6; }

// Tile indices [lo, hi) of the interior tiles along an axis of n points (the
// predicate is monotone in the tile origin, so they are contiguous).
inline void fz_interior_range(int n, int T, int &lo, int &hi)
{
    const int K = (n + T - 1) / T;
    lo = K;
    hi = K;
    for (int k = 0; k < K; k++) {
        int o, e;
        tile_range(k, n, T, o, e);
        if (fz_interior_tile(o, T, n)) {
            if (lo == K) lo = k;
            hi = k + 1;
        }
    }
    if (lo == K) lo = hi = 0;
}

// The march of one CTA over output planes [ya, yb) (all inside [6, ny-6)).
template <int PH>
FWI_HD void fz_prologue(FusedCtx &c, int tid, int ya)
{
    for (int q = ya - 4; q < ya; q++) fz_load_u(c, tid, q, ring<PH>(q));
}

}  // namespace fwi
