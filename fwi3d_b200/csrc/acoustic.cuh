// Acoustic variable-density time step as a 2.5-D marching kernel: every
// output point gets the reference's operator (we_op.cpp:1640-1796) -- D2var
// along x, y, z with the 1/rho coefficient, the SAT penalties of its faces,
// the leapfrog update with K, absorbing scaling and taper -- with the
// pressure of five planes and the coefficient of the output plane staged in
// shared memory.
//
// Blocking: a CTA owns a TZ x TX tile of (z, x) columns and marches along y
// over a chunk of planes; shared memory holds a 5-plane ring of the pressure
// over the tile + 2-point halo and the 1/rho plane of the output plane
// (tile + 2-point halo).  The y-direction coefficients of the own column sit
// in a 5-deep register queue.  Rows of the SBP closures along x and z lie in
// the first and last tile of each axis (tile_range), whose windows hold all
// samples those rows read; along y the closure rows (6 planes at each wall)
// read their column from global memory.  Tiles whose x and z ranges are
// interior (template flag F) take closure-free constant-offset code.
#pragma once

#include "fused.cuh"

namespace fwi {

namespace fa {
constexpr int TZ = 32, TX = 16, NT = TZ * TX;
constexpr int H = 2, ZW = TZ + 2 * H, XW = TX + 2 * H;
constexpr int NR = 5;
}  // namespace fa

struct AcousticSmem {
    float p[fa::NR][fa::XW][fa::ZW];
    float b[fa::XW][fa::ZW];
};

struct AcousticCtx {
    const StepArgs *a;
    int64_t so;
    int x0, z0, xend, zend;
    AcousticSmem *sm;
};

FWI_HD int fa_slot(int q) { return ((q % fa::NR) + fa::NR) % fa::NR; }

// Pressure plane q and (optionally) the 1/rho plane y over the window.
FWI_HD void fa_load(const AcousticCtx &c, int tid, int q, bool with_b, int y)
{
    const Dims &g = c.a->g;
    const int s = fa_slot(q);
    for (int p = tid; p < fa::XW * fa::ZW; p += fa::NT) {
        const int xw = p / fa::ZW, zw = p - xw * fa::ZW;
        const int ix = c.x0 - fa::H + xw, iz = c.z0 - fa::H + zw;
        const bool in = ix >= 0 && ix < g.nx && iz >= 0 && iz < g.nz;
        if (q >= 0 && q < g.ny) c.sm->p[s][xw][zw] = in ? c.a->curr[0][c.so + g.idx(ix, q, iz)] : 0.f;
        if (with_b) c.sm->b[xw][zw] = in ? c.a->m[1][g.idx(ix, y, iz)] : 0.f;
    }
}

// Output phase at plane y of the own point; qb: 1/rho at y-2..y+2 (own column).
template <bool F>
FWI_HD void fa_output(const AcousticCtx &c, int tid, int y, const float *qb)
{
    const StepArgs &a = *c.a;
    const Dims &g = a.g;
    const int lz = tid % fa::TZ, lx = tid / fa::TZ;
    const int ix = c.x0 + lx, iz = c.z0 + lz;
    if (ix >= c.xend || iz >= c.zend) return;
    const int64_t i = g.idx(ix, y, iz);
    const int xw = lx + fa::H, zw = lz + fa::H;
    const AcousticSmem &s = *c.sm;
    const float *pc = &s.p[fa_slot(y)][xw][zw];
    const float *bc = &s.b[xw][zw];
    constexpr int X = fa::ZW;
    const float idx2 = 1.0f / (a.dx * a.dx), idy2 = 1.0f / (a.dy * a.dy), idz2 = 1.0f / (a.dz * a.dz);
    float acc;
    // x (we_op.cpp:1664): interior 5-point variable-coefficient stencil, closure rows per point
    if (F || (ix >= 6 && ix < g.nx - 6)) {
        const W5 w = d2w(bc[-2 * X], bc[-X], bc[0], bc[X], bc[2 * X]);
        acc = d2apply(w, idx2, pc[-2 * X], pc[-X], pc[0], pc[X], pc[2 * X]);
    } else {
        const SX ul{&s.p[fa_slot(y)][0][zw], c.x0 - fa::H, fa::ZW}, bl{&s.b[0][zw], c.x0 - fa::H, fa::ZW};
        acc = d2var_row(ul, bl, ix, g.nx, idx2);
    }
    // y (we_op.cpp:1665)
    if (y >= 6 && y < g.ny - 6) {
        const W5 w = d2w(qb[0], qb[1], qb[2], qb[3], qb[4]);
        const int o = fa::XW * fa::ZW;
        const float *p0 = &s.p[0][xw][zw];
        acc += d2apply(w, idy2, p0[fa_slot(y - 2) * o], p0[fa_slot(y - 1) * o], pc[0], p0[fa_slot(y + 1) * o],
                       p0[fa_slot(y + 2) * o]);
    } else {
        acc += d2var_row(g.ly(a.curr[0] + c.so, ix, iz), g.ly(a.m[1], ix, iz), y, g.ny, idy2);
    }
    // z (we_op.cpp:1666)
    if (F || (iz >= 6 && iz < g.nz - 6)) {
        const W5 w = d2w(bc[-2], bc[-1], bc[0], bc[1], bc[2]);
        acc += d2apply(w, idz2, pc[-2], pc[-1], pc[0], pc[1], pc[2]);
    } else {
        const SZ ul{&s.p[fa_slot(y)][xw][0], c.z0 - fa::H}, bl{&s.b[xw][0], c.z0 - fa::H};
        acc += d2var_row(ul, bl, iz, g.nz, idz2);
    }
    // SAT of the faces within 4 points (we_op.cpp:1668-1755), update, scaling, taper
    const bool nearface = ix < 4 || ix >= g.nx - 4 || iz < 4 || iz >= g.nz - 4 || y < 4 || y >= g.ny - 4;
    if (nearface) {
        StepArgs b = shot_args(a, (int)(c.so / a.sst));
        acc = acoustic_sat(b, acc, ix, y, iz);
    }
    const float dt2 = a.dt * a.dt;
    const bool tz = in_taper(a, ix, y, iz);
    const float p = a.prev[0][c.so + i];
    const float pe = (a.taper_prev && tz) ? taper(a, p, ix, y, iz) : p;
    float v = dt2 * acc * a.m[0][i] + 2.f * pc[0] - pe;
    if (nearface) v = boundary_scale(a, v, 0, ix, y, iz);
    if (tz) v = taper(a, v, ix, y, iz);
    a.next[0][c.so + i] = v;
}

// The march of one CTA over output planes [ya, yb); `par(phase)` runs the
// phase for every thread of the block and then synchronises it.
template <bool F, class Par>
FWI_HD void fa_march(const AcousticCtx &c, int ya, int yb, Par &&par)
{
    const Dims &g = c.a->g;
    par([&](int tid) {
        for (int q = ya - 2; q < ya + 2; q++) fa_load(c, tid, q, false, 0);
    });
    for (int y = ya; y < yb; y++) {
        par([&](int tid) { fa_load(c, tid, y + 2, true, y); });
        par([&](int tid) {
            const int lz = tid % fa::TZ, lx = tid / fa::TZ;
            const int ix = c.x0 + lx, iz = c.z0 + lz;
            float q5[5];
            for (int k = 0; k < 5; k++) {
                const int yy = y - 2 + k;
                q5[k] = (yy >= 0 && yy < g.ny) ? c.a->m[1][g.idx(ix, yy, iz)] : 0.f;
            }
            fa_output<F>(c, tid, y, q5);
        });
    }
}

}  // namespace fwi
