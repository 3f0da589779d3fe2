// Host run of the elastic step's GPU phases, thread by thread, against the
// per-point step (elastic_aux_point + elastic_point, the per-point kernels'
// code).  The fused and marching kernels' phases are host/device functions of
// (context, thread index); this program runs them in the kernels' order with
// every block barrier as a loop boundary, on a seeded grid:
//   planes [6, ny-6): the fused kernel's tiles (chunks along y as the launch
//     splits them; the isotropic edge tiles with the per-axis code of the
//     split launch, the VTI tiles as the single launch), plane copies done
//     synchronously;
//   the 6 planes next to each y wall: the marching kernel in slab mode;
//   then the face SAT pass (k_elastic_face_sat) on every face point.
// PH 2 runs the acoustic marching kernel (k_acoustic_fused: every plane, SAT
// inline) against the acoustic per-point step instead.
// PH 13 / 16 (isotropic / VTI + 10) checks the imaging increments instead:
// the closure-free interior taps of k_image_batch against its
// closure-capable per-point code at every interior point.
// Usage: phases PH nx ny nz nchunks bcset taper tables
//   PH 2 acoustic / 3 isotropic / 6 VTI (13 / 16 imaging); bcset 0..2;
//   tables 1: closure weights from the per-model tables (k_w2c), 0: formed
//   in place.
// Prints "rel <relative L2> max <max abs> nan <count>".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "fused.cuh"
#include "march.cuh"
#include "acoustic.cuh"
#include "imaging.cuh"
#include "host_ops.h"

using namespace fwi;

namespace {

struct Grid {
    int nm, nx, ny, nz;
    int64_t n;
};

// per-point step of every point (the reference-ordered per-point kernels)
void per_point(const StepArgs &a, const Grid &G, std::vector<float> &out)
{
    std::vector<float> aux(9 * G.n);
    AuxArgs x;
    std::memset(&x, 0, sizeof(x));
    x.g = a.g;
    x.dx = a.dx;
    x.dy = a.dy;
    x.dz = a.dz;
    for (int k = 0; k < G.nm; k++) x.m[k] = a.m[k];
    for (int c = 0; c < 3; c++) x.curr[c] = a.curr[c];
    for (int k = 0; k < 9; k++) x.aux[k] = aux.data() + k * G.n;
    if (G.nm == 3) x.aux[AUX_T1] = x.aux[AUX_T2] = x.aux[AUX_T0];
    for (int iy = 0; iy < G.ny; iy++)
        for (int ix = 0; ix < G.nx; ix++)
            for (int iz = 0; iz < G.nz; iz++) {
                if (G.nm == 3) elastic_aux_point<ELASTIC>(x, ix, iy, iz);
                else elastic_aux_point<VTI>(x, ix, iy, iz);
            }
    StepArgs r = a;
    for (int k = 0; k < 9; k++) r.aux[k] = x.aux[k];
    for (int iy = 0; iy < G.ny; iy++)
        for (int ix = 0; ix < G.nx; ix++)
            for (int iz = 0; iz < G.nz; iz++)
                for (int c = 0; c < 3; c++)
                    out[c * G.n + a.g.idx(ix, iy, iz)] = G.nm == 3 ? elastic_point<ELASTIC>(r, c, ix, iy, iz)
                                                                   : elastic_point<VTI>(r, c, ix, iy, iz);
}

// one fused tile column over planes [ya, yb): the kernel's march loop
template <int PH, bool XF, bool ZF, bool AX>
void fused_tile(FusedCtx &c, int ya, int yb)
{
    std::vector<FusedThread> th(fz::NT);
    for (auto &t : th)
        for (int k = 0; k < 5; k++) t.qmu[k] = t.qeps[k] = t.q66[k] = t.qT[k] = t.qX1[k] = t.qZ1[k] = 0.f;
    fill_smem_rows(c.sm->rows, 0, 1);
    for (int t = 0; t < fz::NT; t++) fz_prologue<PH>(c, t, ya);
    for (int y = ya - 4; y < yb; y++) {
        fz_slots<PH>(c, y);
        for (int t = 0; t < fz::NT; t++) {
            if (PH == VTI || y == ya - 4) fz_load_u(c, t, y + 4, c.sl[6]);
            if (y >= ya) fz_load_mat<PH>(c, t, y);
        }
        if (PH == ELASTIC)
            for (int t = 0; t < fz::NT; t++) fz_load_u(c, t, y + 5, ring<PH>(y + 5));
        for (int t = 0; t < fz::NT; t++) fz_column<PH, XF, ZF>(c, th[t], t, y + 2);
        if (y >= ya)
            for (int t = 0; t < fz::NT; t++) fz_derived<PH, XF, ZF>(c, t, y);
        if (y >= ya)
            for (int t = 0; t < fz::NT; t++) {
                if (PH == ELASTIC && !(XF && ZF) && !(AX && (XF || ZF))) fz_output<PH>(c, th[t], t, y);
                else fz_output_t<PH, XF, ZF>(c, th[t], t, y);
            }
    }
}

template <int PH>
void fused_planes(const StepArgs &a, int nch)
{
    const Dims &g = a.g;
    FusedSmem *sm = new FusedSmem;
    const int kz = (g.nz + fz::TZ - 1) / fz::TZ, kx = (g.nx + fz::TX - 1) / fz::TX;
    const int y0 = fz::YPAD, len = g.ny - 2 * fz::YPAD;
    for (int bz = 0; bz < kz; bz++)
        for (int bx = 0; bx < kx; bx++)
            for (int ch = 0; ch < nch; ch++) {
                FusedCtx c;
                c.a = &a;
                c.sm = sm;
                c.shot = 0;
                c.so = 0;
                c.rows.p = sm->rows;
                tile_range(bz, g.nz, fz::TZ, c.z0, c.zend);
                tile_range(bx, g.nx, fz::TX, c.x0, c.xend);
                const int ya = y0 + (int)((int64_t)len * ch / nch), yb = y0 + (int)((int64_t)len * (ch + 1) / nch);
                if (ya >= yb) continue;
                for (size_t k = 0; k < sizeof(FusedSmem) / 4; k++) ((float *)sm)[k] = NAN;
                const bool xf = fz_interior_tile(c.x0, fz::TX, g.nx), zf = fz_interior_tile(c.z0, fz::TZ, g.nz);
                constexpr bool AX = PH == ELASTIC;  // the isotropic edge launch keeps the interior axis
                if (xf && zf) fused_tile<PH, true, true, AX>(c, ya, yb);
                else if (xf) fused_tile<PH, true, false, AX>(c, ya, yb);
                else if (zf) fused_tile<PH, false, true, AX>(c, ya, yb);
                else fused_tile<PH, false, false, AX>(c, ya, yb);
            }
    delete sm;
}

template <int PH>
void march_slabs(const StepArgs &a)
{
    const Dims &g = a.g;
    MarchSmem *sm = new MarchSmem;
    const int kz = (g.nz + f3::TZ - 1) / f3::TZ, kx = (g.nx + f3::TX - 1) / f3::TX;
    auto par = [&](auto &&phase) {
        for (int t = 0; t < f3::NT; t++) phase(t);
    };
    for (int bz = 0; bz < kz; bz++)
        for (int bx = 0; bx < kx; bx++)
            for (int side = 0; side < 2; side++) {
                MarchCtx c;
                c.a = &a;
                c.sm = sm;
                c.so = 0;
                c.rows.p = sm->rows;
                tile_range(bz, g.nz, f3::TZ, c.z0, c.zend);
                tile_range(bx, g.nx, f3::TX, c.x0, c.xend);
                const int ya = side ? g.ny - fz::YPAD : 0, yb = side ? g.ny : fz::YPAD;
                for (size_t k = 0; k < sizeof(MarchSmem) / 4; k++) ((float *)sm)[k] = NAN;
                fill_smem_rows(sm->rows, 0, 1);
                const bool xf = m3_fast(c.x0, g.nx, f3::TX), zf = m3_fast(c.z0, g.nz, f3::TZ);
                if (xf && zf) m3_march<PH, true, true>(c, ya, yb, par);
                else if (xf) m3_march<PH, true, false>(c, ya, yb, par);
                else if (zf) m3_march<PH, false, true>(c, ya, yb, par);
                else m3_march<PH, false, false>(c, ya, yb, par);
            }
    delete sm;
}

// k_elastic_face_sat on every face point
template <int PH>
void face_sat(const StepArgs &a)
{
    const Dims &g = a.g;
    for (int iy = 0; iy < g.ny; iy++)
        for (int ix = 0; ix < g.nx; ix++)
            for (int iz = 0; iz < g.nz; iz++) {
                if (!(ix == 0 || iy == 0 || iz == 0 || ix == g.nx - 1 || iy == g.ny - 1 || iz == g.nz - 1)) continue;
                const int64_t i = g.idx(ix, iy, iz);
                for (int c = 0; c < 3; c++) {
                    const float sat = elastic_sat<PH>(a, 0.f, c, ix, iy, iz, 0);
                    if (sat == 0.f) continue;
                    float v = a.dt * a.dt / a.m[2][i] * sat;
                    v = boundary_scale(a, v, c, ix, iy, iz);
                    v = taper(a, v, ix, iy, iz);
                    a.next[c][i] += v;
                }
            }
}

// k_acoustic_fused over every tile and y chunk
void acoustic_march(const StepArgs &a, int nch)
{
    const Dims &g = a.g;
    AcousticSmem *sm = new AcousticSmem;
    const int kz = (g.nz + fa::TZ - 1) / fa::TZ, kx = (g.nx + fa::TX - 1) / fa::TX;
    auto par = [&](auto &&phase) {
        for (int t = 0; t < fa::NT; t++) phase(t);
    };
    for (int bz = 0; bz < kz; bz++)
        for (int bx = 0; bx < kx; bx++)
            for (int ch = 0; ch < nch; ch++) {
                AcousticCtx c;
                c.a = &a;
                c.sm = sm;
                c.so = 0;
                tile_range(bz, g.nz, fa::TZ, c.z0, c.zend);
                tile_range(bx, g.nx, fa::TX, c.x0, c.xend);
                const int ya = (int)((int64_t)g.ny * ch / nch), yb = (int)((int64_t)g.ny * (ch + 1) / nch);
                if (ya >= yb) continue;
                for (size_t k = 0; k < sizeof(AcousticSmem) / 4; k++) ((float *)sm)[k] = NAN;
                const bool fast = c.x0 >= 6 && c.x0 + fa::TX <= g.nx - 6 && c.z0 >= 6 && c.z0 + fa::TZ <= g.nz - 6;
                if (fast) fa_march<true>(c, ya, yb, par);
                else fa_march<false>(c, ya, yb, par);
            }
    delete sm;
}

// closure-weight tables of k_w2c, on the host
struct W2cHost {
    Line mu, eps, c66;
    int f;
    float operator()(int k) const
    {
        if (f == 0) return mu(k);
        if (f == 1) return c66(k);
        return 2.f * (1.f + 2.f * eps(k)) * mu(k);
    }
};
void w2c_tables(const StepArgs &a, const Grid &G, std::vector<float> tab[3][3], StepArgs &out)
{
    const Dims &g = a.g;
    const int64_t nl[3] = {(int64_t)g.ny * g.nz, (int64_t)g.nx * g.nz, (int64_t)g.ny * g.nx};
    const int nf[3] = {G.nm == 6 ? 3 : 1, G.nm == 6 ? 3 : 1, 1};
    for (int ax = 0; ax < 3; ax++)
        for (int f = 0; f < nf[ax]; f++) {
            tab[ax][f].resize(nl[ax] * 96);
            for (int64_t e = 0; e < nl[ax] * 12; e++) {
                const int64_t line = e / 12;
                const int slot = (int)(e - line * 12);
                int64_t base, stride;
                int n;
                if (ax == 0) {
                    const int64_t y = line / g.nz, z = line - y * g.nz;
                    base = y * g.nx * g.nz + z;
                    stride = g.nz;
                    n = g.nx;
                } else if (ax == 1) {
                    const int64_t x = line / g.nz, z = line - x * g.nz;
                    base = x * g.nz + z;
                    stride = (int64_t)g.nx * g.nz;
                    n = g.ny;
                } else {
                    const int64_t y = line / g.nx, x = line - y * g.nx;
                    base = (y * g.nx + x) * g.nz;
                    stride = 1;
                    n = g.nz;
                }
                const W2cHost l{Line{a.m[1], base, stride}, Line{f == 2 ? a.m[4] : a.m[1], base, stride},
                                Line{f == 1 ? a.m[5] : a.m[1], base, stride}, f};
                const int i = slot < 6 ? slot : n - 1 - (slot - 6);
                const W8 w = d2closure_weights(l, i, n, ConstRows());
                for (int j = 0; j < 8; j++) tab[ax][f][e * 8 + j] = w.w[j];
            }
            out.w2c[ax][f] = tab[ax][f].data();
        }
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 9) {
        std::fprintf(stderr, "usage: phases PH nx ny nz nchunks bcset taper tables\n");
        return 2;
    }
    Grid G;
    G.nm = std::atoi(argv[1]);
    const bool imaging = G.nm > 10;
    if (imaging) G.nm -= 10;
    G.nx = std::atoi(argv[2]);
    G.ny = std::atoi(argv[3]);
    G.nz = std::atoi(argv[4]);
    const int nch = std::atoi(argv[5]), bcs = std::atoi(argv[6]), tw = std::atoi(argv[7]), tables = std::atoi(argv[8]);
    G.n = (int64_t)G.nx * G.ny * G.nz;
    init_sbp_tables();
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    std::vector<float> model(G.nm * G.n);
    for (int64_t i = 0; i < G.n && G.nm == 2; i++) {
        model[i] = 4.0f + 1.0f * U(rng);             // K
        model[G.n + i] = 0.45f + 0.1f * U(rng);      // 1/rho
    }
    for (int64_t i = 0; i < G.n && G.nm != 2; i++) {
        model[i] = 2.0f + 0.5f * U(rng);          // lambda
        model[G.n + i] = 1.5f + 0.4f * U(rng);    // mu
        model[2 * G.n + i] = 2.2f + 0.3f * U(rng);  // rho
        if (G.nm == 6) {
            model[3 * G.n + i] = model[i] * 0.9f;                 // c13
            model[4 * G.n + i] = 0.1f + 0.05f * U(rng);           // eps
            model[5 * G.n + i] = model[G.n + i] * (1.1f + 0.05f * U(rng));  // c66
        }
    }
    std::vector<float> prev(3 * G.n), curr(3 * G.n), ref(3 * G.n, 0.f), got(3 * G.n, NAN);
    for (auto &v : prev) v = U(rng);
    for (auto &v : curr) v = U(rng);
    int bc[6] = {1, 2, 2, 2, 2, 2};
    if (bcs == 1) {
        const int b[6] = {2, 1, 2, 1, 2, 1};
        std::memcpy(bc, b, sizeof(bc));
    } else if (bcs == 2) {
        const int b[6] = {1, 1, 1, 1, 1, 1};
        std::memcpy(bc, b, sizeof(bc));
    }
    const int tapw[6] = {0, tw, tw, tw, tw, tw};
    const float dx = 0.01f, dy = 0.011f, dz = 0.009f, dt = 0.0008f;
    ScaleTables st = boundary_divisors(model.data(), G.nm, G.nx, G.ny, G.nz, dx, dy, dz, dt, bc);
    TaperTables tt = taper_tables(G.nx, G.ny, G.nz, tapw, 0.05f);
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = Dims{G.nx, G.ny, G.nz};
    a.dx = dx;
    a.dy = dy;
    a.dz = dz;
    a.dt = dt;
    a.idx = 1.0f / dx;
    a.idy = 1.0f / dy;
    a.idz = 1.0f / dz;
    const float d[3] = {dx, dy, dz};
    for (int k = 0; k < 3; k++) {
        a.ad1[k] = 1.0f / (d[k] * d[k]);
        a.ad2[k] = 2.0f / (d[k] * d[k]);
    }
    for (int k = 0; k < G.nm; k++) a.m[k] = model.data() + k * G.n;
    int scale = 0;
    for (int f = 0; f < 6; f++) {
        a.bc[f] = bc[f];
        a.tap[f] = tt.t[f].data();
        a.tw[f] = tapw[f];
        scale |= bc[f] == 2;
        for (int c = 0; c < 3; c++) a.sdiv[f][c] = st.f[f][c].data();
    }
    a.scale = scale;
    a.alpha_fs = 0.2508560249f;
    a.taper_prev = 1;
    a.sst = 3 * G.n;
    a.ast = 9 * G.n;
    a.y0 = 0;
    a.y1 = G.ny;
    for (int c = 0; c < 3; c++) {
        a.curr[c] = curr.data() + c * G.n;
        a.prev[c] = prev.data() + c * G.n;
    }
    if (imaging) {
        // three snapshot levels and the lagged / current adjoint fields
        std::vector<float> f3(9 * G.n), adj(3 * G.n), lag(3 * G.n);
        for (auto &v : f3) v = U(rng);
        for (auto &v : adj) v = U(rng);
        for (auto &v : lag) v = U(rng);
        ImageArgs im;
        std::memset(&im, 0, sizeof(im));
        im.g = a.g;
        im.dx = dx;
        im.dy = dy;
        im.dz = dz;
        im.rdx = 1.0f / dx;
        im.rdy = 1.0f / dy;
        im.rdz = 1.0f / dz;
        im.dtimg = dt;
        im.itl = 5;
        im.last = 10;
        for (int k = 0; k < G.nm; k++) im.m[k] = a.m[k];
        for (int l = 0; l < 3; l++)
            for (int c = 0; c < 3; c++) im.fwd[l][c] = f3.data() + (3 * l + c) * G.n;
        for (int c = 0; c < 3; c++) {
            im.adj[c] = adj.data() + c * G.n;
            im.lag[c] = lag.data() + c * G.n;
        }
        double num = 0, den = 0, mx = 0;
        int64_t nan = 0;
        for (int iy = 4; iy < G.ny - 4; iy++)
            for (int ix = 4; ix < G.nx - 4; ix++)
                for (int iz = 4; iz < G.nz - 4; iz++) {
                    double f[3], r[3];
                    if (G.nm == 3) {
                        elastic_image_inc<ELASTIC, true>(im, 0, ix, iy, iz, f[0], f[1], f[2]);
                        elastic_image_inc<ELASTIC, false>(im, 0, ix, iy, iz, r[0], r[1], r[2]);
                    } else {
                        elastic_image_inc<VTI, true>(im, 0, ix, iy, iz, f[0], f[1], f[2]);
                        elastic_image_inc<VTI, false>(im, 0, ix, iy, iz, r[0], r[1], r[2]);
                    }
                    for (int k = 0; k < 3; k++) {
                        if (!std::isfinite(f[k])) {
                            nan++;
                            continue;
                        }
                        num += (f[k] - r[k]) * (f[k] - r[k]);
                        den += r[k] * r[k];
                        mx = std::fmax(mx, std::fabs(f[k] - r[k]));
                    }
                }
        std::printf("rel %.3e max %.3e nan %lld\n", std::sqrt(num / den), mx, (long long)nan);
        return 0;
    }
    if (G.nm == 2) {
        // acoustic: one component
        for (int iy = 0; iy < G.ny; iy++)
            for (int ix = 0; ix < G.nx; ix++)
                for (int iz = 0; iz < G.nz; iz++) ref[a.g.idx(ix, iy, iz)] = acoustic_point(a, ix, iy, iz);
        StepArgs b = a;
        b.next[0] = got.data();
        acoustic_march(b, nch);
        double num = 0, den = 0, mx = 0;
        int64_t nan = 0;
        for (int64_t k = 0; k < G.n; k++) {
            if (!std::isfinite(got[k])) {
                nan++;
                continue;
            }
            const double e = (double)got[k] - ref[k];
            num += e * e;
            den += (double)ref[k] * ref[k];
            mx = std::fmax(mx, std::fabs(e));
        }
        std::printf("rel %.3e max %.3e nan %lld\n", std::sqrt(num / den), mx, (long long)nan);
        return 0;
    }
    per_point(a, G, ref);

    StepArgs b = a;
    for (int c = 0; c < 3; c++) b.next[c] = got.data() + c * G.n;
    std::vector<float> tab[3][3];
    if (tables) w2c_tables(a, G, tab, b);
    if (G.nm == 3) {
        march_slabs<ELASTIC>(b);
        fused_planes<ELASTIC>(b, nch);
        face_sat<ELASTIC>(b);
    } else {
        march_slabs<VTI>(b);
        fused_planes<VTI>(b, nch);
        face_sat<VTI>(b);
    }
    double num = 0, den = 0, mx = 0;
    int64_t nan = 0;
    for (int64_t k = 0; k < 3 * G.n; k++) {
        if (!std::isfinite(got[k])) {
            nan++;
            continue;
        }
        const double e = (double)got[k] - ref[k];
        num += e * e;
        den += (double)ref[k] * ref[k];
        mx = std::fmax(mx, std::fabs(e));
    }
    std::printf("rel %.3e max %.3e nan %lld\n", std::sqrt(num / den), mx, (long long)nan);
    return 0;
}
