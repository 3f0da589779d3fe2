// Paired isotropic interior kernel (pair.cuh): the march of a CTA, the
// kernel and its host launcher.  A translation unit of its own, with its own
// constant-memory copy of the SBP tables (uploaded by pair_init).
#include <cuda_runtime.h>

#include "pair.cuh"
#include "tma.cuh"

namespace fwi {
namespace {

// March of one interior-tile CTA over output planes [ya, yb) of [6, ny-6):
// the ring and plane copies of the fused kernel, with 256 threads that own
// two z-adjacent points each.  Every global load is issued a phase ahead of
// its use: the material plane of the next step by asynchronous copies during
// the update phase, the column's materials before the first barrier, rho and
// prev before the second.  Two block barriers per plane: the derived planes
// and the material plane are written between them, and no phase after the
// second reads the material plane or a ring slot that the next step's copies
// overwrite.
template <bool EVEN, bool XC, bool ZC>
__device__ __forceinline__ void pair_march(FusedCtx &c, int tid, int ya, int yb)
{
    PairThread th;
#pragma unroll
    for (int k = 0; k < 5; k++) th.qmu[k] = th.qT[k] = th.qX1[k] = th.qZ1[k] = f2s(0.f);
    const PairK K = pair_consts(*c.a);
    constexpr bool ZQ = ZC && !XC;  // thread layout of the z-face tiles (pz_pos)
    const PairTaper tp = pair_taper<ZQ>(c, tid);
    if (c.tma && tid == 0) fz_bar_init(c);
    if (XC || ZC) fill_pair_rows(c.sm->rows, tid, pz::NT);
    for (int q = ya - 4; q < ya; q++) pz_load_u<false>(c, tid, q, ring<ELASTIC>(q));
    __syncthreads();
    for (int y = ya - 4; y < yb; y++) {
        fz_slots<ELASTIC>(c, y);
        const ColIn cin = pz_col_in<EVEN, ZQ>(c, tid, y + 2);
        pz_prefetch_next(c, tid, y);
        // plane y+4: copied in here on the first step, else during the previous one
        if (y == ya - 4) {
            if (!c.tma) pz_load_u<false>(c, tid, y + 4, c.sl[6]);
            else if (tid == 0 && !c.dead) fz_tma_issue(c, y + 4, c.sl[6]);
        } else {
            cpa_wait();  // material plane y (and, without bulk copies, ring plane y+4)
        }
        __syncthreads();
        // plane y+5 (< ny - 1) into the slot of plane y-3, which no phase of this step reads
        if (!c.tma) {
            pz_load_u<true>(c, tid, y + 5, ring<ELASTIC>(y + 5));
            cpa_commit();
        } else if (tid == 0 && !c.dead) {
            fz_tma_issue(c, y + 5, ring<ELASTIC>(y + 5));
        }
        if (c.tma) fz_tma_wait(c, c.sl[6]);
        pz_column<XC, ZC>(c, K, th, tid, cin);
        F2 acc[3];
        UpdIn uin;
        if (y >= ya) {
            pz_phase_b<XC, ZC>(c, K, th, tid, y, acc);
            uin = pz_upd_in<EVEN, ZQ>(c, tid, y);
        }
        __syncthreads();
        // material plane y+1 for the next step (phase B of this one has read plane y)
        if (y + 1 >= ya && y + 1 < yb) {
            pz_load_mat<EVEN, true>(c, tid, y + 1);
            cpa_commit();
        }
        if (y >= ya) pz_phase_c<EVEN, XC, ZC>(c, K, th, tid, y, acc, uin, tp);
    }
    cpa_wait();
    if (c.tma) fz_tma_wait(c, ring<ELASTIC>(yb + 4));  // the copy issued in the last step
}

// Paired isotropic step.  grid: (z tiles, x tiles, y chunks x shots), block
// 256.  EVEN: nz even, so every pair is 8-byte aligned in global memory.
// MODE 1: the interior tiles only (tile indices offset by (bz0, bx0)).  The
// edge tiles, with the closure rows of the faces they touch (the grid covers
// every tile, the others return at once): MODE 3 the tiles that touch an x
// face only, MODE 4 a z face only, MODE 5 both.  Separate launches give each
// variant its own register allocation and a smaller instruction footprint.
template <bool EVEN, int MODE>
__global__ void __launch_bounds__(pz::NT, 2)
    k_elastic_pair(const __grid_constant__ StepArgs a, int nchunks, const __grid_constant__ FusedTma t, int bz0,
                   int bx0)
{
    extern __shared__ __align__(128) unsigned char fz_smem[];
    FusedCtx c;
    c.a = &a;
    c.sm = reinterpret_cast<FusedSmem *>(fz_smem);
    c.tmap = &t.u;
    c.err = t.err;
    c.tma = t.on && (fz_saddr(fz_smem) & 127u) == 0;
    c.rows.p = c.sm->rows;
    const int tid = threadIdx.x;
    c.shot = blockIdx.z / nchunks;
    if (shot_idle(a, c.shot)) return;
    const int ch = blockIdx.z - c.shot * nchunks;
    c.so = c.shot * a.sst;
    tile_range(blockIdx.x + (MODE == 1 ? bz0 : 0), a.g.nz, fz::TZ, c.z0, c.zend);
    tile_range(blockIdx.y + (MODE == 1 ? bx0 : 0), a.g.nx, fz::TX, c.x0, c.xend);
    const int len = a.y1 - a.y0;
    const int ya = a.y0 + (int)((int64_t)len * ch / nchunks);
    const int yb = a.y0 + (int)((int64_t)len * (ch + 1) / nchunks);
    if (ya >= yb) return;
    if (MODE == 1) {
        pair_march<EVEN, false, false>(c, tid, ya, yb);
        return;
    }
    const bool xi = fz_interior_tile(c.x0, fz::TX, a.g.nx), zi = fz_interior_tile(c.z0, fz::TZ, a.g.nz);
    if (MODE == 3 && !xi && zi) pair_march<EVEN, true, false>(c, tid, ya, yb);
    if (MODE == 4 && xi && !zi) pair_march<EVEN, false, true>(c, tid, ya, yb);
    if (MODE == 5 && !xi && !zi) pair_march<EVEN, true, true>(c, tid, ya, yb);
}

}  // namespace

template <int MODE>
static void launch_mode(bool even, dim3 grid, size_t smem, cudaStream_t s, const StepArgs &a, int nchunks, const FusedTma &t,
                 int bz0, int bx0)
{
    if (even) k_elastic_pair<true, MODE><<<grid, pz::NT, smem, s>>>(a, nchunks, t, bz0, bx0);
    else k_elastic_pair<false, MODE><<<grid, pz::NT, smem, s>>>(a, nchunks, t, bz0, bx0);
}

cudaError_t pair_init()
{
    init_sbp_tables();
    cudaError_t e = cudaMemcpyToSymbol(c_sbp, &g_sbp_host, sizeof(SbpTables));
    const void *k[8] = {(const void *)k_elastic_pair<true, 1>,  (const void *)k_elastic_pair<true, 3>,
                        (const void *)k_elastic_pair<true, 4>,  (const void *)k_elastic_pair<true, 5>,
                        (const void *)k_elastic_pair<false, 1>, (const void *)k_elastic_pair<false, 3>,
                        (const void *)k_elastic_pair<false, 4>, (const void *)k_elastic_pair<false, 5>};
    for (int i = 0; i < 8 && e == cudaSuccess; i++)
        e = cudaFuncSetAttribute(k[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FusedSmem));
    return e;
}

void pair_launch(bool even, int mode, dim3 grid, size_t smem, cudaStream_t s, const StepArgs &a, int nchunks,
                 const FusedTma &t, int bz0, int bx0)
{
    switch (mode) {
    case 1: launch_mode<1>(even, grid, smem, s, a, nchunks, t, bz0, bx0); break;
    case 3: launch_mode<3>(even, grid, smem, s, a, nchunks, t, 0, 0); break;
    case 4: launch_mode<4>(even, grid, smem, s, a, nchunks, t, 0, 0); break;
    default: launch_mode<5>(even, grid, smem, s, a, nchunks, t, 0, 0); break;
    }
}

}  // namespace fwi
