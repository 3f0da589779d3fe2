// CUDA kernels of one propagation time step and the host time loops.
//
// One time step of the reference (we_op.cpp:623-836 elastic, :1274-1497 VTI,
// :1640-1796 acoustic) becomes, per step and per shot:
//   extract   receivers from curr (forward only)           k_extract
//   aux       first-derivative scratch (elastic/VTI)        k_elastic_aux
//   step      D2var + D1 terms + SAT + update + scale + taper, fused   k_*_step
//   inject    sources (receivers' residual in the adjoint)  k_inject
// and, every `sub` steps of the adjoint, the imaging condition k_image_batch.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "engine.h"
#include "imaging.cuh"
#include "fused.cuh"
#include "tma.cuh"
#include "march.cuh"
#include "acoustic.cuh"
#include "physics.cuh"

namespace fwi {

// Named range of host-side phases (forward, recomputation, adjoint, imaging)
// for timeline tools; without a tool attached a push/pop is a few
// nanoseconds.
struct PhaseRange {
    explicit PhaseRange(const char *name) { nvtxRangePushA(name); }
    ~PhaseRange() { nvtxRangePop(); }
    PhaseRange(const PhaseRange &) = delete;
    PhaseRange &operator=(const PhaseRange &) = delete;
};

#define CK(x)                                                                                               \
    do {                                                                                                    \
        cudaError_t e_ = (x);                                                                               \
        if (e_ != cudaSuccess)                                                                              \
            throw FwiError(e_ == cudaErrorMemoryAllocation ? FWI_ERR_OOM : FWI_ERR_CUDA,                   \
                           std::string(#x) + ": " + cudaGetErrorString(e_));                                \
    } while (0)

// ---------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------
DevBuf::DevBuf(size_t n) { alloc(n); }
DevBuf::~DevBuf()
{
    if (p) cudaFree(p);
}
DevBuf &DevBuf::operator=(DevBuf &&o) noexcept
{
    if (this != &o) {
        if (p) cudaFree(p);
        p = o.p;
        bytes = o.bytes;
        o.p = nullptr;
        o.bytes = 0;
    }
    return *this;
}
void DevBuf::alloc(size_t n)
{
    // same size: keep the buffer (contents are undefined after alloc either
    // way), which spares the batches of an objective evaluation a cudaFree /
    // cudaMalloc pair of their multi-GB snapshot stores
    if (p && bytes == n) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (n == 0) return;
    CK(cudaMalloc(&p, n));
    bytes = n;
}
void DevBuf::zero(void *stream)
{
    if (p) CK(cudaMemsetAsync(p, 0, bytes, (cudaStream_t)stream));
}

// ---------------------------------------------------------------------------
// Kernels (one thread per grid point; launch grid z covers y-blocks x shots)
// ---------------------------------------------------------------------------
namespace {

constexpr int BZ = 32, BX = 4, BY = 2;

// Launch grid z covers (y blocks of planes [y0, y1)) x shots.
__device__ __forceinline__ bool point_of(const Dims &g, int nyb, int y0, int y1, int &ix, int &iy, int &iz, int &s)
{
    iz = blockIdx.x * BZ + threadIdx.x;
    ix = blockIdx.y * BX + threadIdx.y;
    s = blockIdx.z / nyb;
    iy = y0 + (blockIdx.z % nyb) * BY + threadIdx.z;
    return iz < g.nz && ix < g.nx && iy < y1;
}
__device__ __forceinline__ bool point_of(const Dims &g, int nyb, int &ix, int &iy, int &iz, int &s)
{
    return point_of(g, nyb, 0, g.ny, ix, iy, iz, s);
}

int yblocks(int ny) { return (ny + BY - 1) / BY; }
int yblocks(const Dims &g) { return yblocks(g.ny); }
dim3 grid_of(const Dims &g, int nshots, int ny_launch = -1)
{
    return dim3((g.nz + BZ - 1) / BZ, (g.nx + BX - 1) / BX, yblocks(ny_launch < 0 ? g.ny : ny_launch) * nshots);
}

__global__ void k_acoustic_step(StepArgs a)
{
    int ix, iy, iz, s;
    if (!point_of(a.g, a.nyb, a.y0, a.y1, ix, iy, iz, s) || shot_idle(a, s)) return;
    const StepArgs b = shot_args(a, s);
    b.next[0][b.g.idx(ix, iy, iz)] = acoustic_point(b, ix, iy, iz);
}

template <int PH>
__global__ void k_elastic_aux(AuxArgs a)
{
    int ix, iy, iz, s;
    if (!point_of(a.g, a.nyb, a.y0, a.y1, ix, iy, iz, s)) return;
    elastic_aux_point<PH>(shot_args(a, s), ix, iy, iz);
}

template <int PH>
__global__ void k_elastic_step(StepArgs a)
{
    int ix, iy, iz, s;
    if (!point_of(a.g, a.nyb, a.y0, a.y1, ix, iy, iz, s) || shot_idle(a, s)) return;
    const StepArgs b = shot_args(a, s);
    const int64_t i = b.g.idx(ix, iy, iz);
    const float v0 = elastic_point<PH>(b, 0, ix, iy, iz);
    const float v1 = elastic_point<PH>(b, 1, ix, iy, iz);
    const float v2 = elastic_point<PH>(b, 2, ix, iy, iz);
    b.next[0][i] = v0;
    b.next[1][i] = v1;
    b.next[2][i] = v2;
}

// AX: edge tiles of the isotropic kernel take the per-axis output code (the
// split launch); otherwise its edge tiles take the per-point code.
template <int PH, bool XF, bool ZF, bool AX = false>
__device__ __forceinline__ void fused_march(FusedCtx &c, int tid, int ya, int yb)
{
    FusedThread th;
#pragma unroll
    for (int k = 0; k < 5; k++) th.qmu[k] = th.qeps[k] = th.q66[k] = th.qT[k] = th.qX1[k] = th.qZ1[k] = 0.f;
    if (c.tma && tid == 0) fz_bar_init(c);
    fill_smem_rows(c.sm->rows, tid, fz::NT);
    fz_prologue<PH>(c, tid, ya);
    __syncthreads();
    for (int y = ya - 4; y < yb; y++) {
        fz_slots<PH>(c, y);
        // plane y+4: copied in here (VTI, first step) or during the previous
        // iteration (elastic); with bulk-tensor copies it is waited for just
        // before the column phase, the first to read it
        if (PH == VTI || y == ya - 4) {
            if (!c.tma) fz_load_u(c, tid, y + 4, c.sl[6]);
            else if (tid == 0 && !c.dead) fz_tma_issue(c, y + 4, c.sl[6]);
        } else if (!c.tma) {
            cpa_wait();
        }
        if (y >= ya) fz_load_mat<PH>(c, tid, y);
        __syncthreads();
        if (PH == ELASTIC) {
            // plane y+5 (< ny - 1 for every chunk of [6, ny-6)) into the slot of
            // plane y-3, which no phase of this iteration reads
            if (!c.tma) {
                fz_load_u<true>(c, tid, y + 5, ring<PH>(y + 5));
                cpa_commit();
            } else if (tid == 0 && !c.dead) {
                fz_tma_issue(c, y + 5, ring<PH>(y + 5));
            }
        }
        if (c.tma) fz_tma_wait(c, c.sl[6]);
        fz_column<PH, XF, ZF>(c, th, tid, y + 2);
        if (y >= ya) fz_derived<PH, XF, ZF>(c, tid, y);
        __syncthreads();
        if (y >= ya) {
            if (PH == ELASTIC && !(XF && ZF) && !(AX && (XF || ZF))) fz_output<PH>(c, th, tid, y);
            else fz_output_t<PH, XF, ZF>(c, th, tid, y);
        }
        __syncthreads();
    }
    if (!c.tma) cpa_wait();
    else if (PH == ELASTIC) fz_tma_wait(c, ring<PH>(yb + 4));  // the copy issued in the last iteration
}

// Fused elastic step over planes [ylo, yhi) (see fused.cuh).  grid: (z tiles,
// x tiles, y chunks x shots), block (TZ, TX).
template <int PH, int MINB>
__global__ void __launch_bounds__(fz::NT, MINB)
    k_elastic_fused(const __grid_constant__ StepArgs a, int nchunks, const __grid_constant__ FusedTma t)
{
    extern __shared__ __align__(128) unsigned char fz_smem[];
    FusedCtx c;
    c.a = &a;
    c.sm = reinterpret_cast<FusedSmem *>(fz_smem);
    c.tmap = &t.u;
    c.err = t.err;
    c.tma = t.on && (fz_saddr(fz_smem) & 127u) == 0;  // bulk-tensor destinations: 128-byte aligned slots
    c.rows.p = c.sm->rows;
    const int tid = threadIdx.x + fz::TZ * threadIdx.y;
    c.shot = blockIdx.z / nchunks;
    if (shot_idle(a, c.shot)) return;
    const int ch = blockIdx.z - c.shot * nchunks;
    c.so = c.shot * a.sst;
    tile_range(blockIdx.x, a.g.nz, fz::TZ, c.z0, c.zend);
    tile_range(blockIdx.y, a.g.nx, fz::TX, c.x0, c.xend);
    const int len = a.y1 - a.y0;
    const int ya = a.y0 + (int)((int64_t)len * ch / nchunks);
    const int yb = a.y0 + (int)((int64_t)len * (ch + 1) / nchunks);
    if (ya >= yb) return;
    // tiles whose outputs and derived halo are interior in x and z take the
    // closure-free code (block-uniform branch)
    // interior tiles take the closure-free code on both axes; edge tiles of
    // the VTI kernel keep it on their interior axis, those of the isotropic
    // kernel (which measured faster so under the 64-register bound) do not
    const bool xf = c.x0 >= 6 && c.x0 + fz::TX <= a.g.nx - 6, zf = c.z0 >= 6 && c.z0 + fz::TZ <= a.g.nz - 6;
    if (xf && zf) fused_march<PH, true, true>(c, tid, ya, yb);
    else if (PH == VTI && xf) fused_march<PH, true, false>(c, tid, ya, yb);
    else if (PH == VTI && zf) fused_march<PH, false, true>(c, tid, ya, yb);
    else fused_march<PH, false, false>(c, tid, ya, yb);
}

// Isotropic fused step split by tiles: MODE 1 runs the interior tiles only
// (grid tile indices offset by (bz0, bx0)), MODE 2 the edge tiles only (the
// interior tiles of its full grid return at once; with bz0 = 1 also the edge
// tiles that touch no z face).  Separate launches give
// each its own register allocation: the interior code runs without spills
// and the edge tiles can keep the closure-free code on their interior axis.
template <int MODE>
__global__ void __launch_bounds__(fz::NT, 2)
    k_elastic_fused_part(const __grid_constant__ StepArgs a, int nchunks, const __grid_constant__ FusedTma t,
                         int bz0, int bx0)
{
    extern __shared__ __align__(128) unsigned char fz_smem[];
    FusedCtx c;
    c.a = &a;
    c.sm = reinterpret_cast<FusedSmem *>(fz_smem);
    c.tmap = &t.u;
    c.err = t.err;
    c.tma = t.on && (fz_saddr(fz_smem) & 127u) == 0;
    c.rows.p = c.sm->rows;
    const int tid = threadIdx.x + fz::TZ * threadIdx.y;
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
        fused_march<ELASTIC, true, true, true>(c, tid, ya, yb);
        return;
    }
    const bool xf = fz_interior_tile(c.x0, fz::TX, a.g.nx), zf = fz_interior_tile(c.z0, fz::TZ, a.g.nz);
    if (xf && zf) return;
    if (bz0 == 1 && zf) return;  // the tiles that touch an x face only run elsewhere
    if (xf) fused_march<ELASTIC, true, false, true>(c, tid, ya, yb);
    else if (zf) fused_march<ELASTIC, false, true, true>(c, tid, ya, yb);
    else fused_march<ELASTIC, false, false, true>(c, tid, ya, yb);
}

// Acoustic marching step (see acoustic.cuh).  grid: (z tiles, x tiles,
// y chunks x shots), block (TZ, TX).
__global__ void __launch_bounds__(fa::NT, 2) k_acoustic_fused(const __grid_constant__ StepArgs a, int nchunks)
{
    __shared__ AcousticSmem sm;
    AcousticCtx c;
    c.a = &a;
    c.sm = &sm;
    const int tid = threadIdx.x + fa::TZ * threadIdx.y;
    const int shot = blockIdx.z / nchunks;
    if (shot_idle(a, shot)) return;
    const int ch = blockIdx.z - shot * nchunks;
    c.so = shot * a.sst;
    tile_range(blockIdx.x, a.g.nz, fa::TZ, c.z0, c.zend);
    tile_range(blockIdx.y, a.g.nx, fa::TX, c.x0, c.xend);
    const int ya = (int)((int64_t)a.g.ny * ch / nchunks), yb = (int)((int64_t)a.g.ny * (ch + 1) / nchunks);
    if (ya >= yb) return;
    auto par = [&](auto &&phase) {
        phase(tid);
        __syncthreads();
    };
    const bool fast = c.x0 >= 6 && c.x0 + fa::TX <= a.g.nx - 6 && c.z0 >= 6 && c.z0 + fa::TZ <= a.g.nz - 6;
    if (fast) fa_march<true>(c, ya, yb, par);
    else fa_march<false>(c, ya, yb, par);
}

// Marching elastic step over every plane (see march.cuh).  grid: (z tiles,
// x tiles, y chunks x shots), block (TZ, TX), one CTA per SM.
template <int PH, bool XF, bool ZF>
__device__ __forceinline__ void march_tile(const MarchCtx &c, int ya, int yb, int tid)
{
    m3_march<PH, XF, ZF>(c, ya, yb, [&](auto &&phase) {
        phase(tid);
        __syncthreads();
    });
}

template <int PH>
__global__ void __launch_bounds__(f3::NT, 1) k_elastic_march(const __grid_constant__ StepArgs a, int nchunks, int slab)
{
    extern __shared__ __align__(16) unsigned char m3_smem[];
    MarchCtx c;
    c.a = &a;
    c.sm = reinterpret_cast<MarchSmem *>(m3_smem);
    c.rows.p = c.sm->rows;  // filled below; first read after the first phase's barrier
    const int tid = threadIdx.x + f3::TZ * threadIdx.y;
    const int shot = blockIdx.z / nchunks;
    if (shot_idle(a, shot)) return;
    const int ch = blockIdx.z - shot * nchunks;
    c.so = shot * a.sst;
    tile_range(blockIdx.x, a.g.nz, f3::TZ, c.z0, c.zend);
    tile_range(blockIdx.y, a.g.nx, f3::TX, c.x0, c.xend);
    int ya, yb;
    if (slab > 0) {
        // the two y-wall slabs [0, slab) and [ny - slab, ny) of the fused path
        ya = ch == 0 ? 0 : a.g.ny - slab;
        yb = ch == 0 ? slab : a.g.ny;
    } else {
        m3_chunk(a.g.ny, ch, nchunks, ya, yb);
    }
    if (ya >= yb) return;
    fill_smem_rows(c.sm->rows, tid, f3::NT);
    const bool xf = m3_fast(c.x0, a.g.nx, f3::TX), zf = m3_fast(c.z0, a.g.nz, f3::TZ);
    if (xf && zf) march_tile<PH, true, true>(c, ya, yb, tid);
    else if (xf) march_tile<PH, true, false>(c, ya, yb, tid);
    else if (zf) march_tile<PH, false, true>(c, ya, yb, tid);
    else march_tile<PH, false, false>(c, ya, yb, tid);
}

// SAT penalties of the elastic faces for the planes [a.y0, a.y1) computed by
// the fused kernel: next += taper(scale(dt^2 sat / rho)), the contribution the
// reference adds to the operator sum before the update (we_op.cpp:697-804);
// update, scaling and taper are linear in it.  Each boundary point of the
// slab is enumerated once: z faces whole, x faces without z edges, y faces
// (when inside the slab) without x and z edges.
__device__ __forceinline__ bool face_point(const Dims &g, int y0, int y1, int k, int &ix, int &iy, int &iz)
{
    const int ly = y1 - y0;
    const int nzf = g.nx * ly;          // each z face
    const int nxf = (g.nz - 2) * ly;    // each x face
    const int nyf = (g.nx - 2) * (g.nz - 2);
    if (k < 2 * nzf) {
        const int side = k >= nzf;
        const int r = k - side * nzf;
        iz = side ? g.nz - 1 : 0;
        ix = r % g.nx;
        iy = y0 + r / g.nx;
        return true;
    }
    k -= 2 * nzf;
    if (k < 2 * nxf) {
        const int side = k >= nxf;
        const int r = k - side * nxf;
        ix = side ? g.nx - 1 : 0;
        iz = 1 + r % (g.nz - 2);
        iy = y0 + r / (g.nz - 2);
        return true;
    }
    k -= 2 * nxf;
    for (int side = 0; side < 2; side++) {
        const int yy = side ? g.ny - 1 : 0;
        if (yy < y0 || yy >= y1) continue;
        if (k < nyf) {
            iy = yy;
            iz = 1 + k % (g.nz - 2);
            ix = 1 + k / (g.nz - 2);
            return true;
        }
        k -= nyf;
    }
    return false;
}

// One thread per face point and shot (blockIdx.y), the three components in
// turn: a point's samples are read from memory once for the three terms.
template <int PH>
__global__ void k_elastic_face_sat(const __grid_constant__ StepArgs a, int npts)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npts) return;
    int ix, iy, iz;
    if (!face_point(a.g, a.y0, a.y1, k, ix, iy, iz) || shot_idle(a, blockIdx.y)) return;
    const int64_t so = (int64_t)blockIdx.y * a.sst;
    const int64_t i = a.g.idx(ix, iy, iz);
    float sat[3];
#pragma unroll
    for (int c = 0; c < 3; c++) sat[c] = elastic_sat<PH>(a, 0.f, c, ix, iy, iz, so);
    const float dt2r = a.dt * a.dt / a.m[2][i];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (sat[c] == 0.f) continue;
        float v = dt2r * sat[c];
        v = boundary_scale(a, v, c, ix, iy, iz);
        v = taper(a, v, ix, iy, iz);
        a.next[c][so + i] += v;
    }
}

// Face points of planes [y0, y1) (both z faces, both x faces without the z
// edges, the y faces inside the range without x and z edges) as an int grid.
static int face_points(const Problem &pb, int y0, int y1)
{
    const int64_t ly = y1 - y0;
    int64_t nf = 2 * (int64_t)pb.nx * ly + 2 * (int64_t)(pb.nz - 2) * ly;
    if (y0 == 0) nf += (int64_t)(pb.nx - 2) * (pb.nz - 2);
    if (y1 == pb.ny) nf += (int64_t)(pb.nx - 2) * (pb.nz - 2);
    if (nf >= (int64_t)INT32_MAX - 128) throw std::runtime_error("grid faces exceed the SAT kernel's index range");
    return (int)nf;
}

// Post-injection: next += taper(scale(dt^2 (w s)/rho)) (elastic) or dt^2 (w s) K
// (acoustic).  Equivalent to the reference's injection into the operator sum
// before the update (we_op.cpp:691-693): update, scaling and taper are linear in it.
__global__ void k_inject(StepArgs a, int c, const int64_t *gidx, const int *trace, const float *w, int n,
                         const float *src, int nt, int it, const int *itp, const int *t0)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (itp) it += *itp;  // replayed graphs: step offset + time index on the device
    const int64_t nxyz = a.g.nxyz();
    const int64_t gi = gidx[k];
    const int64_t sh = gi / nxyz;
    const int64_t i = gi - sh * nxyz;
    if (t0) {
        it -= t0[sh];  // shot slots: the shot's own time index
        if (it < 0 || it >= nt) return;
    }
    const float sv = w[k] * src[(int64_t)trace[k] * nt + it];
    const int iz = (int)(i % a.g.nz);
    const int ix = (int)((i / a.g.nz) % a.g.nx);
    const int iy = (int)(i / ((int64_t)a.g.nz * a.g.nx));
    const float dt2 = a.dt * a.dt;
    float v = a.m[2] ? dt2 * sv / a.m[2][i] : dt2 * sv * a.m[0][i];
    v = boundary_scale(a, v, c, ix, iy, iz);
    v = taper(a, v, ix, iy, iz);
    atomicAdd(&a.next[c][sh * a.sst + i], v);
}

// Initial condition prev = inject(src[:,0]) then scaled (we_op.cpp:611-619, 1635-1636).
__global__ void k_inject0(float *prev, int64_t sst, int64_t nxyz, const int64_t *gidx, const int *trace,
                          const float *w, int n, const float *src, int nt, int only)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t gi = gidx[k];
    const int64_t sh = gi / nxyz;
    if (only >= 0 && sh != only) return;
    atomicAdd(&prev[sh * sst + (gi - sh * nxyz)], w[k] * src[(int64_t)trace[k] * nt]);
}

__global__ void k_scale0(float *prev, int64_t sst, const float *coef, int64_t n, int nshots, float dt, int acoustic,
                         int only)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int s = only >= 0 ? only : 0; s < (only >= 0 ? only + 1 : nshots); s++) {
        float *p = prev + s * sst + i;
        const float v = *p;
        if (v == 0.f) continue;
        if (acoustic) *p = (float)((double)v * (0.5 * (double)coef[i] * dt * dt));
        else *p = (float)((double)v * (0.5 * dt * dt / (double)coef[i]));
    }
}

// Receivers: rcv[s][c][r][it] = sum_k w_k u_c(g_k) (injector.cpp:118-140).
__global__ void k_extract(const float *u, int64_t sst, int64_t nxyz, int ncomp, const int64_t *gidx, const float *w,
                          int nrec, int nr, float *rcv, int nt, int it, int ntap, const int *itp, const int *t0)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (row >= nrec) return;
    if (itp) it += *itp;
    const int sh = row / nr, r = row - sh * nr;
    if (t0) {
        it -= t0[sh];  // shot slots: the shot's own time index
        if (it < 0 || it >= nt) return;
    }
    const float *uc = u + sh * sst + c * nxyz;
    const int64_t b = (int64_t)ntap * row;
    float acc = 0.f;
    if (ntap == 27) {
#pragma unroll
        for (int k = 0; k < 27; k++) acc += w[b + k] * uc[gidx[b + k] - (int64_t)sh * nxyz];
    } else {
        // dipole rows: taps in (end b, end a) pairs; each pair's difference is
        // formed, rounded, then accumulated, without contraction, as
        // dipole_m3::extract does (injector.cpp:487-489): the two ends nearly
        // cancel, so the rounding order matters
        for (int k = 0; k < ntap; k += 2) {
            const float pb = __fmul_rn(w[b + k], uc[gidx[b + k] - (int64_t)sh * nxyz]);
            const float pa = __fmul_rn(w[b + k + 1], uc[gidx[b + k + 1] - (int64_t)sh * nxyz]);
            acc = __fadd_rn(acc, __fadd_rn(pb, pa));
        }
    }
    rcv[(((int64_t)sh * ncomp + c) * nr + r) * nt + it] = acc;
}

// D2var closure weights of mu for the 12 closure rows of every line along one
// axis (StepArgs::w2c): the fused and marching kernels' d2closure_weights,
// evaluated once per model instead of at every time step.
// Coefficient f of the closure weights along a line: 0 mu, 1 c66, 2 c11b.
struct W2cCoef {
    Line mu, eps, c66;
    int f;
    FWI_HD float operator()(int k) const
    {
        if (f == 0) return mu(k);
        if (f == 1) return c66(k);
        return 2.f * (1.f + 2.f * eps(k)) * mu(k);  // as C11bS / C11bLine
    }
};

__global__ void k_w2c(StepArgs a, int axis, int f, float *out, int64_t nlines)
{
    const Dims &g = a.g;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlines * 12) return;
    const int64_t line = e / 12;
    const int slot = (int)(e - line * 12);
    int64_t base, stride;
    int n;
    if (axis == 0) {
        const int64_t y = line / g.nz, z = line - y * g.nz;
        base = y * g.nx * g.nz + z;
        stride = g.nz;
        n = g.nx;
    } else if (axis == 1) {
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
    const W2cCoef l{Line{a.m[1], base, stride}, Line{f == 2 ? a.m[4] : a.m[1], base, stride},
                    Line{f == 1 ? a.m[5] : a.m[1], base, stride}, f};
    const int i = slot < 6 ? slot : n - 1 - (slot - 6);
    const W8 w = d2closure_weights(l, i, n, ConstRows());
    for (int j = 0; j < 8; j++) out[e * 8 + j] = w.w[j];
}

// Time index of replayed graphs: set once before the replays, advanced by
// one thread at the end of each replayed block of three steps (whose kernels
// add their step's offset 0, 1, 2).
__global__ void k_set_it(int *itp, int it) { *itp = it; }
__global__ void k_tick(int *itp, int by) { *itp += by; }

// Imaging of every shot of a batch at once: the increments of the shots
// (fields at offsets s * sst) are summed in FP64 per point, then added to the
// gradient once.
// Point k of the 4-point shell of the grid (every point within 4 of a face):
// the z rows 0..3 and nz-4..nz-1 whole, then the x rows 0..3 and nx-4..nx-1
// of the other z rows, then the y planes 0..3 and ny-4..ny-1 of the rest.
__device__ __forceinline__ bool shell_point(const Dims &g, int64_t k, int &ix, int &iy, int &iz)
{
    const int64_t nzs = (int64_t)8 * g.nx * g.ny;  // z rows of the shell
    if (k < nzs) {
        const int r = (int)(k % 8);
        iz = r < 4 ? r : g.nz - 8 + r;
        const int64_t q = k / 8;
        ix = (int)(q % g.nx);
        iy = (int)(q / g.nx);
        return true;
    }
    k -= nzs;
    const int mz = g.nz - 8;
    const int64_t nxs = (int64_t)8 * mz * g.ny;
    if (k < nxs) {
        iz = 4 + (int)(k % mz);
        const int64_t q = k / mz;
        const int r = (int)(q % 8);
        ix = r < 4 ? r : g.nx - 8 + r;
        iy = (int)(q / 8);
        return true;
    }
    k -= nxs;
    const int mx = g.nx - 8;
    if (k < (int64_t)8 * mz * mx) {
        iz = 4 + (int)(k % mz);
        const int64_t q = k / mz;
        ix = 4 + (int)(q % mx);
        const int r = (int)(q / mx);
        iy = r < 4 ? r : g.ny - 8 + r;
        return true;
    }
    return false;
}

// gst > 0: one gradient per shot, shot s's at offset s * gst (its increments
// are not summed with the other shots').  The box launch is held to 64
// registers (isotropic; 80 for VTI) for 4 (3) resident blocks per SM: its
// loads are latency-bound (a 400-step 200^3 x 4 adjoint 2.37 -> 2.26 s).
// PART 0: every point; 1: the box of
// points at least 4 from every face, whose derivatives are interior rows
// only, so no warp diverges into the closure rows (z rows selected in place,
// which keeps the lanes' 128-byte alignment); 2: the 4-point shell, one
// thread per shell point (shell_point, 1-D grid).
template <int PH, int PART = 0>
__global__ void __launch_bounds__(BZ * BX * BY, PART == 1 ? (PH == VTI ? 3 : 4) : 1)
    k_image_batch(ImageArgs a, int nshots, int64_t sst, int64_t gst)
{
    int ix, iy, iz, s;
    if (PART == 1) {
        const Dims b{a.g.nx - 8, a.g.ny - 8, a.g.nz};
        if (!point_of(b, (b.ny + BY - 1) / BY, ix, iy, iz, s) || iz < 4 || iz >= a.g.nz - 4) return;
        ix += 4;
        iy += 4;
    } else if (PART == 2) {
        if (!shell_point(a.g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ix, iy, iz)) return;
    } else if (!point_of(a.g, (a.g.ny + BY - 1) / BY, ix, iy, iz, s)) {
        return;
    }
    const int64_t i = a.g.idx(ix, iy, iz);
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    const bool in = PART == 1 || (PART == 0 && ix >= 4 && ix < a.g.nx - 4 && iy >= 4 && iy < a.g.ny - 4 &&
                                  iz >= 4 && iz < a.g.nz - 4);
    for (int sh = 0; sh < nshots; sh++) {
        if (PH == ACOUSTIC) {
            double k, b;
            acoustic_image_inc(a, sh * sst, ix, iy, iz, k, b);
            g0 -= k;
            g1 += b;
        } else {
            double i0, i1, i2;
            if (in) elastic_image_inc<PH, true>(a, sh * sst, ix, iy, iz, i0, i1, i2);
            else elastic_image_inc<PH, false>(a, sh * sst, ix, iy, iz, i0, i1, i2);
            g0 += i0;
            g1 += i1;
            g2 += i2;
        }
        if (gst) {
            const int64_t o = sh * gst + i;
            a.grad[0][o] += g0;
            a.grad[1][o] += g1;
            if (PH != ACOUSTIC) a.grad[2][o] += g2;
            g0 = g1 = g2 = 0.0;
        }
    }
    if (gst) return;
    a.grad[0][i] += g0;
    a.grad[1][i] += g1;
    if (PH != ACOUSTIC) a.grad[2][i] += g2;
}

__global__ void k_d2f(const double *in, float *out, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link against the driver library); null when unavailable.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor map of the three displacement components of every shot at one time
// level (base = component 0 of shot 0), as FusedTma describes.  Needs the
// 16-byte strides of nz % 4 == 0 and a 16-byte aligned base.
static bool encode_level_map(CUtensorMap *m, const float *base, const Problem &pb)
{
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || pb.nz % 4 != 0 || ((uintptr_t)base & 15) != 0) return false;
    const cuuint64_t n = (cuuint64_t)pb.nxyz();
    const cuuint64_t dims[5] = {(cuuint64_t)pb.nz, (cuuint64_t)pb.nx, (cuuint64_t)pb.ny, 3, (cuuint64_t)pb.nshots};
    const cuuint64_t strides[4] = {(cuuint64_t)pb.nz * 4, (cuuint64_t)pb.nx * pb.nz * 4, n * 4, 3 * n * 4};
    const cuuint32_t box[5] = {fz::ZW, fz::XW, 1, 3, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<float *>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

Engine::Engine(int device, const Problem &pb) : device_(device), pb_(pb)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw FwiError(FWI_ERR_NOGPU, "no CUDA device");
    if (device < 0 || device >= ndev) throw FwiError(FWI_ERR_ARG, "device index out of range");
    CK(cudaSetDevice(device));
    if (pb.nx < 12 || pb.ny < 12 || pb.nz < 12)
        throw FwiError(FWI_ERR_ARG, "each grid axis needs at least 12 points (two 6-row SBP closures)");
    if (pb.nshots < 1) throw FwiError(FWI_ERR_ARG, "at least one shot");
    init_sbp_tables();
    CK(cudaMemcpyToSymbol(c_sbp, &g_sbp_host, sizeof(SbpTables)));
    // the y chunking of the marching kernels aims at whole waves of resident CTAs
    CK(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device));
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    stream_ = s;
    const char *isp = std::getenv("FWI_IMAGE_SPLIT");
    image_split_ = !(isp && isp[0] == '0');
    const char *cc = std::getenv("FWI_CONCURRENT");
    conc_ = !(cc && cc[0] == '0');
    if (conc_) {
        cudaStream_t s2;
        cudaEvent_t e0, e1;
        // the side stream (edge tiles, y-wall slabs: the longest CTAs of a
        // step) at the device's highest priority, so that its blocks are
        // dispatched ahead of the interior tiles' (FWI_SIDE_PRIORITY=0: default priority)
        const char *sp = std::getenv("FWI_SIDE_PRIORITY");
        if (!(sp && sp[0] == '0')) {
            int lo = 0, hi = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            CK(cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, hi));
        } else {
            CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        }
        side_ = s2;
        CK(cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
        ev_fork_ = e0;
        CK(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
        ev_join_ = e1;
    }
    const int64_t n = pb.nxyz();
    const int nc = pb.ncomp();
    fields_.alloc(sizeof(float) * 3 * (size_t)pb.nshots * nc * n);
    // Marching kernel over all planes (FWI_MARCH=1, where its tiling applies);
    // otherwise the interior fused kernel plus per-point kernels at the y walls.
    const char *menv = std::getenv("FWI_MARCH");
    march_ = pb.nmodels != 2 && (menv && menv[0] == '1') && pb.nx >= f3::TX + 6 && pb.nz >= f3::TZ + 6 &&
             pb.ny >= 12;
    {
        const char *fe = std::getenv("FWI_FUSED");
        const char *se = std::getenv("FWI_SLAB_MARCH");
        const bool fused = !march_ && pb.nmodels != 2 && !(fe && fe[0] == '0') && pb.nx >= fz::TX + 6 &&
                           pb.nz >= fz::TZ + 6 && pb.ny > 2 * fz::YPAD;
        slab_march_ = fused && !(se && se[0] == '0');
    }
    if (pb.nmodels != 2 && !march_ && !slab_march_)
        aux_.alloc(sizeof(float) * (size_t)pb.nshots * (pb.nmodels == 6 ? 9 : 7) * n);
    if (march_ || slab_march_) {
        CK(cudaFuncSetAttribute(k_elastic_march<ELASTIC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(MarchSmem)));
        CK(cudaFuncSetAttribute(k_elastic_march<VTI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(MarchSmem)));
    }
    {
        const char *ae = std::getenv("FWI_FUSED");
        // the marching kernel pays off once every CTA has enough planes to march
        // over (measured: 1.5x the per-point kernel at 256^3, 0.8x at 101^3)
        afused_ = pb.nmodels == 2 && !(ae && ae[0] == '0') && pb.nx >= fa::TX + 6 && pb.nz >= fa::TZ + 6 &&
                  pb.ny >= 12 && (pb.nxyz() * pb.nshots >= (int64_t)4 << 20 || (ae && ae[0] == '1'));
    }
    const char *env = std::getenv("FWI_FUSED");
    // The tiling keeps every SBP closure row in the first or the last tile only
    // when each axis is at least one tile plus the 6 closure rows long.
    fused_ = !march_ && pb.nmodels != 2 && !(env && env[0] == '0') && pb.nx >= fz::TX + 6 && pb.nz >= fz::TZ + 6 &&
             pb.ny > 2 * fz::YPAD;
    // Occupancy variant of the fused kernel: 2 CTAs per SM with 64 registers
    // (default, the faster on B200) or 1 CTA per SM with up to 128 registers.
    const char *mb = std::getenv("FWI_FUSED_MINB");
    fused_minb_ = (mb && mb[0] == '1') ? 1 : 2;
    // modeling runs replay CUDA graphs of three steps (FWI_GRAPHS=0: plain launches)
    const char *ge = std::getenv("FWI_GRAPHS");
    graphs_ = !(ge && ge[0] == '0');
    // isotropic media: interior and edge tiles in two launches (FWI_FUSED_SPLIT=0: one)
    // y chunks per tile column: about FWI_FUSED_WAVES waves of resident CTAs
    // (measured at 256^3 x 8: 1 12.88, 2 11.05, 4 10.11, 8 9.85, 16 9.84 ms per step)
    const char *fw = std::getenv("FWI_FUSED_WAVES");
    fused_waves_ = fw ? std::max(1, std::atoi(fw)) : 8;
    // the paired kernel's launches aim at about four waves: with the edge
    // tiles and slabs on a second stream beside the interior tiles, longer y
    // chunks (less prologue per plane) beat shorter tails (256^3 x 8: 5.95 ms
    // per step at 4 waves, 6.08 at 8, 6.24 at 16)
    // edge-tile modes on the second stream (FWI_SIDE_MODES, digits of 3..5):
    // the z-face and corner tiles beside the slabs, the x-face tiles after
    // the interior tiles balance the two streams best (256^3 x 8: 5.84 ms per
    // step; all three on the second stream 5.93, mode 4 alone 5.89)
    const char *smo = std::getenv("FWI_SIDE_MODES");
    side_modes_ = 0;
    for (const char *c = smo ? smo : "45"; *c; c++)
        if (*c >= '3' && *c <= '5') side_modes_ |= 1 << (*c - '0');
    // the y-wall slabs (one CTA per SM) after the second stream's edge tiles
    // (256^3 x 8: 5.79 against 5.84 ms per step first)
    const char *sl = std::getenv("FWI_SLABS_LAST");
    slabs_last_ = !(sl && sl[0] == '0');
    const char *pw = std::getenv("FWI_PAIR_WAVES");
    pair_waves_ = pw ? std::max(1, std::atoi(pw)) : 4;
    // isotropic interior tiles: two z-adjacent points per thread in packed
    // FP32 pairs (FWI_PAIR=0: one point per thread)
    const char *pe = std::getenv("FWI_PAIR");
    pair_ = !(pe && pe[0] == '0');
    // its edge tiles (FWI_PAIR_EDGE): 0 all by the one-point kernel, 1 those
    // touching an x face only by the paired kernel, 2 all by the paired kernel
    const char *pee = std::getenv("FWI_PAIR_EDGE");
    pair_edge_ = pee ? std::max(0, std::min(2, std::atoi(pee))) : 2;
    const char *sp = std::getenv("FWI_FUSED_SPLIT");
    fused_split_ = !(sp && sp[0] == '0');
    // plane copies of the fused kernel by the tensor memory accelerator
    // (FWI_TMA=0: per-thread asynchronous copies instead)
    const char *te = std::getenv("FWI_TMA");
    tma_ = fused_ && pb.nmodels != 2 && pb.nz % 4 == 0 && !(te && te[0] == '0') && tensor_map_encoder() != nullptr;
    if (fused_) {
        tma_err_.alloc(sizeof(int));
        tma_err_.zero(stream_);
        CK(cudaFuncSetAttribute(k_elastic_fused<ELASTIC, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(FusedSmem)));
        CK(cudaFuncSetAttribute(k_elastic_fused<VTI, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(FusedSmem)));
        CK(cudaFuncSetAttribute(k_elastic_fused<ELASTIC, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(FusedSmem)));
        CK(cudaFuncSetAttribute(k_elastic_fused<VTI, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(FusedSmem)));
        CK(cudaFuncSetAttribute(k_elastic_fused_part<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(FusedSmem)));
        CK(cudaFuncSetAttribute(k_elastic_fused_part<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(FusedSmem)));
        CK(pair_init());
    }
}

Engine::~Engine()
{
    drop_graph();
    if (stream_) {
        cudaStreamSynchronize((cudaStream_t)stream_);
        cudaStreamDestroy((cudaStream_t)stream_);
    }
    if (side_) {
        cudaStreamSynchronize((cudaStream_t)side_);
        cudaStreamDestroy((cudaStream_t)side_);
    }
    if (ev_fork_) cudaEventDestroy((cudaEvent_t)ev_fork_);
    if (ev_join_) cudaEventDestroy((cudaEvent_t)ev_join_);
    for (void *e : kev_) cudaEventDestroy((cudaEvent_t)e);
}

void Engine::sync()
{
    CK(cudaStreamSynchronize((cudaStream_t)stream_));
    if (tma_) {
        int e = 0;
        CK(cudaMemcpy(&e, tma_err_.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            CK(cudaMemset(tma_err_.p, 0, sizeof(int)));
            throw FwiError(FWI_ERR_CUDA, "fused kernel: a plane copy did not complete within its wait limit");
        }
    }
}

int64_t Engine::device_bytes() const
{
    return model_.bytes + w2c_.bytes + fields_.bytes + aux_.bytes + snaps_.bytes + grad_.bytes + sdiv_.bytes + taper_.bytes +
           src_dev_.bytes + rcv_dev_.bytes + snapq_.bytes + snaps_scale_.bytes + enc_.bytes + amax_.bytes +
           snapz_.bytes + rv_store_.bytes + rv_scale_.bytes + rec_fields_.bytes + grad_f32_.bytes + adj_src_buf_.bytes +
           das_w_.bytes + das_rcv_.bytes + das_src_.bytes;
}

float *Engine::level(int l) const
{
    const int64_t lv = (int64_t)pb_.nshots * pb_.ncomp() * pb_.nxyz();
    return fields_.as<float>() + ((rot_ + l) % 3) * lv;
}

void Engine::set_model(const float *conv)
{
    CK(cudaSetDevice(device_));
    const int64_t n = pb_.nxyz();
    model_.alloc(sizeof(float) * pb_.nmodels * n);
    CK(cudaMemcpyAsync(model_.p, conv, model_.bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream_));
    // closure weights of the D2var coefficients along x, y, z, once per model
    // (FWI_W2C=0: formed in the step kernels): mu on every axis, and for VTI
    // also c66 and c11b along x and y
    const char *we = std::getenv("FWI_W2C");
    for (int ax = 0; ax < 3; ax++)
        for (int f = 0; f < 3; f++) w2c_ptr_[ax][f] = nullptr;
    if (pb_.nmodels != 2 && (fused_ || march_) && !(we && we[0] == '0')) {
        const int64_t nl[3] = {(int64_t)pb_.ny * pb_.nz, (int64_t)pb_.nx * pb_.nz, (int64_t)pb_.ny * pb_.nx};
        const int nf[3] = {pb_.nmodels == 6 ? 3 : 1, pb_.nmodels == 6 ? 3 : 1, 1};
        int64_t tot = 0;
        for (int ax = 0; ax < 3; ax++) tot += nf[ax] * nl[ax];
        w2c_.alloc(sizeof(float) * 12 * 8 * tot);
        float *o = w2c_.as<float>();
        StepArgs ma;
        std::memset(&ma, 0, sizeof(ma));
        ma.g = Dims{pb_.nx, pb_.ny, pb_.nz};
        for (int k = 0; k < pb_.nmodels; k++) ma.m[k] = model_.as<float>() + k * n;
        for (int ax = 0; ax < 3; ax++)
            for (int f = 0; f < nf[ax]; f++) {
                w2c_ptr_[ax][f] = o;
                k_w2c<<<(unsigned)((nl[ax] * 12 + 255) / 256), 256, 0, (cudaStream_t)stream_>>>(ma, ax, f, o, nl[ax]);
                o += 12 * 8 * nl[ax];
            }
        CK(cudaGetLastError());
    } else {
        w2c_.alloc(0);
    }

    ScaleTables st = boundary_divisors(conv, pb_.nmodels, pb_.nx, pb_.ny, pb_.nz, pb_.dx, pb_.dy, pb_.dz, pb_.dt, pb_.bc);
    scale_ = 0;
    for (int f = 0; f < 6; f++) scale_ |= (pb_.bc[f] == BC_ABSORB);
    size_t tot = 0;
    const int nc = pb_.ncomp();
    for (int f = 0; f < 6; f++)
        for (int c = 0; c < nc; c++) tot += st.f[f][c].size();
    std::vector<float> packed(tot);
    size_t off[6][3] = {};
    size_t o = 0;
    for (int f = 0; f < 6; f++)
        for (int c = 0; c < nc; c++) {
            off[f][c] = o;
            std::memcpy(packed.data() + o, st.f[f][c].data(), sizeof(float) * st.f[f][c].size());
            o += st.f[f][c].size();
        }
    sdiv_.alloc(sizeof(float) * tot);
    CK(cudaMemcpy(sdiv_.p, packed.data(), sdiv_.bytes, cudaMemcpyHostToDevice));
    for (int f = 0; f < 6; f++)
        for (int c = 0; c < 3; c++) sdiv_ptr_[f][c] = sdiv_.as<float>() + off[f][c < nc ? c : 0];

    TaperTables tt = taper_tables(pb_.nx, pb_.ny, pb_.nz, pb_.taper, pb_.taper_strength);
    size_t ttot = 0;
    for (int k = 0; k < 6; k++) ttot += tt.t[k].size();
    std::vector<float> tp(ttot);
    size_t toff[6];
    o = 0;
    for (int k = 0; k < 6; k++) {
        toff[k] = o;
        std::memcpy(tp.data() + o, tt.t[k].data(), sizeof(float) * tt.t[k].size());
        o += tt.t[k].size();
    }
    taper_.alloc(sizeof(float) * ttot);
    CK(cudaMemcpy(taper_.p, tp.data(), taper_.bytes, cudaMemcpyHostToDevice));
    for (int k = 0; k < 6; k++) taper_ptr_[k] = taper_.as<float>() + toff[k];
    sync();
}

void Engine::upload_inj(const InjTable &t, int ntrace, DevInj &d)
{
    d.ntrace = ntrace;
    for (int c = 0; c < 3; c++) {
        d.n[c] = (int)t.gidx[c].size();
        d.gidx[c].alloc(sizeof(int64_t) * d.n[c]);
        d.trace[c].alloc(sizeof(int) * d.n[c]);
        d.w[c].alloc(sizeof(float) * d.n[c]);
        if (d.n[c]) {
            CK(cudaMemcpy(d.gidx[c].p, t.gidx[c].data(), d.gidx[c].bytes, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(d.trace[c].p, t.trace[c].data(), d.trace[c].bytes, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(d.w[c].p, t.w[c].data(), d.w[c].bytes, cudaMemcpyHostToDevice));
        }
    }
}

namespace {
StepArgs make_step_args(const Problem &pb, const float *m, const float *const sdiv[6][3], const float *const tap[6],
                        int scale)
{
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = Dims{pb.nx, pb.ny, pb.nz};
    a.dx = pb.dx;
    a.dy = pb.dy;
    a.dz = pb.dz;
    a.dt = pb.dt;
    a.idx = 1.0f / pb.dx;
    a.idy = 1.0f / pb.dy;
    a.idz = 1.0f / pb.dz;
    const float d[3] = {pb.dx, pb.dy, pb.dz};
    for (int k = 0; k < 3; k++) {
        a.ad1[k] = 1.0f / (d[k] * d[k]);
        a.ad2[k] = 2.0f / (d[k] * d[k]);
    }
    const int64_t n = pb.nxyz();
    for (int k = 0; k < pb.nmodels; k++) a.m[k] = m + k * n;
    for (int f = 0; f < 6; f++) {
        a.bc[f] = pb.bc[f];
        a.tap[f] = tap[f];
        a.tw[f] = std::max(0, pb.taper[f]);
        for (int c = 0; c < 3; c++) a.sdiv[f][c] = sdiv[f][c];
    }
    a.scale = scale;
    a.alpha_fs = (float)(0.2508560249 / pb.free_surface_stiffness);
    a.nyb = yblocks(a.g);
    a.y0 = 0;
    a.y1 = pb.ny;
    a.sst = (int64_t)pb.ncomp() * n;
    a.ast = (int64_t)(pb.nmodels == 6 ? 9 : 7) * n;
    return a;
}
}  // namespace

void Engine::init_prev(const DevInj &inj, const float *src_dev, float *prev, int only_shot)
{
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nc = pb_.ncomp();
    const int64_t sst = (int64_t)nc * n;
    for (int c = 0; c < nc; c++) {
        if (inj.n[c] == 0) continue;
        k_inject0<<<(inj.n[c] + 255) / 256, 256, 0, s>>>(prev + c * n, sst, n, inj.gidx[c].as<int64_t>(),
                                                          inj.trace[c].as<int>(), inj.w[c].as<float>(), inj.n[c],
                                                          src_dev, pb_.nt, only_shot);
        const float *coef = model_.as<float>() + (pb_.nmodels == 2 ? 0 : 2 * n);
        k_scale0<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(prev + c * n, sst, coef, n, pb_.nshots, pb_.dt,
                                                               pb_.nmodels == 2, only_shot);
    }
    CK(cudaGetLastError());
}

void Engine::step(float *prev, float *curr, float *next, bool taper_prev)
{
    cudaStream_t s = (cudaStream_t)stream_;
    const Dims g{pb_.nx, pb_.ny, pb_.nz};
    const int64_t n = pb_.nxyz();
    StepArgs a = make_step_args(pb_, model_.as<float>(), sdiv_ptr_, taper_ptr_, scale_);
    const int nc = pb_.ncomp();
    for (int c = 0; c < nc; c++) {
        a.curr[c] = curr + c * n;
        a.prev[c] = prev + c * n;
        a.next[c] = next + c * n;
    }
    for (int ax = 0; ax < 3; ax++)
        for (int f = 0; f < 3; f++) a.w2c[ax][f] = w2c_ptr_[ax][f];
    a.taper_prev = taper_prev ? 1 : 0;
    a.active = continuous_ ? shot_active_.as<int>() : nullptr;
    const dim3 blk(BZ, BX, BY);
    // per-point launch over planes [y0, y1)
    auto range = [&](StepArgs &st, int y0, int y1) {
        st.y0 = y0;
        st.y1 = y1;
        st.nyb = yblocks(y1 - y0);
        return grid_of(g, pb_.nshots, y1 - y0);
    };
    if (pb_.nmodels == 2) {
        if (afused_) {
            const int kz = (pb_.nz + fa::TZ - 1) / fa::TZ, kx = (pb_.nx + fa::TX - 1) / fa::TX;
            const int tiles = kz * kx * pb_.nshots;
            int nch = (sm_count_ * 2 * 4 + tiles - 1) / tiles;  // about four waves of resident CTAs
            nch = std::max(1, std::min(nch, pb_.ny / 8));
            kmark(true, "k_acoustic_fused", n * pb_.nshots);
            k_acoustic_fused<<<dim3(kz, kx, nch * pb_.nshots), dim3(fa::TZ, fa::TX), 0, s>>>(a, nch);
            kmark(false, nullptr, 0);
        } else {
            const dim3 grd = range(a, 0, pb_.ny);
            kmark(true, "k_acoustic_step", n * pb_.nshots);
            k_acoustic_step<<<grd, blk, 0, s>>>(a);
            kmark(false, nullptr, 0);
        }
        CK(cudaGetLastError());
        return;
    }
    if (march_) {
        const int kz = (pb_.nz + f3::TZ - 1) / f3::TZ, kx = (pb_.nx + f3::TX - 1) / f3::TX;
        const int tiles = kz * kx * pb_.nshots;
        const int target = sm_count_ * 3;  // about three waves of resident CTAs
        int nch = (target + tiles - 1) / tiles;
        nch = std::max(1, std::min(nch, (pb_.ny - 12) / 24));
        const dim3 grd(kz, kx, nch * pb_.nshots), mblk(f3::TZ, f3::TX);
        kmark(true, "k_elastic_march", n * pb_.nshots);
        if (pb_.nmodels == 3) k_elastic_march<ELASTIC><<<grd, mblk, sizeof(MarchSmem), s>>>(a, nch, 0);
        else k_elastic_march<VTI><<<grd, mblk, sizeof(MarchSmem), s>>>(a, nch, 0);
        kmark(false, nullptr, 0);
        // SAT of every face point
        StepArgs f = a;
        f.y0 = 0;
        f.y1 = pb_.ny;
        const int nf = face_points(pb_, f.y0, f.y1);
        const dim3 sgrd((unsigned)((nf + 127) / 128), pb_.nshots);
        if (pb_.nmodels == 3) k_elastic_face_sat<ELASTIC><<<sgrd, 128, 0, s>>>(f, nf);
        else k_elastic_face_sat<VTI><<<sgrd, 128, 0, s>>>(f, nf);
        CK(cudaGetLastError());
        return;
    }
    AuxArgs x;
    std::memset(&x, 0, sizeof(x));
    x.g = g;
    x.dx = pb_.dx;
    x.dy = pb_.dy;
    x.dz = pb_.dz;
    x.sst = a.sst;
    x.ast = a.ast;
    for (int k = 0; k < pb_.nmodels; k++) x.m[k] = a.m[k];
    for (int c = 0; c < 3; c++) x.curr[c] = curr + c * n;
    float *ab = aux_.as<float>();
    if (pb_.nmodels == 3) {
        // one shared divergence array in slots 0..2, then the six derivatives
        x.aux[AUX_T0] = x.aux[AUX_T1] = x.aux[AUX_T2] = ab;
        for (int k = 3; k < 9; k++) x.aux[k] = ab + (k - 2) * n;
    } else {
        for (int k = 0; k < 9; k++) x.aux[k] = ab + k * n;
    }
    for (int k = 0; k < 9; k++) a.aux[k] = x.aux[k];
    auto aux_range = [&](int y0, int y1) {
        x.y0 = y0;
        x.y1 = y1;
        x.nyb = yblocks(y1 - y0);
        const dim3 grd = grid_of(g, pb_.nshots, y1 - y0);
        if (pb_.nmodels == 3) k_elastic_aux<ELASTIC><<<grd, blk, 0, s>>>(x);
        else k_elastic_aux<VTI><<<grd, blk, 0, s>>>(x);
    };
    auto step_range = [&](int y0, int y1) {
        const dim3 grd = range(a, y0, y1);
        if (pb_.nmodels == 3) k_elastic_step<ELASTIC><<<grd, blk, 0, s>>>(a);
        else k_elastic_step<VTI><<<grd, blk, 0, s>>>(a);
    };
    const int P = fz::YPAD;
    if (!fused_) {
        aux_range(0, pb_.ny);
        kmark(true, "k_elastic_step", n * pb_.nshots);
        step_range(0, pb_.ny);
        kmark(false, nullptr, 0);
    } else {
        // With a second stream the y-wall slabs and the paired kernel's edge
        // tiles run on it beside the interior tiles (they write disjoint
        // points of next); the SAT, which adds to face points of all of them,
        // follows the join.  The main-kernel timing keeps one stream.
        const bool conc = side_ && slab_march_ && pb_.nmodels == 3 && pair_ && pair_edge_ == 2 && !ktime_;
        cudaStream_t se = s;
        if (conc) {
            se = (cudaStream_t)side_;
            CK(cudaEventRecord((cudaEvent_t)ev_fork_, s));
            CK(cudaStreamWaitEvent(se, (cudaEvent_t)ev_fork_, 0));
        }
        // planes near the y walls: the marching kernel (y closures), two chunks per tile column
        auto slabs = [&]() {
            const int kz3 = (pb_.nz + f3::TZ - 1) / f3::TZ, kx3 = (pb_.nx + f3::TX - 1) / f3::TX;
            const dim3 grd3(kz3, kx3, 2 * pb_.nshots), mblk(f3::TZ, f3::TX);
            if (pb_.nmodels == 3) k_elastic_march<ELASTIC><<<grd3, mblk, sizeof(MarchSmem), se>>>(a, 2, P);
            else k_elastic_march<VTI><<<grd3, mblk, sizeof(MarchSmem), se>>>(a, 2, P);
        };
        const bool slabs_last = conc && slabs_last_;
        if (slab_march_) {
            if (!slabs_last) slabs();
        } else {
            // planes near the y walls: per-point kernels (derivative scratch two planes deeper)
            if (pb_.ny < 2 * (P + 2)) {
                aux_range(0, pb_.ny);
            } else {
                aux_range(0, P + 2);
                aux_range(pb_.ny - P - 2, pb_.ny);
            }
            step_range(0, P);
            step_range(pb_.ny - P, pb_.ny);
        }
        // interior planes: fused kernel
        StepArgs f = a;
        f.y0 = P;
        f.y1 = pb_.ny - P;
        for (int k = 0; k < 9; k++) f.aux[k] = nullptr;
        const int kz = (pb_.nz + fz::TZ - 1) / fz::TZ, kx = (pb_.nx + fz::TX - 1) / fz::TX;
        FusedTma tm;
        std::memset(&tm, 0, sizeof(tm));
        tm.err = tma_err_.as<int>();
        tm.on = tma_ && encode_level_map(&tm.u, curr, pb_) ? 1 : 0;
        const dim3 fblk(fz::TZ, fz::TX);
        const size_t sm = sizeof(FusedSmem);
        // y chunks per tile column: about fused_waves_ waves of resident CTAs,
        // at least 16 planes per chunk
        auto chunks = [&](int64_t tiles, int minb, int waves = 0) {
            const int64_t target = (int64_t)sm_count_ * minb * (waves > 0 ? waves : fused_waves_);
            const int64_t c = (target + tiles - 1) / tiles;
            return (int)std::max<int64_t>(1, std::min<int64_t>(c, (f.y1 - f.y0) / 16));
        };
        // interior tiles form the index box [zl, zh) x [xl, xh)
        int zl, zh, xl, xh;
        fz_interior_range(pb_.nz, fz::TZ, zl, zh);
        fz_interior_range(pb_.nx, fz::TX, xl, xh);
        const bool el = pb_.nmodels == 3;
        const bool split = fused_split_active();
        kmark(true, el && pair_ ? "k_elastic_pair" : "k_elastic_fused",
              (int64_t)(f.y1 - f.y0) * pb_.nx * pb_.nz * pb_.nshots);
        if (el && pair_) {
            // paired kernel: edge tiles (all of them when no tile is interior), then interior tiles
            const int64_t ti = (int64_t)(zh - zl) * (xh - xl) * pb_.nshots;
            const int64_t te = (int64_t)kz * kx * pb_.nshots - ti;
            const int ne = chunks(te, 2, pair_waves_), ni = chunks(std::max<int64_t>(ti, 1), 2, pair_waves_);
            const bool even = pb_.nz % 2 == 0;
            // tiles touching an x face only (mode 3), a z face only (4), both (5): y chunks per launch;
            // the modes of side_modes_ on the second stream, the others after the interior tiles
            const int64_t nzi = zh - zl, nxi = xh - xl;
            const int64_t tiles[3] = {(kx - nxi) * nzi, nxi * (kz - nzi), (kx - nxi) * (kz - nzi)};
            auto edges = [&](bool side, cudaStream_t st) {
                for (int mode = 3; mode <= 5; mode++) {
                    if (tiles[mode - 3] == 0 || (((side_modes_ >> mode) & 1) != 0) != side) continue;
                    const int nm = chunks(tiles[mode - 3] * pb_.nshots, 2, pair_waves_);
                    pair_launch(even, mode, dim3(kz, kx, nm * pb_.nshots), sm, st, f, nm, tm, 0, 0);
                }
            };
            if (te > 0 && pair_edge_ == 2) {
                edges(true, se);
            } else if (te > 0) {
                // tiles with a z face: the one-point-per-thread kernel; with x faces only: the paired one
                k_elastic_fused_part<2><<<dim3(kz, kx, ne * pb_.nshots), fblk, sm, s>>>(f, ne, tm, pair_edge_, 0);
                if (pair_edge_ == 1) pair_launch(even, 3, dim3(kz, kx, ne * pb_.nshots), sm, s, f, ne, tm, 0, 0);
            }
            if (slabs_last) slabs();
            if (ti > 0) pair_launch(even, 1, dim3(zh - zl, xh - xl, ni * pb_.nshots), sm, s, f, ni, tm, zl, xl);
            if (te > 0 && pair_edge_ == 2) edges(false, s);
            if (conc) {
                CK(cudaEventRecord((cudaEvent_t)ev_join_, se));
                CK(cudaStreamWaitEvent(s, (cudaEvent_t)ev_join_, 0));
            }
        } else if (split) {
            const int64_t ti = (int64_t)(zh - zl) * (xh - xl) * pb_.nshots;
            const int64_t te = (int64_t)kz * kx * pb_.nshots - ti;
            const int ne = chunks(te, 2), ni = chunks(ti, 2);
            const dim3 ge(kz, kx, ne * pb_.nshots), gi(zh - zl, xh - xl, ni * pb_.nshots);
            k_elastic_fused_part<2><<<ge, fblk, sm, s>>>(f, ne, tm, 0, 0);
            k_elastic_fused_part<1><<<gi, fblk, sm, s>>>(f, ni, tm, zl, xl);
        } else {
            const int nch = chunks((int64_t)kz * kx * pb_.nshots, fused_minb_);
            const dim3 grd(kz, kx, nch * pb_.nshots);
            if (fused_minb_ == 2) {
                if (el) k_elastic_fused<ELASTIC, 2><<<grd, fblk, sm, s>>>(f, nch, tm);
                else k_elastic_fused<VTI, 2><<<grd, fblk, sm, s>>>(f, nch, tm);
            } else {
                if (el) k_elastic_fused<ELASTIC, 1><<<grd, fblk, sm, s>>>(f, nch, tm);
                else k_elastic_fused<VTI, 1><<<grd, fblk, sm, s>>>(f, nch, tm);
            }
        }
        kmark(false, nullptr, 0);
        // SAT of the x/z faces of the fused planes (and, with the marching
        // slabs, of every face of the grid)
        StepArgs sat = f;
        if (slab_march_) {
            sat.y0 = 0;
            sat.y1 = pb_.ny;
        }
        const int nf = face_points(pb_, sat.y0, sat.y1);
        const dim3 sgrd((unsigned)((nf + 127) / 128), pb_.nshots);
        if (pb_.nmodels == 3) k_elastic_face_sat<ELASTIC><<<sgrd, 128, 0, s>>>(sat, nf);
        else k_elastic_face_sat<VTI><<<sgrd, 128, 0, s>>>(sat, nf);
    }
    CK(cudaGetLastError());
}

void Engine::inject(const DevInj &inj, const float *src_dev, int it, float *next)
{
    cudaStream_t s = (cudaStream_t)stream_;
    StepArgs a = make_step_args(pb_, model_.as<float>(), sdiv_ptr_, taper_ptr_, scale_);
    const int nc = pb_.ncomp();
    const int64_t n = pb_.nxyz();
    for (int c = 0; c < nc; c++) a.next[c] = next + c * n;
    for (int c = 0; c < nc; c++) {
        if (inj.n[c] == 0) continue;
        k_inject<<<(inj.n[c] + 127) / 128, 128, 0, s>>>(a, c, inj.gidx[c].as<int64_t>(), inj.trace[c].as<int>(),
                                                         inj.w[c].as<float>(), inj.n[c], src_dev, pb_.nt, it, itp_,
                                                         continuous_ ? shot_t0_.as<int>() : nullptr);
    }
    CK(cudaGetLastError());
}

void Engine::extract(const DevExt &ext, const float *curr, float *rcv_dev, int it)
{
    if (ext.nrec == 0) return;
    cudaStream_t s = (cudaStream_t)stream_;
    const int nc = pb_.ncomp();
    const int64_t n = pb_.nxyz();
    const dim3 grd((ext.nrec + 127) / 128, nc);
    k_extract<<<grd, 128, 0, s>>>(curr, (int64_t)nc * n, n, nc, ext.gidx.as<int64_t>(), ext.w.as<float>(), ext.nrec,
                                  ext.nr, rcv_dev, pb_.nt, it, ext.ntap, itp_,
                                  continuous_ ? shot_t0_.as<int>() : nullptr);
    CK(cudaGetLastError());
}

void Engine::kmark(bool begin, const char *name, int64_t pts)
{
    if (!ktime_ || kev_used_ >= (int)kev_.size() / 2) return;
    cudaEvent_t e = (cudaEvent_t)kev_[2 * kev_used_ + (begin ? 0 : 1)];
    CK(cudaEventRecord(e, (cudaStream_t)stream_));
    if (begin) {
        kname_ = name;
        kpts_ = pts;
    } else {
        kev_used_++;
    }
}

void Engine::time_main_kernel(int max_launches)
{
    CK(cudaSetDevice(device_));
    sync();
    for (void *e : kev_) cudaEventDestroy((cudaEvent_t)e);
    kev_.clear();
    kev_used_ = 0;
    ktime_ = max_launches > 0;
    for (int k = 0; k < 2 * std::max(0, max_launches); k++) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        kev_.push_back(e);
    }
}

double Engine::main_kernel_ms(int *launches, int64_t *points, const char **name)
{
    sync();
    double ms = 0;
    for (int k = 0; k < kev_used_; k++) {
        float t = 0;
        CK(cudaEventElapsedTime(&t, (cudaEvent_t)kev_[2 * k], (cudaEvent_t)kev_[2 * k + 1]));
        ms += t;
    }
    if (launches) *launches = kev_used_;
    if (points) *points = kpts_;
    if (name) *name = kname_;
    return ms;
}

bool Engine::fused_split_active() const
{
    int zl, zh, xl, xh;
    fz_interior_range(pb_.nz, fz::TZ, zl, zh);
    fz_interior_range(pb_.nx, fz::TX, xl, xh);
    return pb_.nmodels == 3 && fused_split_ && fused_minb_ == 2 && zh > zl && xh > xl;
}

int Engine::launches_per_step() const
{
    int k = (pb_.nmodels == 2 ? 1
                              : (march_ ? 2 : (fused_ ? (slab_march_ ? 3 : (pb_.ny < 2 * (fz::YPAD + 2) ? 5 : 6)) : 2)));
    if (fused_ && pb_.nmodels == 3 && pair_) {
        int zl, zh, xl, xh;
        fz_interior_range(pb_.nz, fz::TZ, zl, zh);
        fz_interior_range(pb_.nx, fz::TX, xl, xh);
        if (zh > zl && xh > xl) k += 1;  // interior and edge tiles launched apart
        if (pair_edge_ == 2) {
            // edge tiles in up to three launches (x faces only, z faces only, both)
            const int nzi = zh - zl, nxi = xh - xl, kz = (pb_.nz + fz::TZ - 1) / fz::TZ,
                      kx = (pb_.nx + fz::TX - 1) / fz::TX;
            k += ((kx - nxi) * nzi > 0) + (nxi * (kz - nzi) > 0) + ((kx - nxi) * (kz - nzi) > 0) - 1;
        } else {
            k += pair_edge_;  // edge tiles in two launches (1) or one (0)
        }
    } else if (fused_ && fused_split_active()) {
        k += 1;
    }
    if (ext_.nrec) k += 1;
    for (int c = 0; c < 3; c++) k += inj_.n[c] ? 1 : 0;
    return k;
}

void Engine::set_sources(const InjTable &inj, int ntrace, const float *src)
{
    CK(cudaSetDevice(device_));
    upload_inj(inj, ntrace, inj_);
    src_dev_.alloc(sizeof(float) * (size_t)ntrace * pb_.nt);
    CK(cudaMemcpyAsync(src_dev_.p, src, src_dev_.bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream_));
}

void Engine::set_receivers(const ExtTable &ext, int nr)
{
    CK(cudaSetDevice(device_));
    cudaStream_t s = (cudaStream_t)stream_;
    ext_.nrec = ext.nrec;
    ext_.nr = nr;
    ext_.ntap = ext.ntap;
    ext_.gidx.alloc(sizeof(int64_t) * ext.gidx.size());
    ext_.w.alloc(sizeof(float) * ext.w.size());
    if (ext.nrec) {
        CK(cudaMemcpyAsync(ext_.gidx.p, ext.gidx.data(), ext_.gidx.bytes, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(ext_.w.p, ext.w.data(), ext_.w.bytes, cudaMemcpyHostToDevice, s));
    }
    rcv_dev_.alloc(sizeof(float) * (size_t)pb_.ncomp() * ext.nrec * pb_.nt);
    rcv_dev_.zero(s);
}

void Engine::reset()
{
    CK(cudaSetDevice(device_));
    cudaStream_t s = (cudaStream_t)stream_;
    rot_ = 0;
    fields_.zero(s);
    if (rcv_dev_.p) rcv_dev_.zero(s);
    if (continuous_) {
        // every slot restarts at step 0, active
        shot_t0_.zero(s);
        const std::vector<int> ones(pb_.nshots, 1);
        CK(cudaMemcpyAsync(shot_active_.p, ones.data(), shot_active_.bytes, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
    }
    init_prev(inj_, src_dev_.as<float>(), level(0));
    // capture the replayed steps here (nothing runs), so that the first run
    // does not pay for the capture and instantiation
    if (graphs_ && !ktime_ && pb_.nt > 9 && (!graph_exec_ || graph_key_ != graph_key())) capture_graph();
}

void Engine::run_step(int it, bool taper_prev)
{
    if (!no_extract_) extract(ext_, level(1), rcv_dev_.as<float>(), it);
    step(level(0), level(1), level(2), taper_prev);
    inject(inj_, src_dev_.as<float>(), it, level(2));
    rot_ = (rot_ + 1) % 3;
}

// Everything a captured step sequence bakes in: buffers, tables, options.
uint64_t Engine::graph_key() const
{
    const void *ptrs[] = {fields_.p, model_.p, src_dev_.p, rcv_dev_.p, inj_.gidx[0].p, inj_.gidx[1].p, inj_.gidx[2].p,
                          inj_.trace[0].p, inj_.w[0].p, ext_.gidx.p, ext_.w.p, sdiv_.p, taper_.p, w2c_.p,
                          continuous_ ? shot_t0_.p : nullptr, continuous_ ? shot_active_.p : nullptr};
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
    for (const void *p : ptrs) mix((uint64_t)(uintptr_t)p);
    for (int c = 0; c < 3; c++) mix((uint64_t)inj_.n[c]);
    mix((uint64_t)ext_.nrec);
    mix((uint64_t)no_extract_);
    mix((uint64_t)pb_.nt);
    return h;
}

void Engine::drop_graph()
{
    if (graph_exec_) cudaGraphExecDestroy((cudaGraphExec_t)graph_exec_);
    graph_exec_ = nullptr;
}

// Capture three steps (the rotation period of the time levels) starting at
// rotation 0 with the time index read from the device; false if the capture
// fails (the steps then run as plain launches).
bool Engine::capture_graph()
{
    drop_graph();
    cudaStream_t s = (cudaStream_t)stream_;
    if (!it_dev_.p) it_dev_.alloc(sizeof(int));
    itp_ = it_dev_.as<int>();
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        try {
            // kernels read the time index as k + *itp; it > 0 (taper of prev) as every step after the first
            for (int k = 0; k < 3; k++) run_step(k, true);
            k_tick<<<1, 1, 0, s>>>(itp_, 3);
        } catch (const FwiError &) {
            ok = false;
        }
        ok = cudaStreamEndCapture(s, &g) == cudaSuccess && ok;
    }
    cudaGraphExec_t ex = nullptr;
    ok = ok && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    itp_ = nullptr;
    cudaGetLastError();
    if (!ok) {
        graphs_ = false;
        return false;
    }
    graph_exec_ = ex;
    graph_key_ = graph_key();
    return true;
}

void Engine::run(int it0, int nsteps)
{
    // shot slots run past nt: each shot's sources and receivers stop at its own end
    const int end = continuous_ ? it0 + nsteps : std::min(it0 + nsteps, pb_.nt - 1);
    int it = it0;
    // CUDA graph replay in rotation-aligned blocks of three steps when the
    // run is long enough; step kernels take their per-step arguments from the
    // rotation and the device time index (the main-kernel timing keeps plain
    // launches, its events are per launch)
    const bool graph = graphs_ && !ktime_;
    while (it < end && graph && (rot_ != 0 || it == 0)) {
        run_step(it, it > 0);
        it++;
    }
    const int reps = graph ? (end - it) / 3 : 0;
    if (reps >= 1) {
        if (!graph_exec_ || graph_key_ != graph_key()) capture_graph();
        if (graph_exec_) {
            cudaStream_t s = (cudaStream_t)stream_;
            k_set_it<<<1, 1, 0, s>>>(it_dev_.as<int>(), it);
            for (int r = 0; r < reps; r++) CK(cudaGraphLaunch((cudaGraphExec_t)graph_exec_, s));
            it += 3 * reps;
        }
    }
    while (it < end) {
        run_step(it, it > 0);
        it++;
    }
}

void Engine::extract_last() { extract(ext_, level(1), rcv_dev_.as<float>(), pb_.nt - 1); }

void Engine::set_continuous()
{
    if (continuous_) return;
    CK(cudaSetDevice(device_));
    shot_t0_.alloc(sizeof(int) * pb_.nshots);
    shot_t0_.zero(stream_);
    const std::vector<int> ones(pb_.nshots, 1);
    shot_active_.alloc(sizeof(int) * pb_.nshots);
    CK(cudaMemcpy(shot_active_.p, ones.data(), shot_active_.bytes, cudaMemcpyHostToDevice));
    continuous_ = true;
}

void Engine::release_shot(int slot)
{
    if (slot < 0 || slot >= pb_.nshots) throw FwiError(FWI_ERR_ARG, "slot out of range");
    if (!continuous_) throw FwiError(FWI_ERR_STATE, "slots are not enabled");
    const int zero = 0;
    CK(cudaMemcpyAsync(shot_active_.as<int>() + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, (cudaStream_t)stream_));
    sync();
}

// Tables of every shot into the existing device buffers (a reallocation
// when a count changed; the next run recaptures its graph then).
void Engine::upload_tables(const InjTable &inj, const ExtTable &ext)
{
    cudaStream_t s = (cudaStream_t)stream_;
    for (int c = 0; c < 3; c++) {
        const int n = (int)inj.gidx[c].size();
        if (n != inj_.n[c]) {
            inj_.n[c] = n;
            inj_.gidx[c].alloc(sizeof(int64_t) * n);
            inj_.trace[c].alloc(sizeof(int) * n);
            inj_.w[c].alloc(sizeof(float) * n);
        }
        if (n) {
            CK(cudaMemcpyAsync(inj_.gidx[c].p, inj.gidx[c].data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(inj_.trace[c].p, inj.trace[c].data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(inj_.w[c].p, inj.w[c].data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
        }
    }
    if (ext.nrec != ext_.nrec || ext.ntap != ext_.ntap)
        throw FwiError(FWI_ERR_ARG, "a slot keeps the batch's receiver count");
    CK(cudaMemcpyAsync(ext_.gidx.p, ext.gidx.data(), ext_.gidx.bytes, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ext_.w.p, ext.w.data(), ext_.w.bytes, cudaMemcpyHostToDevice, s));
    // the host tables may go out of scope after return
    sync();
}

void Engine::join_shot(int slot, const InjTable &inj, const ExtTable &ext, int t0)
{
    if (slot < 0 || slot >= pb_.nshots) throw FwiError(FWI_ERR_ARG, "slot out of range");
    CK(cudaSetDevice(device_));
    set_continuous();
    const int64_t n = pb_.nxyz();
    const Dims g{pb_.nx, pb_.ny, pb_.nz};
    StepArgs a = make_step_args(pb_, model_.as<float>(), sdiv_ptr_, taper_ptr_, scale_);
    for (int c = 0; c < 3; c++)
        for (int64_t gi : inj.gidx[c]) {
            if (gi / n != slot) continue;
            const int64_t i = gi % n;
            const int iz = (int)(i % g.nz), ix = (int)((i / g.nz) % g.nx), iy = (int)(i / ((int64_t)g.nz * g.nx));
            if (in_taper(a, ix, iy, iz))
                throw FwiError(FWI_ERR_UNSUPPORTED, "a source point of the joining shot lies in a taper zone");
        }
    upload_tables(inj, ext);
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t sst = (int64_t)pb_.ncomp() * n;
    for (int l = 0; l < 3; l++) CK(cudaMemsetAsync(level(l) + slot * sst, 0, sizeof(float) * sst, s));
    const size_t rows = (size_t)pb_.ncomp() * ext_.nr * pb_.nt;
    CK(cudaMemsetAsync(rcv_dev_.as<float>() + slot * rows, 0, sizeof(float) * rows, s));
    init_prev(inj_, src_dev_.as<float>(), level(0), slot);
    CK(cudaMemcpyAsync(shot_t0_.as<int>() + slot, &t0, sizeof(int), cudaMemcpyHostToDevice, s));
    const int one = 1;
    CK(cudaMemcpyAsync(shot_active_.as<int>() + slot, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    sync();
}

// Strain along the fibre (dipole_to_strain forward, misc.cpp:11-42):
// (w0 u0 + w1 u1 + w2 u2) / gl per sample, in the host formulation's order
// and rounding.  grid: (samples of a shot / 256, shots), raw [.][3][nr][nt].
__global__ void k_das_strain(const float *raw, float *out, const float *w, int nr, int nt, float gl, int s0)
{
    const int64_t cs = (int64_t)nr * nt;
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cs) return;
    const int sh = s0 + blockIdx.y;
    const float *wr = w + ((int64_t)sh * nr + k / nt) * 3;
    const float *p = raw + (int64_t)sh * 3 * cs + k;
    const float v = __fadd_rn(__fadd_rn(__fmul_rn(wr[0], p[0]), __fmul_rn(wr[1], p[cs])), __fmul_rn(wr[2], p[2 * cs]));
    out[(int64_t)blockIdx.y * cs + k] = __fdiv_rn(v, gl);
}

// Its adjoint: u2 = w2 s / gl, u1 = w1 s / gl, u0 = s (w0 / gl), as the host
// formulation rounds them.  src [nsh][nr][nt] -> out [nsh][3][nr][nt].
__global__ void k_das_spread(const float *src, float *out, const float *w, int nr, int nt, float gl)
{
    const int64_t cs = (int64_t)nr * nt;
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cs) return;
    const int sh = blockIdx.y;
    const float *wr = w + ((int64_t)sh * nr + k / nt) * 3;
    const float s = src[(int64_t)sh * cs + k];
    float *o = out + (int64_t)sh * 3 * cs + k;
    o[2 * cs] = __fdiv_rn(__fmul_rn(wr[2], s), gl);
    o[cs] = __fdiv_rn(__fmul_rn(wr[1], s), gl);
    o[0] = __fmul_rn(s, __fdiv_rn(wr[0], gl));
}

void Engine::set_das(const std::vector<float> &w, int nr, float gl)
{
    CK(cudaSetDevice(device_));
    if ((int64_t)w.size() != (int64_t)pb_.nshots * nr * 3) throw FwiError(FWI_ERR_ARG, "DAS weights of every shot's channels");
    das_nr_ = nr;
    das_gl_ = gl;
    das_w_.alloc(sizeof(float) * w.size());
    CK(cudaMemcpyAsync(das_w_.p, w.data(), das_w_.bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream_));
    sync();  // w may go out of scope
}

const float *Engine::strain_traces(int s0, int nsh)
{
    if (das_gl_ <= 0.f) throw FwiError(FWI_ERR_STATE, "no DAS channels set");
    const int64_t cs = (int64_t)das_nr_ * pb_.nt;
    das_rcv_.alloc(sizeof(float) * nsh * cs);
    const dim3 grd((unsigned)((cs + 255) / 256), nsh);
    k_das_strain<<<grd, 256, 0, (cudaStream_t)stream_>>>(rcv_dev_.as<float>(), das_rcv_.as<float>(), das_w_.as<float>(),
                                                         das_nr_, pb_.nt, das_gl_, s0);
    CK(cudaGetLastError());
    return das_rcv_.as<float>();
}

const float *Engine::strain_adjoint(const float *src_dev)
{
    if (das_gl_ <= 0.f) throw FwiError(FWI_ERR_STATE, "no DAS channels set");
    const int64_t cs = (int64_t)das_nr_ * pb_.nt;
    das_src_.alloc(sizeof(float) * pb_.nshots * 3 * cs);
    const dim3 grd((unsigned)((cs + 255) / 256), pb_.nshots);
    k_das_spread<<<grd, 256, 0, (cudaStream_t)stream_>>>(src_dev, das_src_.as<float>(), das_w_.as<float>(), das_nr_,
                                                         pb_.nt, das_gl_);
    CK(cudaGetLastError());
    return das_src_.as<float>();
}

void Engine::copy_strain(int s0, int nsh, float *rcv)
{
    const float *d = strain_traces(s0, nsh);
    CK(cudaMemcpyAsync(rcv, d, sizeof(float) * nsh * das_nr_ * pb_.nt, cudaMemcpyDeviceToHost, (cudaStream_t)stream_));
    sync();
}

void Engine::copy_shot_traces(int slot, float *rcv)
{
    if (slot < 0 || slot >= pb_.nshots) throw FwiError(FWI_ERR_ARG, "slot out of range");
    const size_t rows = (size_t)pb_.ncomp() * ext_.nr * pb_.nt;
    CK(cudaMemcpyAsync(rcv, rcv_dev_.as<float>() + slot * rows, sizeof(float) * rows, cudaMemcpyDeviceToHost,
                       (cudaStream_t)stream_));
    sync();
}

void Engine::copy_traces(float *rcv)
{
    CK(cudaMemcpyAsync(rcv, rcv_dev_.p, rcv_dev_.bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream_));
    sync();
}

// ---------------------------------------------------------------------------
// Snapshot storage.  FP32 keeps every snapshot as is.  FP16P keeps, per
// snapshot k, the second-difference residual r_k = u_k - (2 e_{k-1} - e_{k-2})
// (e = the reconstructed snapshots, FP64; predictions e_{k-1} for k = 1 and 0
// for k = 0) as FP16 scaled by max|r_k| per shot and component.  The encoder
// is closed-loop, so the error of every snapshot is one quantisation step of
// its own residual, and e_{k+1} - 2 e_k + e_{k-1} -- the second time
// difference the density imaging term uses -- is the stored residual itself.
// The adjoint decodes backwards from the encoder's final state:
// e_{j-1} = 2 e_j - e_{j+1} + r_{j+1}.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ double enc_pred(const double *e1, const double *e2, int64_t i, int k)
{
    return k >= 2 ? 2.0 * e1[i] - e2[i] : (k == 1 ? e1[i] : 0.0);
}

// grid (x: points, y: shot*ncomp); e: [2][nsc][n], level 0 = e_{k-1}, level 1 = e_{k-2}
__global__ void k_enc_max(const float *u, const double *e, int64_t n, int nsc, int k, unsigned *amax)
{
    const int sc = blockIdx.y;
    const double *e1 = e + (int64_t)sc * n, *e2 = e + ((int64_t)nsc + sc) * n;
    const float *us = u + (int64_t)sc * n;
    float m = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, (float)fabs((double)us[i] - enc_pred(e1, e2, i, k)));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&amax[sc], __float_as_uint(m));
}

__global__ void k_enc_quant(const float *u, double *e, int64_t n, int nsc, int k, const unsigned *amax, __half *q,
                            float *scales)
{
    const int sc = blockIdx.y;
    double *e1 = e + (int64_t)sc * n, *e2 = e + ((int64_t)nsc + sc) * n;
    const float *us = u + (int64_t)sc * n;
    __half *qs = q + (int64_t)sc * n;
    float sf = __uint_as_float(amax[sc]);
    if (!(sf > 0.f)) sf = 1.f;
    if (blockIdx.x == 0 && threadIdx.x == 0) scales[sc] = sf;
    const double sd = sf;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double p = enc_pred(e1, e2, i, k);
        const __half h = __float2half_rn((float)(((double)us[i] - p) / sd));
        qs[i] = h;
        const double ek = p + (double)__half2float(h) * sd;
        e2[i] = e1[i];
        e1[i] = ek;
    }
}

// One backward step: state (A = e_{j+1}, B = e_j) -> (e_j, e_{j-1}); out = float(e_{j-1}).
__global__ void k_dec_step(double *e, int64_t n, int nsc, const __half *q, const float *scales, float *out)
{
    const int sc = blockIdx.y;
    double *A = e + (int64_t)sc * n, *B = e + ((int64_t)nsc + sc) * n;
    const __half *qs = q + (int64_t)sc * n;
    const double sd = scales[sc];
    float *o = out + (int64_t)sc * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double b = B[i];
        const double v = 2.0 * b - A[i] + (double)__half2float(qs[i]) * sd;
        A[i] = b;
        B[i] = v;
        o[i] = (float)v;
    }
}

__global__ void k_d2f_strided(const double *in, float *out, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

dim3 stream_grid(int64_t n, int nsc)
{
    const int64_t bx = std::min<int64_t>((n + 255) / 256, 1184);
    return dim3((unsigned)std::max<int64_t>(bx, 1), (unsigned)nsc);
}
}  // namespace

void Engine::snap_store(int k)
{
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nsc = pb_.nshots * pb_.ncomp();
    if (k > nsnap_ - 1) return;
    nwritten_ = std::max(nwritten_, k + 1);
    if (rv_C_ > 0) {
        // binomial checkpointing: the forward sweep keeps the states its schedule marks
        if (k < (int)rv_mark_.size() && rv_mark_[k]) {
            const int slot = rv_free_.back();
            rv_free_.pop_back();
            rv_store(slot, level(0), level(1));
            rv_pos_stack_.push_back(k);
            rv_slot_stack_.push_back(slot);
        }
        return;
    }
    if (storage_ == STORE_FP32) {
        CK(cudaMemcpyAsync(snaps_.as<float>() + (int64_t)k * nsc * n, level(1), sizeof(float) * nsc * n,
                           cudaMemcpyDeviceToDevice, s));
        return;
    }
    CK(cudaMemsetAsync(amax_.p, 0, amax_.bytes, s));
    const dim3 grd = stream_grid(n, nsc);
    k_enc_max<<<grd, 256, 0, s>>>(level(1), enc_.as<double>(), n, nsc, k, amax_.as<unsigned>());
    k_enc_quant<<<grd, 256, 0, s>>>(level(1), enc_.as<double>(), n, nsc, k, amax_.as<unsigned>(),
                                    snapq_.as<__half>() + (int64_t)k * nsc * n, snaps_scale_.as<float>() + (int64_t)k * nsc);
    CK(cudaGetLastError());
}

const float *Engine::snap_fp32(int kk)
{
    const int64_t n = pb_.nxyz();
    const int nsc = pb_.nshots * pb_.ncomp();
    const int64_t S = (int64_t)nsc * n;
    if (rv_C_ > 0) {
        if (kk >= nwritten_) return snapz_.as<float>();
        for (int r = 0; r < 3; r++)
            if (ring_[r] == kk) return snaps_.as<float>() + (int64_t)r * S;
        // visit the states below the ring's lowest in decreasing order (the
        // schedule's order) down to kk, keeping each one's current level
        int lo = rv_K_ + 1;
        for (int r = 0; r < 3; r++)
            if (ring_[r] >= 0) lo = std::min(lo, ring_[r]);
        if (kk > lo) throw FwiError(FWI_ERR_STATE, "snapshot requested above the states already visited");
        cudaStream_t s = (cudaStream_t)stream_;
        for (int t = lo - 1; t >= kk; t--) {
            rv_goto(t);
            const int r = t % 3;
            CK(cudaMemcpyAsync(snaps_.as<float>() + (int64_t)r * S, rec_fields_.as<float>() + ((rv_rot_ + 1) % 3) * S,
                               sizeof(float) * S, cudaMemcpyDeviceToDevice, s));
            ring_[r] = t;
        }
        return snaps_.as<float>() + (int64_t)(kk % 3) * S;
    }
    if (storage_ == STORE_FP32) return snaps_.as<float>() + (int64_t)kk * nsc * n;
    if (kk >= nwritten_) return snapz_.as<float>();
    cudaStream_t s = (cudaStream_t)stream_;
    const dim3 grd = stream_grid(n, nsc);
    while (kk < dec_lo_) {
        // decode e_{dec_lo_-1} with the residual of snapshot dec_lo_+1
        const int j = dec_lo_;
        k_dec_step<<<grd, 256, 0, s>>>(enc_.as<double>(), n, nsc, snapq_.as<__half>() + (int64_t)(j + 1) * nsc * n,
                                       snaps_scale_.as<float>() + (int64_t)(j + 1) * nsc,
                                       snaps_.as<float>() + (int64_t)((j - 1) % 3) * nsc * n);
        CK(cudaGetLastError());
        dec_lo_ = j - 1;
    }
    return snaps_.as<float>() + (int64_t)(kk % 3) * nsc * n;
}

// ---------------------------------------------------------------------------
// Binomial checkpointing.  The chain is the sequence of snapshot states
// 0..K (state k: time levels (prev, curr) at step k*sub; one chain step is sub
// time steps).  reverse(s, e, c) visits states e, e-1, ..., s with state s in a
// slot and c free slots: advance d steps from s, keep state s+d in a slot,
// reverse(s+d, e, c-1), then reverse(s, s+d-1, c).  With no free slot every
// state is reached from s again.  The cost table R(l, c) (forward chain steps
// for l = e - s) and the minimising d come from the recursion
//   R(0, c) = 0,  R(l, 0) = l (l + 1) / 2,
//   R(l, c) = min over 1 <= d <= l of  d + R(l - d, c - 1) + R(d - 1, c),
// whose minimum is the binomial bound of Griewank and Walther (revolve).
// ---------------------------------------------------------------------------
struct RevolveTable {
    int K = -1, C = -1;
    std::vector<int32_t> split;  // [(K+1) x (C+1)]
    std::vector<int64_t> cost;
};

static const RevolveTable &revolve_table(int K, int C)
{
    static std::mutex mu;
    static std::vector<std::unique_ptr<RevolveTable>> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (auto &t : cache)
        if (t->K == K && t->C == C) return *t;
    auto t = std::make_unique<RevolveTable>();
    t->K = K;
    t->C = C;
    const int W = C + 1;
    t->split.assign((size_t)(K + 1) * W, 0);
    t->cost.assign((size_t)(K + 1) * W, 0);
    auto R = [&](int l, int c) -> int64_t & { return t->cost[(size_t)l * W + c]; };
    for (int l = 0; l <= K; l++) {
        R(l, 0) = (int64_t)l * (l + 1) / 2;
        t->split[(size_t)l * W] = l;
    }
    // the minimising d does not decrease with l: the search for l starts at
    // the split of l - 1 (any d gives a valid schedule; this one is optimal)
    for (int c = 1; c <= C; c++) {
        int dlo = 1;
        for (int l = 1; l <= K; l++) {
            int64_t best = -1;
            int bd = dlo;
            for (int d = dlo; d <= l; d++) {
                const int64_t v = d + R(l - d, c - 1) + R(d - 1, c);
                if (best < 0 || v < best) {
                    best = v;
                    bd = d;
                }
            }
            R(l, c) = best;
            t->split[(size_t)l * W + c] = bd;
            dlo = bd;
        }
    }
    cache.push_back(std::move(t));
    if (cache.size() > 8) cache.erase(cache.begin());
    return *cache.back();
}

namespace {
// Per (shot, component) max |a - b| of one state (b null: max |a|), as float bits.
__global__ void k_ck_amax(const float *a, const float *b, int64_t n, unsigned *amax)
{
    const int f = blockIdx.y;
    const float *p = a + (int64_t)f * n, *q = b ? b + (int64_t)f * n : nullptr;
    float m = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(q ? p[i] - q[i] : p[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(amax + f, __float_as_uint(m));
}
// 16-bit slot values (a - b) / scale (BF16 or FP16, round to nearest), scale =
// max |a - b| of the (shot, component) field (1 for an all-zero field)
template <class T>
__global__ void k_ck_quant(const float *a, const float *b, int64_t n, const unsigned *amax, T *q, float *scale)
{
    const int f = blockIdx.y;
    const float mx = __uint_as_float(amax[f]);
    const float sc = mx > 0.f ? mx : 1.f;
    const float inv = 1.0f / sc;
    if (blockIdx.x == 0 && threadIdx.x == 0) scale[f] = sc;
    const float *p = a + (int64_t)f * n, *r = b ? b + (int64_t)f * n : nullptr;
    T *o = q + (int64_t)f * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = (r ? p[i] - r[i] : p[i]) * inv;
        if constexpr (std::is_same<T, __half>::value) o[i] = __float2half_rn(v);
        else o[i] = __float2bfloat16_rn(v);
    }
}
// v = q * scale, or (base non-null) v = base - q * scale
template <class T>
__global__ void k_ck_dequant(const T *q, int64_t n, const float *scale, const float *base, float *v)
{
    const int f = blockIdx.y;
    const float sc = scale[f];
    const T *p = q + (int64_t)f * n;
    const float *b = base ? base + (int64_t)f * n : nullptr;
    float *o = v + (int64_t)f * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x;
        if constexpr (std::is_same<T, __half>::value) x = __half2float(p[i]) * sc;
        else x = __bfloat162float(p[i]) * sc;
        o[i] = b ? b[i] - x : x;
    }
}
}  // namespace

// One restart state (prev, curr of the batch) into checkpoint slot `slot`.
// FP32: both levels as they are.  16-bit: curr and the step difference
// curr - prev, each scaled by its own max per (shot, component), so that the
// rounding of the restart keeps the relative precision of the wave's time
// difference as well as of its value.
void Engine::rv_store(int slot, const float *prev, const float *curr)
{
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nsc = pb_.nshots * pb_.ncomp();
    const int64_t S = (int64_t)nsc * n;
    if (rv_prec_ == 0) {
        float *d = rv_store_.as<float>() + (int64_t)slot * 2 * S;
        CK(cudaMemcpyAsync(d, prev, sizeof(float) * S, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(d + S, curr, sizeof(float) * S, cudaMemcpyDeviceToDevice, s));
        return;
    }
    const dim3 grd((unsigned)std::min<int64_t>((n + 255) / 256, 1024), nsc);
    for (int l = 0; l < 2; l++) {
        const float *b = l == 0 ? nullptr : prev;  // level 0: curr; level 1: curr - prev
        CK(cudaMemsetAsync(amax_.p, 0, sizeof(unsigned) * nsc, s));
        k_ck_amax<<<grd, 256, 0, s>>>(curr, b, n, amax_.as<unsigned>());
        float *sc = rv_scale_.as<float>() + ((int64_t)slot * 2 + l) * nsc;
        const int64_t off = ((int64_t)slot * 2 + l) * S;
        if (rv_prec_ == 1)
            k_ck_quant<__nv_bfloat16><<<grd, 256, 0, s>>>(curr, b, n, amax_.as<unsigned>(),
                                                           rv_store_.as<__nv_bfloat16>() + off, sc);
        else
            k_ck_quant<__half><<<grd, 256, 0, s>>>(curr, b, n, amax_.as<unsigned>(), rv_store_.as<__half>() + off, sc);
    }
    CK(cudaGetLastError());
}

// Checkpoint `slot` into the recomputation levels (prev at level 0, curr at level 1).
void Engine::rv_restore(int slot)
{
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nsc = pb_.nshots * pb_.ncomp();
    const int64_t S = (int64_t)nsc * n;
    float *lev = rec_fields_.as<float>();
    rv_rot_ = 0;
    if (rv_prec_ == 0) {
        const float *c = rv_store_.as<float>() + (int64_t)slot * 2 * S;
        CK(cudaMemcpyAsync(lev, c, sizeof(float) * 2 * S, cudaMemcpyDeviceToDevice, s));
        return;
    }
    const dim3 grd((unsigned)std::min<int64_t>((n + 255) / 256, 1024), nsc);
    const float *sc0 = rv_scale_.as<float>() + (int64_t)slot * 2 * nsc, *sc1 = sc0 + nsc;
    const int64_t off0 = (int64_t)slot * 2 * S, off1 = off0 + S;
    // curr into level 1, then prev = curr - (curr - prev) into level 0
    if (rv_prec_ == 1) {
        k_ck_dequant<__nv_bfloat16><<<grd, 256, 0, s>>>(rv_store_.as<__nv_bfloat16>() + off0, n, sc0, nullptr, lev + S);
        k_ck_dequant<__nv_bfloat16><<<grd, 256, 0, s>>>(rv_store_.as<__nv_bfloat16>() + off1, n, sc1, lev + S, lev);
    } else {
        k_ck_dequant<__half><<<grd, 256, 0, s>>>(rv_store_.as<__half>() + off0, n, sc0, nullptr, lev + S);
        k_ck_dequant<__half><<<grd, 256, 0, s>>>(rv_store_.as<__half>() + off1, n, sc1, lev + S, lev);
    }
    CK(cudaGetLastError());
}

// d chain steps (d*sub time steps) on the recomputation levels from state rv_pos_.
void Engine::rv_advance(int d)
{
    std::swap(fields_, rec_fields_);
    const int rot_save = rot_;
    const bool graphs_save = graphs_;
    rot_ = rv_rot_;
    no_extract_ = true;
    graphs_ = false;  // the levels swap in and out: plain launches
    run(rv_pos_ * pb_.sub, d * pb_.sub);
    graphs_ = graphs_save;
    no_extract_ = false;
    rv_rot_ = rot_;
    rot_ = rot_save;
    std::swap(fields_, rec_fields_);
    rv_pos_ += d;
    rv_steps_ += d;
}

// Brings the recomputation levels to state t, below every state visited so
// far: drops the checkpoints above t, restores the highest remaining one and
// advances, keeping the states where the schedule splits the remaining
// interval while free slots last.
void Engine::rv_goto(int t)
{
    PhaseRange phase_range("fwi3d recompute");
    if (rv_pos_ == t) return;
    while (rv_pos_stack_.size() > 1 && rv_pos_stack_.back() > t) {
        rv_free_.push_back(rv_slot_stack_.back());
        rv_pos_stack_.pop_back();
        rv_slot_stack_.pop_back();
    }
    if (rv_pos_ < rv_pos_stack_.back() || rv_pos_ > t) {
        rv_restore(rv_slot_stack_.back());
        rv_pos_ = rv_pos_stack_.back();
    }
    const RevolveTable &T = revolve_table(rv_K_, rv_C_);
    const int W = rv_C_ + 1;
    const int64_t lv = (int64_t)pb_.nshots * pb_.ncomp() * pb_.nxyz();
    while (rv_pos_ < t) {
        const int c = (int)rv_free_.size(), l = t - rv_pos_;
        const int d = c == 0 ? l : T.split[(size_t)l * W + std::min(c, rv_C_)];
        rv_advance(d);
        if (rv_pos_ < t && !rv_free_.empty()) {
            const int slot = rv_free_.back();
            rv_free_.pop_back();
            rv_store(slot, rec_fields_.as<float>() + (rv_rot_ % 3) * lv,
                     rec_fields_.as<float>() + ((rv_rot_ + 1) % 3) * lv);
            rv_pos_stack_.push_back(rv_pos_);
            rv_slot_stack_.push_back(slot);
        }
    }
}

void Engine::forward(const InjTable &inj, int ntrace, const float *src, const ExtTable &ext, float *rcv, bool store)
{
    PhaseRange phase_range("fwi3d forward");
    CK(cudaSetDevice(device_));
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nsc = pb_.nshots * pb_.ncomp();
    set_sources(inj, ntrace, src);
    set_receivers(ext, ext.nrec / pb_.nshots);
    snaps_valid_ = false;
    nwritten_ = 0;
    const bool keep = store && pb_.sub > 0;
    rv_C_ = 0;
    rv_pos_ = -1;
    rv_pos_stack_.clear();
    rv_slot_stack_.clear();
    rv_free_.clear();
    rv_mark_.clear();
    ring_[0] = ring_[1] = ring_[2] = -1;
    if (keep) {
        nsnap_ = 1 + pb_.nt / pb_.sub;
        // FP16P needs at least three stored snapshots to decode backwards
        const int written = 1 + (pb_.nt - 1) / pb_.sub;
        if (storage_ == STORE_FP16P && written < 3) storage_ = STORE_FP32;
        const int64_t S = (int64_t)sizeof(float) * nsc * n;  // one snapshot of the batch
        const int64_t full = storage_ == STORE_FP32 ? nsnap_ * S : nsnap_ * S / 2 + 8 * S;
        // checkpoint slot bytes (two levels) and the fixed part: recomputation
        // levels, FP32 ring of three snapshots, zero snapshot
        const int64_t slot_bytes = rv_prec_ == 0 ? 2 * S : S;
        const int64_t fixed = 7 * S;
        int C = 0;
        if (rv_C_req_ > 0) {
            C = rv_C_req_;
        } else if (budget_ > 0 && full > budget_) {
            if (budget_ < fixed + 2 * slot_bytes)
                throw FwiError(FWI_ERR_OOM, "snapshot budget of " + std::to_string(budget_) +
                                                " bytes is below the checkpointing minimum of " +
                                                std::to_string(fixed + 2 * slot_bytes));
            C = (int)std::min<int64_t>((budget_ - fixed) / slot_bytes, written);
        }
        if (C > 0) {
            // binomial checkpointing over the chain 0..K; slot 0 keeps state 0
            rv_K_ = written - 1;
            // more slots than states, or than 256 (the schedule's table grows with them), gain nothing here
            rv_C_ = std::max(1, std::min({C, std::max(1, rv_K_), 256}));
            snapq_.alloc(0);
            snaps_scale_.alloc(0);
            enc_.alloc(0);
            rv_store_.alloc((size_t)rv_C_ * slot_bytes);
            rv_scale_.alloc(rv_prec_ == 0 ? 0 : sizeof(float) * 2 * (size_t)rv_C_ * nsc);
            amax_.alloc(sizeof(unsigned) * (size_t)nsc);
            rec_fields_.alloc(3 * (size_t)S);
            snaps_.alloc(3 * (size_t)S);
            snapz_.alloc((size_t)S);
            snapz_.zero(s);
            for (int k = rv_C_ - 1; k >= 0; k--) rv_free_.push_back(k);
            // the forward sweep keeps state 0 and the splits of the schedule's first descent
            rv_mark_.assign(rv_K_ + 1, 0);
            rv_mark_[0] = 1;
            const RevolveTable &T = revolve_table(rv_K_, rv_C_);
            int p = 0, c = rv_C_ - 1;
            while (c > 0 && p < rv_K_) {
                p += T.split[(size_t)(rv_K_ - p) * (rv_C_ + 1) + c];
                if (p >= rv_K_) break;
                rv_mark_[p] = 1;
                c--;
            }
        } else if (storage_ == STORE_FP32) {
            rv_store_.alloc(0);
            rv_scale_.alloc(0);
            rec_fields_.alloc(0);
            snapq_.alloc(0);
            snaps_scale_.alloc(0);
            enc_.alloc(0);
            snapz_.alloc(0);
            snaps_.alloc(sizeof(float) * (size_t)nsnap_ * nsc * n);
            snaps_.zero(s);
        } else {
            rv_store_.alloc(0);
            rv_scale_.alloc(0);
            rec_fields_.alloc(0);
            snaps_.alloc(sizeof(float) * 3 * (size_t)nsc * n);
            snapq_.alloc(sizeof(__half) * (size_t)nsnap_ * nsc * n);
            snaps_scale_.alloc(sizeof(float) * (size_t)nsnap_ * nsc);
            enc_.alloc(sizeof(double) * 2 * (size_t)nsc * n);
            enc_.zero(s);
            amax_.alloc(sizeof(unsigned) * (size_t)nsc);
            snapz_.alloc(sizeof(float) * (size_t)nsc * n);
            snapz_.zero(s);
        }
    }
    reset();
    for (int it = 0; it < pb_.nt - 1; it++) {
        if (keep && it % pb_.sub == 0) snap_store(it / pb_.sub);
        run(it, 1);
    }
    if (keep && (pb_.nt - 1) % pb_.sub == 0) snap_store((pb_.nt - 1) / pb_.sub);
    if (keep && rv_C_ > 0 && (pb_.nt - 1) % pb_.sub == 0) {
        // the last state stays available: the recomputation levels start from it
        const int64_t S = (int64_t)nsc * n;
        CK(cudaMemcpyAsync(rec_fields_.as<float>(), level(0), sizeof(float) * S, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(rec_fields_.as<float>() + S, level(1), sizeof(float) * S, cudaMemcpyDeviceToDevice, s));
        rv_rot_ = 0;
        rv_pos_ = rv_K_;
    }
    rv_steps_ = 0;
    if (keep && rv_C_ == 0 && storage_ == STORE_FP16P) {
        // decoder starts from the encoder's final state (e_K, e_{K-1})
        const int K = nwritten_ - 1;
        const double *e = enc_.as<double>();
        const dim3 grd = stream_grid((int64_t)nsc * n, 1);
        k_d2f_strided<<<grd, 256, 0, s>>>(e, snaps_.as<float>() + (int64_t)(K % 3) * nsc * n, (int64_t)nsc * n);
        k_d2f_strided<<<grd, 256, 0, s>>>(e + (int64_t)nsc * n, snaps_.as<float>() + (int64_t)((K - 1) % 3) * nsc * n,
                                          (int64_t)nsc * n);
        CK(cudaGetLastError());
        dec_lo_ = K - 1;
    }
    extract_last();
    if (rcv) copy_traces(rcv);
    snaps_valid_ = keep;
}

// ---------------------------------------------------------------------------
// Device residual of the FWI objective (ResidualArgs in engine.h).  Each
// sample is formed with the host path's float / double operations, without
// contraction, in the same order; only the misfit sum is reassociated (FP64
// partials per trace, summed in trace order on the host).
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ float rs_tap(float acc, float v, float s, double w)
{
    // acc = (float)((double)acc + (double)(v * s) * w)   (operator.cpp:472-520)
    return __double2float_rn(__dadd_rn((double)acc, __dmul_rn((double)__fmul_rn(v, s), w)));
}

// Dt of one trace (misc.cpp:70-94), adj as apply_dt
__device__ void rs_dt(bool adj, const float *in, float *out, int nt, float dt)
{
    for (int it = threadIdx.x; it < nt; it += blockDim.x) {
        float v;
        if (!adj) {
            if (it == 0) v = __fdiv_rn(__fsub_rn(in[1], in[0]), dt);
            else if (it == nt - 1) v = __fdiv_rn(__fsub_rn(in[nt - 1], in[nt - 2]), dt);
            else v = __fdiv_rn(__fsub_rn(in[it + 1], in[it - 1]), __fmul_rn(2.f, dt));
        } else {
            if (it == 0) v = __fdiv_rn(__fadd_rn(in[1], in[0]), dt);
            else if (it == nt - 1) v = __fdiv_rn(__fsub_rn(-in[nt - 1], in[nt - 2]), dt);
            else v = __fdiv_rn(__fsub_rn(in[it + 1], in[it - 1]), __fmul_rn(2.f, dt));
        }
        out[it] = v;
    }
}

// Modeling output of one trace (blockIdx.x): Dt for velocity data, times
// alpha, adjoint resampling to the data axis (the first half of k_residual,
// without the observed data).
__global__ void k_trace_data(ResidualArgs a)
{
    extern __shared__ float rs_sm[];
    const int nt = a.nt, ntd = a.ntd;
    float *r = rs_sm, *tmp = rs_sm + nt;
    const int64_t tr = blockIdx.x;
    const float *src = a.rcv + tr * nt;
    for (int it = threadIdx.x; it < nt; it += blockDim.x) r[it] = src[it];
    __syncthreads();
    if (a.seismotype == 1) {
        rs_dt(false, r, tmp, nt, a.dt);
        __syncthreads();
        for (int it = threadIdx.x; it < nt; it += blockDim.x) r[it] = tmp[it];
        __syncthreads();
    }
    for (int it = threadIdx.x; it < nt; it += blockDim.x) r[it] = __fmul_rn(r[it], a.alpha);
    __syncthreads();
    for (int j = threadIdx.x; j < ntd; j += blockDim.x) {
        float d = 0.f;
        for (int itd = a.jlo[j]; itd < a.jhi[j]; itd++) {
            const int k = j - a.first[itd];
            if (k < 0 || k >= a.count[itd]) continue;
            const int q = a.off[itd] + k;
            d = rs_tap(d, r[itd], a.s[q], a.win[q]);
        }
        a.resid[tr * ntd + j] = d;
    }
}

__global__ void k_residual(ResidualArgs a)
{
    extern __shared__ float rs_sm[];
    const int nt = a.nt, ntd = a.ntd;
    float *r = rs_sm, *syn = rs_sm + nt, *as = syn + ntd, *tmp = as + nt;
    __shared__ double red[32];
    const int64_t tr = blockIdx.x;
    const float *src = a.rcv + tr * nt;
    bool bad = false;
    for (int it = threadIdx.x; it < nt; it += blockDim.x) {
        const float v = src[it];
        bad |= !isfinite(v);
        r[it] = v;
    }
    if (bad) atomicOr(a.bad, 1);
    __syncthreads();
    if (a.seismotype == 1) {
        rs_dt(false, r, tmp, nt, a.dt);
        __syncthreads();
        for (int it = threadIdx.x; it < nt; it += blockDim.x) r[it] = tmp[it];
        __syncthreads();
    }
    for (int it = threadIdx.x; it < nt; it += blockDim.x) r[it] = __fmul_rn(r[it], a.alpha);
    __syncthreads();
    // adjoint resampling (gather over the propagation samples that reach j,
    // in increasing order as the host's scatter adds them), minus observed
    const float *ob = a.obs + tr * ntd;
    double ss = 0.0;
    for (int j = threadIdx.x; j < ntd; j += blockDim.x) {
        float d = 0.f;
        for (int itd = a.jlo[j]; itd < a.jhi[j]; itd++) {
            const int k = j - a.first[itd];
            if (k < 0 || k >= a.count[itd]) continue;
            const int q = a.off[itd] + k;
            d = rs_tap(d, r[itd], a.s[q], a.win[q]);
        }
        d = __fsub_rn(d, ob[j]);
        syn[j] = d;
        if (a.resid) a.resid[tr * ntd + j] = d;
        ss = __dadd_rn(ss, __dmul_rn((double)d, (double)d));
    }
    // block sum of the squares (FP64)
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        const double a0 = syn[0], a1 = syn[ntd - 1];
        a.part[tr] = t - 0.5 * (a0 * a0 + a1 * a1);
    }
    __syncthreads();
    // Ht on the data axis (misc.cpp:44-68)
    for (int j = threadIdx.x; j < ntd; j += blockDim.x) {
        const float v = syn[j];
        tmp[j] = (j == 0 || j == ntd - 1) ? __double2float_rn(__dmul_rn(__dmul_rn((double)v, 0.5), (double)a.dtd))
                                           : __fmul_rn(v, a.dtd);
    }
    __syncthreads();
    // forward resampling to the propagation axis, Ht^-1
    for (int it = threadIdx.x; it < nt; it += blockDim.x) {
        float acc = 0.f;
        const int f0 = a.first[it], c0 = a.count[it], q0 = a.off[it];
        for (int k = 0; k < c0; k++) acc = rs_tap(acc, tmp[f0 + k], a.s[q0 + k], a.win[q0 + k]);
        as[it] = (it == 0 || it == nt - 1) ? __double2float_rn(__ddiv_rn((double)acc, __dmul_rn(0.5, (double)a.dt)))
                                           : __fdiv_rn(acc, a.dt);
    }
    __syncthreads();
    // time reversal and -alpha, then Dt^T for velocity data
    const float na = -a.alpha;
    for (int it = threadIdx.x; it < nt; it += blockDim.x) r[it] = __fmul_rn(as[nt - 1 - it], na);
    __syncthreads();
    const float *fin = r;
    if (a.seismotype == 1) {
        rs_dt(true, r, tmp, nt, a.dt);
        __syncthreads();
        fin = tmp;
    }
    float *dst = a.asrc + tr * nt;
    for (int it = threadIdx.x; it < nt; it += blockDim.x) dst[it] = fin[it];
}
}  // namespace

void DeviceResidual::set_observed(int device, const std::vector<float> &obs)
{
    if (device_ == device && obs_.bytes == sizeof(float) * obs.size()) return;
    CK(cudaSetDevice(device));
    obs_.alloc(sizeof(float) * obs.size());
    CK(cudaMemcpy(obs_.p, obs.data(), obs_.bytes, cudaMemcpyHostToDevice));
    device_ = device;
}

void DeviceResidual::set_axes(int hl, int ntd, float dtd, int nt, float dt)
{
    if (hl == hl_ && ntd == ntd_ && dtd == dtd_ && nt == nt_ && dt == dt_) return;
    std::vector<int> first, count;
    std::vector<float> sv;
    std::vector<double> wv;
    sinc_resample_taps(hl, ntd, dtd, nt, dt, first, count, sv, wv);
    std::vector<int> off(nt + 1, 0), jlo(ntd, nt), jhi(ntd, 0);
    for (int it = 0; it < nt; it++) off[it + 1] = off[it] + count[it];
    for (int it = 0; it < nt; it++)
        for (int k = 0; k < count[it]; k++) {
            const int j = first[it] + k;
            jlo[j] = std::min(jlo[j], it);
            jhi[j] = std::max(jhi[j], it + 1);
        }
    for (int j = 0; j < ntd; j++)
        if (jlo[j] >= jhi[j]) jlo[j] = jhi[j] = 0;
    auto up = [](DevBuf &b, const void *h, size_t bytes) {
        b.alloc(std::max<size_t>(bytes, 8));
        if (bytes) CK(cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice));
    };
    up(first_, first.data(), sizeof(int) * first.size());
    up(count_, count.data(), sizeof(int) * count.size());
    up(off_, off.data(), sizeof(int) * off.size());
    up(s_, sv.data(), sizeof(float) * sv.size());
    up(win_, wv.data(), sizeof(double) * wv.size());
    up(jlo_, jlo.data(), sizeof(int) * jlo.size());
    up(jhi_, jhi.data(), sizeof(int) * jhi.size());
    hl_ = hl;
    ntd_ = ntd;
    dtd_ = dtd;
    nt_ = nt;
    dt_ = dt;
}

void DeviceResidual::data(Engine &eng, const float *traces, int ntraces, int seismotype, float alpha, float *out)
{
    if (ntraces <= 0) return;
    cudaStream_t st = (cudaStream_t)eng.stream();
    const size_t nt = (size_t)nt_, ntd = (size_t)ntd_;
    if (resid_.bytes < sizeof(float) * ntraces * ntd) resid_.alloc(sizeof(float) * ntraces * ntd);
    ResidualArgs a{};
    a.rcv = traces;
    a.resid = resid_.as<float>();
    a.first = first_.as<int>();
    a.count = count_.as<int>();
    a.off = off_.as<int>();
    a.s = s_.as<float>();
    a.win = win_.as<double>();
    a.jlo = jlo_.as<int>();
    a.jhi = jhi_.as<int>();
    a.nt = nt_;
    a.ntd = ntd_;
    a.seismotype = seismotype;
    a.alpha = alpha;
    a.dt = dt_;
    a.dtd = dtd_;
    static std::once_flag once;
    std::call_once(once, [] {
        CK(cudaFuncSetAttribute(k_trace_data, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(float) * 2 * kResidualMaxSamples)));
    });
    k_trace_data<<<ntraces, 128, sizeof(float) * 2 * nt, st>>>(a);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, resid_.p, sizeof(float) * ntraces * ntd, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

double DeviceResidual::run(Engine &eng, size_t obs_offset, int ntraces, int seismotype, float alpha, float *residual,
                           double *per_trace, const float *traces)
{
    if (ntraces <= 0) return 0.0;
    cudaStream_t st = (cudaStream_t)eng.stream();
    const size_t nt = (size_t)nt_, ntd = (size_t)ntd_;
    if (asrc_.bytes < sizeof(float) * ntraces * nt) asrc_.alloc(sizeof(float) * ntraces * nt);
    if (part_.bytes < sizeof(double) * ntraces) part_.alloc(sizeof(double) * ntraces);
    if (residual && resid_.bytes < sizeof(float) * ntraces * ntd) resid_.alloc(sizeof(float) * ntraces * ntd);
    if (!bad_.p) bad_.alloc(sizeof(int));
    CK(cudaMemsetAsync(bad_.p, 0, sizeof(int), st));
    ResidualArgs a{};
    a.rcv = traces ? traces : eng.traces_dev();  // DAS: the strain traces
    a.obs = obs_.as<float>() + obs_offset;
    a.asrc = asrc_.as<float>();
    a.resid = residual ? resid_.as<float>() : nullptr;
    a.part = part_.as<double>();
    a.bad = bad_.as<int>();
    a.first = first_.as<int>();
    a.count = count_.as<int>();
    a.off = off_.as<int>();
    a.s = s_.as<float>();
    a.win = win_.as<double>();
    a.jlo = jlo_.as<int>();
    a.jhi = jhi_.as<int>();
    a.nt = nt_;
    a.ntd = ntd_;
    a.seismotype = seismotype;
    a.alpha = alpha;
    a.dt = dt_;
    a.dtd = dtd_;
    static std::once_flag once;
    std::call_once(once, [] {
        CK(cudaFuncSetAttribute(k_residual, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(float) * 4 * kResidualMaxSamples)));
    });
    const size_t sm = sizeof(float) * (2 * nt + 2 * std::max(nt, ntd));
    k_residual<<<ntraces, 128, sm, st>>>(a);
    CK(cudaGetLastError());
    std::vector<double> part(ntraces);
    int bad = 0;
    CK(cudaMemcpyAsync(part.data(), part_.p, sizeof(double) * ntraces, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&bad, bad_.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (residual) CK(cudaMemcpyAsync(residual, resid_.p, sizeof(float) * ntraces * ntd, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (bad) throw FwiError(FWI_ERR_NAN, "non-finite values in the traces");
    double sum = 0.0;
    for (int k = 0; k < ntraces; k++) sum += part[k];
    if (per_trace) std::copy(part.begin(), part.end(), per_trace);
    return sum;
}

void Engine::image(int itl, const float *curr, const float *prevl)
{
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nc = pb_.ncomp();
    ImageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = Dims{pb_.nx, pb_.ny, pb_.nz};
    a.dx = pb_.dx;
    a.dy = pb_.dy;
    a.dz = pb_.dz;
    a.rdx = 1.0f / pb_.dx;
    a.rdy = 1.0f / pb_.dy;
    a.rdz = 1.0f / pb_.dz;
    a.dtimg = pb_.sub * pb_.dt;
    a.itl = itl;
    a.last = pb_.nt / pb_.sub;
    for (int k = 0; k < pb_.nmodels; k++) a.m[k] = model_.as<float>() + k * n;
    const float *lev[3];
    for (int l = 0; l < 3; l++) {
        const int k = itl - 1 + l;
        lev[l] = snap_fp32(std::min(std::max(k, 0), nsnap_ - 1));
    }
    PhaseRange phase_range("fwi3d imaging");  // after the snapshots' retrieval (decoding, recomputation)
    const dim3 blk(BZ, BX, BY), grd = grid_of(a.g, 1);
    for (int l = 0; l < 3; l++)
        for (int c = 0; c < 3; c++) a.fwd[l][c] = lev[l] + (int64_t)(c < nc ? c : 0) * n;
    for (int c = 0; c < 3; c++) {
        const int cc = c < nc ? c : 0;
        a.adj[c] = curr + cc * n;
        a.lag[c] = prevl + cc * n;
        a.grad[c] = grad_.as<double>() + (int64_t)(c < (pb_.nmodels == 2 ? 2 : 3) ? c : 0) * n;
    }
    const int64_t sst = (int64_t)nc * n;
    const int64_t gst = per_shot_grad_ ? (int64_t)std::min(3, pb_.nmodels) * n : 0;
    if (image_split_ && pb_.nmodels != 2 && pb_.nx > 8 && pb_.ny > 8 && pb_.nz > 8) {
        // interior box and shell apart: the box's warps take the interior rows only
        const dim3 gbox = grid_of(Dims{pb_.nx - 8, pb_.ny - 8, pb_.nz}, 1);
        const int64_t nsh = n - (int64_t)(pb_.nx - 8) * (pb_.ny - 8) * (pb_.nz - 8);
        const unsigned gsh = (unsigned)((nsh + 255) / 256);
        if (pb_.nmodels == 3) {
            k_image_batch<ELASTIC, 1><<<gbox, blk, 0, s>>>(a, pb_.nshots, sst, gst);
            k_image_batch<ELASTIC, 2><<<gsh, 256, 0, s>>>(a, pb_.nshots, sst, gst);
        } else {
            k_image_batch<VTI, 1><<<gbox, blk, 0, s>>>(a, pb_.nshots, sst, gst);
            k_image_batch<VTI, 2><<<gsh, 256, 0, s>>>(a, pb_.nshots, sst, gst);
        }
    } else if (pb_.nmodels == 2) {
        k_image_batch<ACOUSTIC><<<grd, blk, 0, s>>>(a, pb_.nshots, sst, gst);
    } else if (pb_.nmodels == 3) {
        k_image_batch<ELASTIC><<<grd, blk, 0, s>>>(a, pb_.nshots, sst, gst);
    } else {
        k_image_batch<VTI><<<grd, blk, 0, s>>>(a, pb_.nshots, sst, gst);
    }
    CK(cudaGetLastError());
}

void Engine::adjoint(const InjTable &inj, int ntrace, const float *adj_src, float *grad)
{
    adjoint_impl(inj, ntrace, adj_src, nullptr, grad);
}

void Engine::adjoint_dev(const InjTable &inj, int ntrace, const float *adj_src_dev, float *grad)
{
    adjoint_impl(inj, ntrace, nullptr, adj_src_dev, grad);
}

void Engine::adjoint_impl(const InjTable &inj, int ntrace, const float *adj_src, const float *adj_src_dev, float *grad)
{
    PhaseRange phase_range("fwi3d adjoint");
    CK(cudaSetDevice(device_));
    if (!snaps_valid_) throw FwiError(FWI_ERR_STATE, "adjoint needs the snapshots of a preceding forward with sub > 0");
    cudaStream_t s = (cudaStream_t)stream_;
    const int64_t n = pb_.nxyz();
    const int nm = std::min(3, pb_.nmodels);
    // adjoint source tables, host adjoint sources and the FP32 gradient live
    // in members of the engine: a repeated evaluation (same counts) reuses
    // them instead of a cudaMalloc / cudaFree pair, which would synchronise
    // the device under other sessions' work
    DevInj &dinj = adj_inj_;
    upload_inj(inj, ntrace, dinj);
    const float *asrc_p = adj_src_dev;
    if (!asrc_p) {
        adj_src_buf_.alloc(sizeof(float) * (size_t)ntrace * pb_.nt);
        CK(cudaMemcpyAsync(adj_src_buf_.p, adj_src, adj_src_buf_.bytes, cudaMemcpyHostToDevice, s));
        asrc_p = adj_src_buf_.as<float>();
    }
    const int64_t ng = (per_shot_grad_ ? pb_.nshots : 1) * nm * n;  // one gradient, or one per shot
    grad_.alloc(sizeof(double) * ng);
    grad_.zero(s);
    rot_ = 0;
    fields_.zero(s);
    init_prev(dinj, asrc_p, level(0));
    const int sub = pb_.sub;
    for (int it = 0; it < pb_.nt - 1; it++) {
        if ((pb_.nt - 1 - it) % sub == 0 && it != 0) image((pb_.nt - 1 - it) / sub, level(1), level(0));
        step(level(0), level(1), level(2), it > 0);
        inject(dinj, asrc_p, it, level(2));
        rot_ = (rot_ + 1) % 3;
    }
    image(0, level(1), level(0));
    DevBuf &gf = grad_f32_;
    gf.alloc(sizeof(float) * ng);
    k_d2f<<<(unsigned)((ng + 255) / 256), 256, 0, s>>>(grad_.as<double>(), gf.as<float>(), ng);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(grad, gf.p, gf.bytes, cudaMemcpyDeviceToHost, s));
    sync();
    // the FP16P decoder state and the checkpoint stack are consumed by the adjoint
    snaps_valid_ = rv_C_ == 0 && storage_ == STORE_FP32;
}

// ---------------------------------------------------------------------------
// Allocation-free elastic step on caller-owned buffers (fwi_elastic_step_static)
// ---------------------------------------------------------------------------
// The first-derivative scratch of this entry point is the file-scope array
// below: kStaticMaxPoints grid points x 9 derivative fields = 9 MiB.  Nothing
// in it needs to start at zero, because k_elastic_aux writes every point that
// k_elastic_step reads in the same call.  All calls on one device share it,
// so calls that overlap in time on one device (two streams, two host threads)
// race on it; the caller serialises them.  The per-point step kernel always
// multiplies by the six taper tables; a taper-free step points all six at a
// second static array of ones, written once at set-up.
namespace {
constexpr int64_t kStaticMaxPoints = int64_t(1) << 18;  // 262,144 points, e.g. 64^3
constexpr int kStaticMaxAxis = 2048;                    // >= 2^18 / (12 * 12)
constexpr int kStaticMaxDevices = 64;
}  // namespace

static __device__ __align__(256) float g_static_aux[9 * kStaticMaxPoints];
static __device__ __align__(256) float g_static_ones[kStaticMaxAxis];

namespace {
__global__ void k_static_fill_ones()
{
    for (int i = threadIdx.x; i < kStaticMaxAxis; i += blockDim.x) g_static_ones[i] = 1.f;
}

struct StaticScratch {
    float *aux = nullptr;   // device address of g_static_aux
    float *ones = nullptr;  // device address of g_static_ones
};
std::mutex g_static_mu;
StaticScratch g_static[kStaticMaxDevices];

// Set-up, once per device with that device current: resolve the scratch
// addresses, fill the table of ones and load the SBP coefficient tables into
// constant memory.  These are synchronous runtime calls, so the first call on
// a device belongs before any stream capture on it.
StaticScratch static_scratch(int dev)
{
    std::lock_guard<std::mutex> lock(g_static_mu);
    StaticScratch &st = g_static[dev];
    if (!st.aux) {
        float *aux = nullptr, *ones = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&aux, g_static_aux);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void **)&ones, g_static_ones);
        if (e != cudaSuccess || !aux || !ones)
            throw FwiError(FWI_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
        init_sbp_tables();
        CK(cudaMemcpyToSymbol(c_sbp, &g_sbp_host, sizeof(SbpTables)));
        k_static_fill_ones<<<1, 256, 0, 0>>>();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(0));
        st.ones = ones;
        st.aux = aux;
    }
    return st;
}

void require_device_ptr(const void *p, int dev, const char *name)
{
    cudaPointerAttributes at;
    CK(cudaPointerGetAttributes(&at, p));
    if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != dev)
        throw FwiError(FWI_ERR_ARG, std::string(name) + " is not device memory of the current device");
}
}  // namespace

void static_elastic_step(const fwi_grid &grid, int nmodels, const int bc[6], float dt, const float *model,
                         const float *prev, const float *curr, float *next, void *stream)
{
    if (nmodels != 3 && nmodels != 6) throw FwiError(FWI_ERR_ARG, "nmodels must be 3 (elastic) or 6 (VTI)");
    if (grid.nx < 12 || grid.ny < 12 || grid.nz < 12)
        throw FwiError(FWI_ERR_ARG, "each grid axis needs at least 12 points (two 6-row SBP closures)");
    const int64_t n = (int64_t)grid.nx * grid.ny * grid.nz;
    if (n > kStaticMaxPoints)
        throw FwiError(FWI_ERR_ARG, "grid of " + std::to_string(n) + " points exceeds the static scratch limit of " +
                                        std::to_string(kStaticMaxPoints) + " points");
    if (std::max(grid.nx, std::max(grid.ny, grid.nz)) > kStaticMaxAxis)
        throw FwiError(FWI_ERR_ARG, "a grid axis exceeds " + std::to_string(kStaticMaxAxis) + " points");
    if (!(grid.dx > 0 && grid.dy > 0 && grid.dz > 0 && dt > 0)) throw FwiError(FWI_ERR_ARG, "spacings and dt must be > 0");
    for (int f = 0; f < 6; f++)
        if (bc[f] != BC_NONE && bc[f] != BC_FREE)
            throw FwiError(FWI_ERR_UNSUPPORTED,
                           "only bc 0 (none) and 1 (traction-free) faces: absorbing and rigid faces need the "
                           "model-dependent boundary tables that the operator and batch paths build");
    // next is written at every point while curr is read at neighbouring
    // points and prev at the point itself: next may be prev (the leapfrog
    // in place) but may overlap neither curr nor the model, nor prev in part
    {
        const uintptr_t nb = (uintptr_t)next, ne = nb + sizeof(float) * 3 * (size_t)n;
        auto overlaps = [&](const float *p, size_t count) {
            const uintptr_t b = (uintptr_t)p, e = b + sizeof(float) * count;
            return b < ne && nb < e;
        };
        if (overlaps(curr, 3 * (size_t)n)) throw FwiError(FWI_ERR_ARG, "next overlaps curr");
        if (overlaps(model, (size_t)nmodels * n)) throw FwiError(FWI_ERR_ARG, "next overlaps the model");
        if (next != prev && overlaps(prev, 3 * (size_t)n))
            throw FwiError(FWI_ERR_ARG, "next overlaps prev in part (it may only be prev itself)");
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) throw FwiError(FWI_ERR_NOGPU, "no CUDA device");
    if (dev >= kStaticMaxDevices) throw FwiError(FWI_ERR_ARG, "device ordinal above the static set-up table");
    require_device_ptr(model, dev, "model");
    require_device_ptr(prev, dev, "prev");
    require_device_ptr(curr, dev, "curr");
    require_device_ptr(next, dev, "next");
    const StaticScratch st = static_scratch(dev);
    float *scr = st.aux;

    Problem pb{};
    pb.nmodels = nmodels;
    pb.nx = grid.nx;
    pb.ny = grid.ny;
    pb.nz = grid.nz;
    pb.dx = grid.dx;
    pb.dy = grid.dy;
    pb.dz = grid.dz;
    pb.dt = dt;
    pb.nt = 2;
    pb.sub = 0;
    for (int f = 0; f < 6; f++) {
        pb.bc[f] = bc[f];
        pb.taper[f] = 0;
    }
    pb.taper_strength = 0.f;
    pb.free_surface_stiffness = 1.f;
    pb.nshots = 1;
    const float *no_sdiv[6][3] = {};  // read only when a face is absorbing
    const float *ones[6] = {st.ones, st.ones, st.ones, st.ones, st.ones, st.ones};
    StepArgs a = make_step_args(pb, model, no_sdiv, ones, 0);
    AuxArgs x;
    std::memset(&x, 0, sizeof(x));
    x.g = a.g;
    x.dx = pb.dx;
    x.dy = pb.dy;
    x.dz = pb.dz;
    for (int k = 0; k < nmodels; k++) x.m[k] = a.m[k];
    for (int c = 0; c < 3; c++) {
        a.curr[c] = x.curr[c] = curr + c * n;
        a.prev[c] = prev + c * n;
        a.next[c] = next + c * n;
    }
    a.taper_prev = 0;
    // scratch layout as the engine's: elastic shares one divergence slot for T0..T2
    if (nmodels == 3) {
        x.aux[AUX_T0] = x.aux[AUX_T1] = x.aux[AUX_T2] = scr;
        for (int k = 3; k < 9; k++) x.aux[k] = scr + (k - 2) * n;
    } else {
        for (int k = 0; k < 9; k++) x.aux[k] = scr + k * n;
    }
    for (int k = 0; k < 9; k++) a.aux[k] = x.aux[k];
    a.y0 = x.y0 = 0;
    a.y1 = x.y1 = pb.ny;
    a.nyb = x.nyb = yblocks(pb.ny);
    x.sst = a.sst;
    x.ast = a.ast;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 blk(BZ, BX, BY), grd = grid_of(a.g, 1, pb.ny);
    if (nmodels == 3) {
        k_elastic_aux<ELASTIC><<<grd, blk, 0, s>>>(x);
        k_elastic_step<ELASTIC><<<grd, blk, 0, s>>>(a);
    } else {
        k_elastic_aux<VTI><<<grd, blk, 0, s>>>(x);
        k_elastic_step<VTI><<<grd, blk, 0, s>>>(a);
    }
    CK(cudaGetLastError());
}

}  // namespace fwi
