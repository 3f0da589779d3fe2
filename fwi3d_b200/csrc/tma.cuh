// Bulk-tensor (TMA) plane copies of the marching elastic kernels: the tensor
// map of one time level, the ring slots' completion barriers, issue and
// bounded wait; shared by the fused kernel (engine.cu) and the paired
// interior kernel (pair.cu).  Also the host entry points of pair.cu.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "fused.cuh"

namespace fwi {

// Tensor map of one time level for the fused kernel's plane copies: 5-D
// (z, x, y, component, shot) over the [shot][component][y][x][z] layout, box
// ZW x XW x 1 x 3 x 1 = one ring slot; out-of-grid positions read as zeros.
struct FusedTma {
    CUtensorMap u;
    int *err;  // set to 1 when a wait for a copy gave up
    int on;
};

__device__ __forceinline__ unsigned fz_saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void fz_bar_init(FusedCtx &c)
{
    for (int k = 0; k < 8; k++)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(fz_saddr(&c.sm->bar[k])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// One thread: copy plane q (three components, tile window with halo) into
// ring slot `slot`; completion is signalled on the slot's barrier.
__device__ __forceinline__ void fz_tma_issue(const FusedCtx &c, int q, int slot)
{
    const unsigned bar = fz_saddr(&c.sm->bar[slot]);
    // order the block's earlier shared-memory accesses of the slot before the copy
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(FZ_PLANE_BYTES)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];\n" ::"r"(fz_saddr(&c.sm->u[slot][0][0][0])),
        "l"(c.tmap), "r"(c.z0 - fz::HW), "r"(c.x0 - fz::HW), "r"(q), "r"(0), "r"(c.shot), "r"(bar)
        : "memory");
}

// Every thread: wait for the copy into `slot`.  The wait gives up after two
// seconds (the copy takes microseconds), sets the error flag that the host
// reads at its next synchronisation, and later waits of this thread return
// at once, so that the kernel always ends.
__device__ __forceinline__ void fz_tma_wait(FusedCtx &c, int slot)
{
    const unsigned bar = fz_saddr(&c.sm->bar[slot]);
    const unsigned parity = (c.ph >> slot) & 1u;
    c.ph ^= 1u << slot;
    if (c.dead) return;
    unsigned long long t0 = 0;
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return;
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t0 == 0) {
            t0 = t;
        } else if (t - t0 > 2000000000ull) {
            atomicOr(c.err, 1);
            c.dead = true;
            return;
        }
    }
}

// pair.cu: uploads its copy of the SBP tables to the current device and sets
// the kernels' shared-memory limit (once per engine, device current).
cudaError_t pair_init();
// Launches the paired isotropic kernel (pair.cuh).  mode 1: the interior
// tiles (grid: interior z tiles, interior x tiles, chunks x shots; tile
// indices offset by (bz0, bx0)); modes 3, 4, 5: the edge tiles touching an x
// face only, a z face only, both (grid: every tile, chunks x shots).  even:
// nz is even (8-byte global pair accesses).
void pair_launch(bool even, int mode, dim3 grid, size_t smem, cudaStream_t s, const StepArgs &a, int nchunks,
                 const FusedTma &t, int bz0, int bx0);

}  // namespace fwi
