// ring.cuh -- pieces shared by the stage kernels of every precision: the
// TMA/mbarrier primitives of the shared-memory plane ring (bounded waits) and
// the store of a cell together with its periodic halo copies.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace mhd3d {

constexpr long WAIT_LIMIT = 1L << 22;   // bounded mbarrier polls (~seconds)

// ---- TMA and mbarrier primitives (PTX) ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned cnt)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(cnt) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase with the given parity; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long limit = WAIT_LIMIT)
{
    for (long it = 0; it < limit; ++it) {
        if (mbar_test(bar, parity)) return true;
        if (it > 32) __nanosleep(128);
    }
    return false;
}
__device__ __forceinline__ void tma_load4(void* dst, const CUtensorMap* map, unsigned long long* bar, int x, int y,
                                          int z, int f)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(f),
          "r"(smem_u32(bar))
        : "memory");
}

// Periodic halo copies of one interior column: plane offsets of the copies
// COMMUNICATE makes at I=1/NX and J=1/NY, formed once per thread.
struct HaloCols {
    int hx, hy, hxy;   // x copy, y copy, corner copy
    bool ex, ey;
};
__device__ __forceinline__ HaloCols halo_cols(int npx, int npy, int upitch, int gi, int gj)
{
    const int cx = (gi == 0) ? npx + 1 : (gi == npx - 1) ? 0 : -1;
    const int cy = (gj == 0) ? npy + 1 : (gj == npy - 1) ? 0 : -1;
    HaloCols h;
    h.ex = cx >= 0;
    h.ey = cy >= 0;
    h.hx = (gj + 1) * upitch + cx;
    h.hy = cy * upitch + (gi + 1);
    h.hxy = cy * upitch + cx;
    return h;
}

// store N fields of one cell of U (pl: the plane's base) and their halo
// copies; the copies are one branch for the columns that have none
template <int N, typename T>
__device__ __forceinline__ void store_cell(T* __restrict__ pl, size_t uf, size_t ucol, const HaloCols& h,
                                           const int (&f)[N], const T (&v)[N])
{
#pragma unroll
    for (int i = 0; i < N; ++i) pl[(size_t)f[i] * uf + ucol] = v[i];
    if (h.ex || h.ey) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            T* q = pl + (size_t)f[i] * uf;
            if (h.ex) q[h.hx] = v[i];
            if (h.ey) q[h.hy] = v[i];
            if (h.ex && h.ey) q[h.hxy] = v[i];
        }
    }
}

}  // namespace mhd3d
