// closure.cu -- kernels of the learned subgrid closure (no counterpart in the
// reference): a 3-layer 3-D convolutional network on the coarse grid, BF16
// weights and activations, FP32 accumulation.
//
// Activations are channels-last BF16 arrays [z][y][x][C] over the coarse
// interior, periodic in x and y, zero outside in z.  A 3x3x3 convolution is an
// implicit GEMM: D[m][n] = sum_k A[m][k] B[n][k], m = 128 consecutive x points
// of one (y, z) row, n = output channel, k = tap*CIN + input channel.
//
//  - k_conv3d (forward, and the input gradient with transposed, flipped
//    weights): tcgen05.mma (kind::f16, BF16 in, FP32 accumulator in TMEM,
//    M=128, N=COUT, K=16 per instruction) issued by one thread.  The input
//    block of a row (130 x 3 x 3 voxels) sits in shared memory as
//    [8-channel chunk][voxel] 16-byte rows, which is the canonical K-major
//    no-swizzle layout with 8-row groups 128 bytes apart: the A operand of
//    tap (dx,dy,dz) is the same descriptor moved by whole 16-byte rows.  The
//    weights stay in shared memory in the same canonical layout for all rows
//    of the persistent CTA.  The accumulator is read back with tcgen05.ld;
//    the epilogue adds the bias, applies ReLU or the ReLU mask of the layer
//    below, and writes BF16 (and FP32) outputs.  A CTA walks a contiguous run
//    of rows along y and keeps a ring of four y rows (each with its z
//    neighbours): a tile loads one new row, by cp.async, while the previous
//    tile's MMAs run, and the taps address the ring's slots.
//  - k_conv3d_wgrad: dW[n][tap*CIN+ci] = sum over voxels of dY[v][n] *
//    X[v+tap][ci], an FP32 CUDA-core reduction (its M = COUT is below the
//    64 rows of a tcgen05 instruction and its K runs over all voxels).
//
// Every wait is bounded; a CTA that gives up records an error and releases
// its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mhd3d.h"
#include "ring.cuh"

namespace mhd3d {
namespace clo {

constexpr int CT = 128;            // threads of a convolution CTA (4 warps: TMEM lanes 0..127)
constexpr int MT = 128;            // output voxels per tile: one 128-point x segment
constexpr int BX = MT + 2;         // input block: x with halo
constexpr int VB = BX * 3 * 3;     // voxels of the input block (y, z halos)

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor, no swizzle: start address, leading
// (K-direction) and stride (8-row group) byte offsets, SM100 version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[N]);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Issue the asynchronous copies of the input block of tile (x0, y, z) into sx:
// [chunk][voxel] 16-byte rows, periodic in x and y, zeros outside in z (a
// zero-byte source fills zeros).  The caller commits and waits for the group.
template <int CIN, int NTH>
__device__ __forceinline__ void load_block_async(unsigned char* sx, const __nv_bfloat16* __restrict__ x, int x0,
                                                 int y, int z, int nx, int ny, int nz)
{
    constexpr int NC = CIN / 8;
    const uint32_t sbase = smem_u32(sx);
    for (int q = threadIdx.x; q < VB * NC; q += NTH) {
        const int c = q / VB, v = q % VB;
        const int xi = v % BX, yi = (v / BX) % 3, zi = v / (BX * 3);
        int gx = x0 - 1 + xi;
        if (nx >= MT) gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
        else gx = (gx + nx) % nx;   // a 128-point tile spans 128/nx periods
        int gy = y - 1 + yi;
        gy = gy < 0 ? gy + ny : (gy >= ny ? gy - ny : gy);
        int gz = z - 1 + zi;
        const uint32_t nbytes = (gz >= 0 && gz < nz) ? 16u : 0u;
        gz = gz < 0 ? 0 : (gz >= nz ? nz - 1 : gz);
        const __nv_bfloat16* src = x + (((size_t)gz * ny + gy) * nx + gx) * CIN + c * 8;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sbase + (uint32_t)((c * VB + v) * 16)),
                     "l"(src), "r"(nbytes)
                     : "memory");
    }
}
// Ring of y rows for the convolution: [chunk][slot 0..3][z plane 0..2][BX voxels]
// of 16-byte rows; row yr (unwrapped) lives in slot yr & 3.
constexpr int RSEG = 4 * 3 * BX;   // voxel rows of one chunk of the ring
template <int CIN, int NTH>
__device__ __forceinline__ void load_row_async(unsigned char* ring, const __nv_bfloat16* __restrict__ x, int x0,
                                               int yr, int z, int nx, int ny, int nz)
{
    constexpr int NC = CIN / 8;
    const int slot = yr & 3;
    int gy = yr % ny;
    gy = gy < 0 ? gy + ny : gy;
    const uint32_t sbase = smem_u32(ring);
    for (int q = threadIdx.x; q < 3 * BX * NC; q += NTH) {
        const int c = q / (3 * BX), r = q % (3 * BX);
        const int zi = r / BX, xi = r % BX;
        int gx = x0 - 1 + xi;
        if (nx >= MT) gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
        else gx = (gx + nx) % nx;   // a 128-point tile spans 128/nx periods
        int gz = z - 1 + zi;
        const uint32_t nbytes = (gz >= 0 && gz < nz) ? 16u : 0u;
        gz = gz < 0 ? 0 : (gz >= nz ? nz - 1 : gz);
        const __nv_bfloat16* src = x + (((size_t)gz * ny + gy) * nx + gx) * CIN + c * 8;
        const uint32_t dst = sbase + (uint32_t)((c * RSEG + (slot * 3 + zi) * BX + xi) * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int CIN, int COUT>
struct ConvLay {
    static constexpr int K = 27 * CIN;
    static constexpr size_t W_B = (size_t)COUT * K * 2;
    static constexpr size_t X_OFF = (W_B + 127) / 128 * 128;
    static constexpr size_t X_B = ((size_t)CIN * RSEG * 2 + 127) / 128 * 128;  // ring of four y rows
    static constexpr size_t BAR_OFF = X_OFF + X_B;
    static constexpr size_t BYTES = BAR_OFF + 16 + 128;
};

// Y = act(conv(X, W) + bias) [* (mask > 0)], persistent over (x segment, y, z) tiles.
// w: [COUT][27*CIN] BF16, k = tap*CIN + ci with tap = dx+1 + 3*(dy+1) + 9*(dz+1).
template <int CIN, int COUT>
__global__ void __launch_bounds__(CT, 1) k_conv3d(const __nv_bfloat16* __restrict__ x,
                                                  const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
                                                  const __nv_bfloat16* __restrict__ mask, int relu,
                                                  __nv_bfloat16* __restrict__ y, float* __restrict__ yf, int nx, int ny,
                                                  int nz, int* err)
{
    using L = ConvLay<CIN, COUT>;
    constexpr int K = L::K;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    unsigned char* const sw = sb;
    unsigned char* const sx = sb + L::X_OFF;
    unsigned long long* const bar = reinterpret_cast<unsigned long long*>(sb + L::BAR_OFF);
    uint32_t* const tslot = reinterpret_cast<uint32_t*>(sb + L::BAR_OFF + 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // weights -> canonical K-major layout: (n, k) at ((n/8)*(K/8) + k/8)*128 + (n%8)*16 + (k%8)*2
    for (int q = tid; q < COUT * (K / 8); q += CT) {
        const int n = q / (K / 8), kc = q % (K / 8);
        const uint4 v = *reinterpret_cast<const uint4*>(w + (size_t)n * K + kc * 8);
        *reinterpret_cast<uint4*>(sw + ((size_t)(n >> 3) * (K / 8) + kc) * 128 + (n & 7) * 16) = v;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(32u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // tiles in (segment, z, y) order with y fastest; each CTA takes one
    // contiguous run, so consecutive tiles share two of their three y rows
    const int nseg = (nx + MT - 1) / MT;
    const int ntile = nseg * ny * nz;
    constexpr uint32_t IDESC = idesc_bf16(MT, COUT);
    const uint32_t sw_a = smem_u32(sw), sx_a = smem_u32(sx);
    const int t_begin = (int)(((long)ntile * blockIdx.x) / gridDim.x);
    const int t_end = (int)(((long)ntile * (blockIdx.x + 1)) / gridDim.x);
    auto tile_of = [&](int t, int& x0, int& yy, int& zz) {
        yy = t % ny;
        zz = (t / ny) % nz;
        x0 = (t / (ny * nz)) * MT;
    };
    unsigned phase = 0;
    bool failed = false;
    for (int t = t_begin; t < t_end && !failed; ++t) {
        int x0, yy, zz;
        tile_of(t, x0, yy, zz);
        const bool fresh = t == t_begin || yy == 0;   // a new (segment, z) run: rows y-1, y, y+1
        if (fresh) {
            for (int d = -1; d <= 1; ++d) load_row_async<CIN, CT>(sx, x, x0, yy + d, zz, nx, ny, nz);
            cp_async_commit();
        }
        // the next tile's new row streams in while this tile is multiplied
        if (t + 1 < t_end && yy + 1 < ny) load_row_async<CIN, CT>(sx, x, x0, yy + 2, zz, nx, ny, nz);
        cp_async_commit();
        cp_async_wait<1>();
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            for (int tap = 0; tap < 27; ++tap) {
                const int dxi = tap % 3, dyi = (tap / 3) % 3, dzi = tap / 9;
                const int row = ((((yy + dyi - 1) & 3) * 3 + dzi) * BX + dxi);
#pragma unroll
                for (int kk = 0; kk < CIN / 16; ++kk) {
                    const uint64_t da = smem_desc(sx_a + (uint32_t)((2 * kk) * RSEG + row) * 16u, RSEG * 16, 128);
                    const uint64_t db = smem_desc(sw_a + (uint32_t)((tap * CIN + kk * 16) >> 3) * 128u, 128,
                                                  (K / 8) * 128);
                    umma_bf16(tmem, da, db, IDESC, (tap | kk) != 0 ? 1u : 0u);
                }
            }
            umma_commit(bar);
        }
        if (!mbar_wait(bar, phase)) {
            failed = true;
            if (tid == 0) atomicExch(err, 1);
        }
        phase ^= 1u;
        tc_fence_after();
        if (!failed) {
            float acc[COUT];
            tmem_ld<COUT>(tmem + ((uint32_t)(warp * 32) << 16), acc);
            const int m = warp * 32 + lane;
            const bool own = x0 + m < nx;   // for nx < 128 the tile repeats the row's period
            const size_t vox = ((size_t)zz * ny + yy) * nx + (own ? x0 + m : 0);
#pragma unroll
            for (int n = 0; n < COUT; ++n) {
                float o = acc[n] + (bias ? bias[n] : 0.f);
                if (relu) o = o > 0.f ? o : 0.f;
                if (mask && !(__bfloat162float(mask[vox * COUT + n]) > 0.f)) o = 0.f;
                acc[n] = o;
            }
            if (y && own) {
#pragma unroll
                for (int n = 0; n < COUT; n += 8) {
                    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16_rn(acc[n + i]);
                    *reinterpret_cast<uint4*>(y + vox * COUT + n) = *reinterpret_cast<const uint4*>(h);
                }
            }
            if (yf && own) {
#pragma unroll
                for (int n = 0; n < COUT; n += 4)
                    *reinterpret_cast<float4*>(yf + vox * COUT + n) =
                        make_float4(acc[n], acc[n + 1], acc[n + 2], acc[n + 3]);
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    cp_async_wait<0>();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u));
}

// dW[n][tap*CIN+ci] += sum_v dY[v][n] * X[v+tap][ci], db[n] += sum_v dY[v][n].
// Thread t owns output channel n = t/(CIN/4) and input channels 4*(t%(CIN/4))..+3.
template <int CIN, int COUT>
__global__ void __launch_bounds__(COUT * CIN / 4) k_conv3d_wgrad(const __nv_bfloat16* __restrict__ x,
                                                                const __nv_bfloat16* __restrict__ dy,
                                                                float* __restrict__ dw, float* __restrict__ db, int nx,
                                                                int ny, int nz)
{
    constexpr int NTH = COUT * CIN / 4;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* const sx = smem_raw;                              // CIN/8 x VB x 16 B
    float* const sdy = reinterpret_cast<float*>(smem_raw + (size_t)CIN * VB * 2);   // MT x COUT
    const int tid = threadIdx.x;
    const int n = tid / (CIN / 4), c4 = tid % (CIN / 4);
    float acc[27][4];
#pragma unroll
    for (int t = 0; t < 27; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
    float bacc = 0.f;
    const int nseg = (nx + MT - 1) / MT;
    const int ntile = nseg * ny * nz;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
        const int seg = t % nseg, yy = (t / nseg) % ny, zz = t / (nseg * ny);
        const int x0 = seg * MT;
        __syncthreads();
        load_block_async<CIN, NTH>(sx, x, x0, yy, zz, nx, ny, nz);
        cp_async_commit();
        const size_t row = ((size_t)zz * ny + yy) * nx + x0;
        const int mlim = nx - x0 < MT ? nx - x0 : MT;   // voxels of this tile that are the row's own
        for (int q = threadIdx.x; q < mlim * COUT; q += NTH) sdy[q] = __bfloat162float(dy[row * COUT + q]);
        cp_async_wait<0>();
        __syncthreads();
        // channels 4*c4..4*c4+3 live in chunk c4/2, halves (c4%2)
        const unsigned char* xb = sx + (size_t)(c4 >> 1) * VB * 16 + (c4 & 1) * 8;
        for (int m = 0; m < mlim; ++m) {
            const float g = sdy[m * COUT + n];
            bacc += g;
#pragma unroll
            for (int tap = 0; tap < 27; ++tap) {
                const int v = m + (tap % 3) + BX * ((tap / 3) % 3) + BX * 3 * (tap / 9);
                const uint2 p = *reinterpret_cast<const uint2*>(xb + (size_t)v * 16);
                const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&p.x);
                const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&p.y);
                const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
                acc[tap][0] += g * fa.x;
                acc[tap][1] += g * fa.y;
                acc[tap][2] += g * fb.x;
                acc[tap][3] += g * fb.y;
            }
        }
    }
    constexpr int K = 27 * CIN;
#pragma unroll
    for (int tap = 0; tap < 27; ++tap)
#pragma unroll
        for (int i = 0; i < 4; ++i) atomicAdd(&dw[(size_t)n * K + tap * CIN + 4 * c4 + i], acc[tap][i]);
    if (c4 == 0 && db) atomicAdd(&db[n], bacc);
}

// W[n][tap*CIN+ci] -> Wt[ci][(26-tap)*COUT+n]: the input-gradient convolution
__global__ void k_wtranspose(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt, int cin, int cout)
{
    const int K = 27 * cin;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cout * K; q += gridDim.x * blockDim.x) {
        const int n = q / K, k = q % K, tap = k / cin, ci = k % cin;
        wt[(size_t)ci * (27 * cout) + (26 - tap) * cout + n] = w[q];
    }
}

template <int CIN, int COUT>
cudaError_t launch_conv_t(const void* x, const void* w, const float* bias, const void* mask, int relu, void* y,
                          float* yf, int nx, int ny, int nz, int* err, cudaStream_t st)
{
    using L = ConvLay<CIN, COUT>;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_conv3d<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)L::BYTES);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntile = ((nx + MT - 1) / MT) * ny * nz;
    const int grid = ntile < sms ? ntile : sms;
    k_conv3d<CIN, COUT><<<grid, CT, L::BYTES, st>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), bias,
        static_cast<const __nv_bfloat16*>(mask), relu, static_cast<__nv_bfloat16*>(y), yf, nx, ny, nz, err);
    return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t launch_wgrad_t(const void* x, const void* dy, float* dw, float* db, int nx, int ny, int nz, cudaStream_t st)
{
    const size_t smem = (size_t)CIN * VB * 2 + (size_t)MT * COUT * 4;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_conv3d_wgrad<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntile = ((nx + MT - 1) / MT) * ny * nz;
    const int grid = ntile < 2 * sms ? ntile : 2 * sms;
    k_conv3d_wgrad<CIN, COUT><<<grid, COUT * CIN / 4, smem, st>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), dw, db, nx, ny, nz);
    return cudaGetLastError();
}

}  // namespace clo
}  // namespace mhd3d

using namespace mhd3d::clo;

extern "C" {

int mhd3d_conv3d(int32_t cin, int32_t cout, const void* x, const void* w, const float* bias, const void* mask,
                 int32_t relu, void* y, float* yf, int32_t nx, int32_t ny, int32_t nz, int32_t* err, void* stream)
{
    if (!x || !w || !err || nx <= 0 || (nx % MT && MT % nx) || ny <= 0 || nz <= 0 || (!y && !yf))
        return MHD3D_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (cin == 16 && cout == 32) e = launch_conv_t<16, 32>(x, w, bias, mask, relu, y, yf, nx, ny, nz, err, st);
    else if (cin == 32 && cout == 32) e = launch_conv_t<32, 32>(x, w, bias, mask, relu, y, yf, nx, ny, nz, err, st);
    else if (cin == 32 && cout == 16) e = launch_conv_t<32, 16>(x, w, bias, mask, relu, y, yf, nx, ny, nz, err, st);
    else return MHD3D_ERR_ARG;
    return e == cudaSuccess ? MHD3D_OK : MHD3D_ERR_CUDA;
}

int mhd3d_conv3d_wgrad(int32_t cin, int32_t cout, const void* x, const void* dy, float* dw, float* db, int32_t nx,
                       int32_t ny, int32_t nz, void* stream)
{
    if (!x || !dy || !dw || nx <= 0 || (nx % MT && MT % nx) || ny <= 0 || nz <= 0) return MHD3D_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (cin == 16 && cout == 32) e = launch_wgrad_t<16, 32>(x, dy, dw, db, nx, ny, nz, st);
    else if (cin == 32 && cout == 32) e = launch_wgrad_t<32, 32>(x, dy, dw, db, nx, ny, nz, st);
    else if (cin == 32 && cout == 16) e = launch_wgrad_t<32, 16>(x, dy, dw, db, nx, ny, nz, st);
    else return MHD3D_ERR_ARG;
    return e == cudaSuccess ? MHD3D_OK : MHD3D_ERR_CUDA;
}

int mhd3d_conv3d_wtranspose(int32_t cin, int32_t cout, const void* w, void* wt, void* stream)
{
    if (!w || !wt || cin <= 0 || cout <= 0) return MHD3D_ERR_ARG;
    k_wtranspose<<<64, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(w),
                                                                  static_cast<__nv_bfloat16*>(wt), cin, cout);
    return cudaGetLastError() == cudaSuccess ? MHD3D_OK : MHD3D_ERR_CUDA;
}

}  // extern "C"
