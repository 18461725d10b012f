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
//    weights): tcgen05.mma (kind::f16, BF16 in, FP32 accumulators in TMEM,
//    M=128, K=16 per instruction) issued by one thread.  Input rows (130 x
//    3 z planes) sit in a shared-memory ring, so the A operand of tap
//    (dx, dz) is one descriptor moved by whole voxel rows: with 32 input
//    channels and x a multiple of 128, 64-byte voxel rows in the copy
//    engine's 64-byte swizzle (one TMA box per plane); otherwise
//    [8-channel chunk][voxel] 16-byte rows, the canonical K-major no-swizzle
//    layout with 8-row groups 128 bytes apart.  Any nx: a tile that runs past
//    the row's end reads the row again from its start (periodic), and only
//    its first nx - x0 outputs are stored (for nx < 128 the tile holds the
//    row's period more than once).  One MMA serves three output rows (N = 3*COUT,
//    the y taps stacked in the B operand), see k_conv3d.  Warp roles: a
//    loader (TMA boxes, or cp.async when nx is not a multiple of 128), one
//    MMA thread and four epilogue warps, handing off through mbarriers.  The
//    epilogue adds the bias, applies ReLU or the ReLU mask of the layer
//    below, and writes BF16 (and FP32) outputs.
//  - k_conv3d_wgrad_tc: dW[n][tap*CIN+ci] = sum over voxels of dY[v][n] *
//    X[v+tap][ci] on tcgen05 as well, with K running over voxels: per x
//    segment the shifted dY rows form A (M = 3*COUT, the x taps) and the
//    input rows of the y taps form B (N = 3*CIN, the z taps), both staged
//    K-major by the CTA's threads; per-CTA partials are added in CTA order
//    by k_wgrad_reduce.
//
// Every wait is bounded; a CTA that gives up records an error and releases
// its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/mhd3d.h"
#include "ring.cuh"
#include "smem_attr.cuh"

namespace mhd3d {
namespace clo {

constexpr int NLW = 4;             // loader warps of a convolution CTA
constexpr int CT = 32 * (4 + NLW + 1);   // threads: 4 epilogue warps (TMEM lanes 0..127), loaders, MMA
constexpr int RING = 4;            // input rows held in the ring: the loaders run up to three steps ahead
constexpr int MT = 128;            // output voxels per tile: one 128-point x segment
constexpr int BX = MT + 2;         // input block: x with halo

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

// Ring of input rows for the convolution: [chunk][slot 0..RING-1][z plane 0..2]
// [BXP] of 16-byte rows (or, in the swizzled form, [slot][z plane][BXP] of
// 64-byte rows), voxel xi (x0-1+xi) at row XR0+xi, so that the 128 interior
// voxels start on a 128-byte (512-byte) boundary, a TMA destination; step s
// of a CTA keeps its input row in slot s % RING.
constexpr int XR0 = 7;
constexpr int BXP = 144;              // XR0 + BX rounded up to 8 rows
constexpr int RSEG = RING * 3 * BXP;  // voxel rows of one chunk of the ring
template <int CIN, int NTH>
__device__ __forceinline__ void load_row_async(unsigned char* ring, const __nv_bfloat16* __restrict__ x, int x0,
                                               int yr, int z, int nx, int ny, int nz, int tix, int slot)
{
    constexpr int NC = CIN / 8;
    int gy = yr % ny;
    gy = gy < 0 ? gy + ny : gy;
    const uint32_t sbase = smem_u32(ring);
    for (int q = tix; q < 3 * BX * NC; q += NTH) {
        const int c = q / (3 * BX), r = q % (3 * BX);
        const int zi = r / BX, xi = r % BX;
        int gx = x0 - 1 + xi;
        if (nx >= MT) gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
        else gx = (gx + nx) % nx;   // a 128-point tile spans 128/nx periods
        int gz = z - 1 + zi;
        const uint32_t nbytes = (gz >= 0 && gz < nz) ? 16u : 0u;
        gz = gz < 0 ? 0 : (gz >= nz ? nz - 1 : gz);
        const __nv_bfloat16* src = x + (((size_t)gz * ny + gy) * nx + gx) * CIN + c * 8;
        const uint32_t dst = sbase + (uint32_t)((c * RSEG + (slot * 3 + zi) * BXP + XR0 + xi) * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The input row of a step by TMA (x segments of 128 voxels, nx a multiple of
// 128): one 5-D box (8 channels, 1 chunk, 128 x, 1 y, 1 z) per chunk and z
// plane into the ring's interior rows, zeros outside z (out-of-range box);
// the two periodic x halo voxels by cp.async from the calling warp.  The
// TMA bytes complete on bar (after the caller's expect_tx); each lane's
// copies are signalled by the caller's cp.async.mbarrier.arrive.
template <int CIN>
__device__ __forceinline__ void load_row_tma(unsigned char* ring, const CUtensorMap* map, unsigned long long* bar,
                                             const __nv_bfloat16* __restrict__ x, int x0, int yr, int z, int nx,
                                             int ny, int nz, int lane, int slot)
{
    constexpr int NC = CIN / 8;
    int gy = yr % ny;
    gy = gy < 0 ? gy + ny : gy;
    const uint32_t sbase = smem_u32(ring);
    if (lane == 0) {
        for (int c = 0; c < NC; ++c)
            for (int zi = 0; zi < 3; ++zi) {
                const uint32_t dst = sbase + (uint32_t)((c * RSEG + (slot * 3 + zi) * BXP + XR0 + 1) * 16);
                asm volatile(
                    "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                    "%3, %4, %5, %6}], [%7];" ::"r"(dst),
                    "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(c), "r"(x0), "r"(gy), "r"(z - 1 + zi),
                    "r"(smem_u32(bar))
                    : "memory");
            }
    }
    for (int q = lane; q < 2 * NC * 3; q += 32) {
        const int side = q & 1, c = (q >> 1) % NC, zi = (q >> 1) / NC;
        const int xi = side ? BX - 1 : 0;
        int gx = x0 - 1 + xi;
        gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
        int gz = z - 1 + zi;
        const uint32_t nbytes = (gz >= 0 && gz < nz) ? 16u : 0u;
        gz = gz < 0 ? 0 : (gz >= nz ? nz - 1 : gz);
        const __nv_bfloat16* src = x + (((size_t)gz * ny + gy) * nx + gx) * CIN + c * 8;
        const uint32_t dst = sbase + (uint32_t)((c * RSEG + (slot * 3 + zi) * BXP + XR0 + xi) * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
    }
}

// The input row of a step by TMA for 32 input channels, in the 64-byte
// swizzled K-major layout: plane p = slot*3 + zi of the ring is BXP voxel
// rows of 64 bytes (all 32 channels) from byte p*BXP*64, and the 16-byte
// chunk j (channels 8j..8j+7) of row R sits at chunk position j ^ ((R >> 1) & 3)
// -- the copy engine's SWIZZLE_64B pattern (address bits 4-5 XOR bits 7-8,
// planes 512-byte aligned), which SWIZZLE_64B matrix descriptors read back.
// One 4-D box (32 channels, 128 x, 1 y, 1 z) per plane lands the interior at
// row XR0+1; the two periodic halo voxels come by cp.async, placed by the
// same rule.
__device__ __forceinline__ void load_row_tma_sw64(unsigned char* ring, const CUtensorMap* map,
                                                  unsigned long long* bar, const __nv_bfloat16* __restrict__ x,
                                                  int x0, int yr, int z, int nx, int ny, int nz, int lane, int slot)
{
    constexpr int CIN = 32;
    int gy = yr % ny;
    gy = gy < 0 ? gy + ny : gy;
    const uint32_t sbase = smem_u32(ring);
    if (lane == 0) {
        for (int zi = 0; zi < 3; ++zi) {
            const uint32_t dst = sbase + (uint32_t)(((slot * 3 + zi) * BXP + XR0 + 1) * 64);
            asm volatile(
                "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                "%3, %4, %5}], [%6];" ::"r"(dst),
                "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(x0), "r"(gy), "r"(z - 1 + zi),
                "r"(smem_u32(bar))
                : "memory");
        }
    }
    if (lane < 24) {
        const int side = lane & 1, j = (lane >> 1) & 3, zi = lane >> 3;
        const int xi = side ? BX - 1 : 0;
        int gx = x0 - 1 + xi;
        gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
        int gz = z - 1 + zi;
        const uint32_t nbytes = (gz >= 0 && gz < nz) ? 16u : 0u;
        gz = gz < 0 ? 0 : (gz >= nz ? nz - 1 : gz);
        const __nv_bfloat16* src = x + (((size_t)gz * ny + gy) * nx + gx) * CIN + j * 8;
        const int R = XR0 + xi;
        const uint32_t dst = sbase + (uint32_t)(((slot * 3 + zi) * BXP + R) * 64 + ((j ^ ((R >> 1) & 3)) * 16));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
    }
}

// shared-memory matrix descriptor of a K-major operand in the 64-byte swizzled
// layout: 64-byte rows, 8-row groups 512 bytes apart (the leading offset is
// unused when the K of one MMA lies inside a row), SM100 version 1, base
// offset 0.  The pattern follows the absolute address bits, so a start moved
// by whole rows (an x tap) or by 32 bytes inside a row (the second K half)
// reads the rows the copy engine wrote there (checked against the numpy
// convolution by the GPU parity tests).
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t saddr)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(512 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// bounded wait without sleeping between polls: mbarrier.try_wait itself
// suspends the thread for a while, and the pipeline's hand-offs between warp
// roles are on the critical path; false when it gave up
__device__ __forceinline__ bool mbar_wait_fast(unsigned long long* bar, unsigned parity)
{
    for (long it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_test(bar, parity)) return true;
    return false;
}

template <int N>
__device__ __forceinline__ void tmem_st_zero(uint32_t taddr);

template <>
__device__ __forceinline__ void tmem_st_zero<16>(uint32_t taddr)
{
    const uint32_t z = 0;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};\n" ::"r"(taddr),
        "r"(z)
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

template <>
__device__ __forceinline__ void tmem_st_zero<32>(uint32_t taddr)
{
    const uint32_t z = 0;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
        "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};\n" ::"r"(taddr),
        "r"(z)
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// The steps of a CTA: its range of output rows forms runs along y within one
// (x segment, z) column; a run of output rows ya..yb takes input rows
// ya-1..yb+1, one step each.  f(s, x0, z, r, first, emit) for every step s in
// order: r the unwrapped input row, first the run's first step, emit whether
// output row r-1 is in the run; f returns false to stop.
template <class F>
__device__ __forceinline__ void for_steps(int t_begin, int t_end, int ny, int nz, F f)
{
    int s = 0;
    for (int t = t_begin; t < t_end;) {
        const int ya = t % ny, z = (t / ny) % nz, x0 = (t / (ny * nz)) * MT;
        const int run = (t_end - t) < (ny - ya) ? (t_end - t) : (ny - ya);
        const int yb = ya + run - 1;
        for (int r = ya - 1; r <= yb + 1; ++r, ++s)
            if (!f(s, x0, z, r, r == ya - 1, r - 1 >= ya && r - 1 <= yb)) return;
        t += run;
    }
}

template <int CIN, int COUT>
struct ConvLay {
    static constexpr int K = 27 * CIN;
    static constexpr int KB = 9 * CIN;          // K of one y-tap block: (dz, dx, ci)
    static constexpr int NW = 3 * COUT;         // N of an MMA: three output rows
    static constexpr uint32_t NCOL = NW <= 32 ? 32 : NW <= 64 ? 64 : 128;   // TMEM: three accumulator slots
    static constexpr size_t W_B = (size_t)5 * COUT * KB * 2;   // y-tap blocks 2, 1, 0, 2, 1
    static constexpr size_t X_OFF = (W_B + 1023) / 1024 * 1024;   // the ring's planes 512-byte aligned
    static constexpr size_t X_B = ((size_t)CIN * RSEG * 2 + 127) / 128 * 128;  // ring of RING input rows
    static constexpr size_t BAR_OFF = X_OFF + X_B;
    // barriers: ready[4], mmadone[4], accfull, accempty; then the TMEM
    // address, the abort flag and the last committed step
    static constexpr size_t BYTES = BAR_OFF + 10 * 8 + 16 + 1024;   // + alignment of the base to 1024 bytes
};

// Y = act(conv(X, W) + bias) [* (mask > 0)], persistent over (x segment, y, z) tiles.
// w: [COUT][27*CIN] BF16, k = tap*CIN + ci with tap = dx+1 + 3*(dy+1) + 9*(dz+1).
//
// One MMA serves three output rows: an input row r (one of the CTA's steps)
// contributes to output rows r+1, r, r-1 through the weights of y-taps 0, 1,
// 2.  Three accumulators of COUT columns sit side by side in TMEM, output row
// y in slot y mod 3, and the B operand stacks the y-tap blocks in the slot
// order, which rotates with r mod 3: the weights are kept as the y-tap blocks
// 2, 1, 0, 2, 1 and each step reads the window of three starting at
// (1 - r) mod 3.  Per input row the MMAs are 9 * CIN/16 of N = 3*COUT
// (instead of 27 * CIN/16 of N = COUT per output row), so each input tile
// is read from shared memory a third as often.  After step r, output row r-1
// is complete: the epilogue reads its slot, zeroes it for output row r+2 and
// stores.  The first MMA of a run starts all three slots from zero.
//
// Warp roles, pipelined over the CTA's steps s (ready and mmadone by s & 3):
//   loaders: the step's input row (three z planes, periodic in x and y,
//     zeros outside z) into ring slot s % RING.  With use_tma (nx a multiple
//     of 128) warp 4 alone: one TMA box per z plane of 32 channels x 128
//     voxels in 64-byte swizzled rows (CIN = 32), or of 8 channels x 128
//     voxels per chunk and plane (CIN = 16), complete_tx on ready(s), and
//     the two x-halo voxels by cp.async; otherwise warps 4..4+NLW-1 by
//     cp.async.  Each loader thread's
//     copies arrive on ready(s) as they land (cp.async.mbarrier.arrive), and a
//     slot is reused once the MMAs of step s - RING have completed (mmadone).
//   warp 4+NLW, lane 0 (MMA): waits ready(s) and the release of step s-1's
//     finished slot (accempty), issues the step's MMAs, commits to accfull
//     and to mmadone(s).
//   warps 0-3 (epilogue): wait accfull(s), read and zero the finished slot
//     (TMEM lanes 32*warp..), release it (accempty) and store while the next
//     step's MMAs run.
template <int CIN, int COUT>
__global__ void __launch_bounds__(CT, 1) k_conv3d(const __grid_constant__ CUtensorMap xmap, int use_tma,
                                                  const __nv_bfloat16* __restrict__ x,
                                                  const __nv_bfloat16* __restrict__ w, const float* __restrict__ bias,
                                                  const __nv_bfloat16* __restrict__ mask, int relu,
                                                  __nv_bfloat16* __restrict__ y, float* __restrict__ yf, int nx, int ny,
                                                  int nz, int* err)
{
    using L = ConvLay<CIN, COUT>;
    constexpr int K = L::K, KB = L::KB;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* const sb = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    unsigned char* const sw = sb;
    unsigned char* const sx = sb + L::X_OFF;
    unsigned long long* const bars = reinterpret_cast<unsigned long long*>(sb + L::BAR_OFF);
    unsigned long long* const ready = bars;
    unsigned long long* const mmadone = bars + 4;
    unsigned long long* const accfull = bars + 8;
    unsigned long long* const accempty = bars + 9;
    uint32_t* const tslot = reinterpret_cast<uint32_t*>(sb + L::BAR_OFF + 80);
    volatile int* const abort_flag = reinterpret_cast<volatile int*>(sb + L::BAR_OFF + 84);
    volatile int* const last_commit = reinterpret_cast<volatile int*>(sb + L::BAR_OFF + 88);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // weights -> y-tap blocks 2,1,0,2,1 of [COUT][KB], k' = (dz*3 + dx)*CIN + ci, in
    // the canonical K-major layout: row n', k' at ((n'/8)*(KB/8) + k'/8)*128 + (n'%8)*16 + (k'%8)*2
    {
        // eight loads in flight per thread before their stores
        constexpr int NQ = 5 * COUT * (KB / 8), BATCH = 8;
        for (int q0 = tid; q0 < NQ; q0 += CT * BATCH) {
            uint4 v[BATCH];
            int dst[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int q = q0 + u * CT;
                dst[u] = -1;
                if (q < NQ) {
                    const int blk = q / (COUT * (KB / 8)), rem = q % (COUT * (KB / 8));
                    const int n = rem / (KB / 8), kc = rem % (KB / 8);
                    const int dyi = blk == 2 ? 0 : (blk == 1 || blk == 4) ? 1 : 2;
                    const int dzdx = (kc * 8) / CIN, ci = (kc * 8) % CIN, dzi = dzdx / 3, dxi = dzdx % 3;
                    const int tap = dxi + 3 * dyi + 9 * dzi;
                    v[u] = __ldg(reinterpret_cast<const uint4*>(w + (size_t)n * K + tap * CIN + ci));
                    const int nr = blk * COUT + n;
                    dst[u] = (int)(((nr >> 3) * (KB / 8) + kc) * 128 + (nr & 7) * 16);
                }
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u)
                if (dst[u] >= 0) *reinterpret_cast<uint4*>(sw + dst[u]) = v[u];
        }
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(L::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < 4; ++b) {
            // TMA: the expect_tx arrival and one completion arrival per lane of
            // the loader warp; cp.async only: one per loader thread
            mbar_init(ready + b, use_tma ? 1 + 32 : 32 * NLW);
            mbar_init(mmadone + b, 1);
        }
        mbar_init(accfull, 1);
        mbar_init(accempty, 4);
        *abort_flag = 0;
        *last_commit = -1;
        fence_mbar_init();
    }
    fence_proxy_async();   // the weights, written by plain stores, are read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // output rows in (segment, z, y) order with y fastest; each CTA takes one
    // contiguous range, walked as runs along y
    const int nseg = (nx + MT - 1) / MT;
    const int ntile = nseg * ny * nz;
    const int t_begin = (int)(((long)ntile * blockIdx.x) / gridDim.x);
    const int t_end = (int)(((long)ntile * (blockIdx.x + 1)) / gridDim.x);
    auto give_up = [&]() {
        *abort_flag = 1;
        atomicExch(err, 1);
    };

    if (use_tma && warp == 4) {
        // one warp: the TMA boxes of the step's row and its two halo voxels
        for_steps(t_begin, t_end, ny, nz, [&](int s, int x0, int zz, int r, bool, bool) {
            if (*abort_flag) return false;
            const int jw = s - RING;   // slot s % RING was last read by step s - RING
            if (jw >= 0 && !mbar_wait_fast(mmadone + (jw & 3), (unsigned)(jw >> 2) & 1u)) {
                give_up();
                return false;
            }
            unsigned long long* const bar = ready + (s & 3);
            if (lane == 0) mbar_expect_tx(bar, (unsigned)(CIN / 8 * 3 * MT * 16));
            if constexpr (CIN == 32) load_row_tma_sw64(sx, &xmap, bar, x, x0, r, zz, nx, ny, nz, lane, s % RING);
            else load_row_tma<CIN>(sx, &xmap, bar, x, x0, r, zz, nx, ny, nz, lane, s % RING);
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
            return true;
        });
        cp_async_wait<0>();
    } else if (!use_tma && warp >= 4 && warp < 4 + NLW) {
        // each loader thread's copies of step s arrive on ready(s) when they
        // land, so the loaders run ahead as far as the ring allows
        const int tix = tid - 128;
        for_steps(t_begin, t_end, ny, nz, [&](int s, int x0, int zz, int r, bool, bool) {
            if (*abort_flag) return false;
            // slot s % RING was last read by step s - RING
            const int jw = s - RING;
            if (jw >= 0 && !mbar_wait_fast(mmadone + (jw & 3), (unsigned)(jw >> 2) & 1u)) {
                give_up();
                return false;
            }
            load_row_async<CIN, 32 * NLW>(sx, x, x0, r, zz, nx, ny, nz, tix, s % RING);
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(ready + (s & 3)))
                         : "memory");
            return true;
        });
        cp_async_wait<0>();
    } else if (warp == 4 + NLW) {
        if (lane == 0) {
            constexpr uint32_t IDESC = idesc_bf16(MT, L::NW);
            const uint64_t da0 = smem_desc(smem_u32(sx), RSEG * 16, 128);
            const uint64_t da0s = smem_desc_sw64(smem_u32(sx));
            const uint64_t db0 = smem_desc(smem_u32(sw), 128, (KB / 8) * 128);
            for_steps(t_begin, t_end, ny, nz, [&](int s, int, int, int r, bool first, bool) {
                if (*abort_flag) return false;
                if (!mbar_wait_fast(ready + (s & 3), (unsigned)(s >> 2) & 1u) ||
                    (s > 0 && !mbar_wait_fast(accempty, (unsigned)(s - 1) & 1u))) {
                    give_up();
                    return false;
                }
                fence_proxy_async();   // the ring row, written by cp.async, is read by the tensor cores
                tc_fence_after();
                // window of y-tap blocks for slots 0, 1, 2: starts at (1 - r) mod 3
                const uint32_t st = (uint32_t)(((1 - r) % 3 + 3) % 3);
                const uint32_t as = (uint32_t)((s % RING) * 3 * BXP + XR0);
                // the step's descriptors first (their low words: the start
                // addresses; the high words are fixed), then its MMAs back to
                // back.  Tap (dz, dx) moves the A start by whole voxel rows:
                // 64-byte rows in the swizzled form (the second K half 32
                // bytes into the row), 16-byte rows otherwise (the second K
                // half one chunk of the ring further)
                constexpr int NM = 9 * CIN / 16, KH = CIN / 16;
                const bool swz = CIN == 32 && use_tma;
                const uint64_t dab = swz ? da0s : da0;
                const uint32_t a0 = (uint32_t)dab + (swz ? as * 4 : as);
                const uint32_t b0 = (uint32_t)db0 + st * (COUT / 8) * (KB / 8) * 8;
                uint32_t alo[NM], blo[NM];
#pragma unroll
                for (int j = 0; j < NM; ++j) {
                    const int dz = j / (3 * KH), dx = (j / KH) % 3, kk = j % KH;
                    alo[j] = a0 + (swz ? (uint32_t)((dz * BXP + dx) * 4 + 2 * kk)
                                       : (uint32_t)(2 * kk * RSEG + dz * BXP + dx));
                    blo[j] = b0 + (uint32_t)((((dz * 3 + dx) * CIN + kk * 16) >> 3) * 8);
                }
                const uint64_t ahi = dab & 0xFFFFFFFF00000000ull, bhi = db0 & 0xFFFFFFFF00000000ull;
#pragma unroll
                for (int j = 0; j < NM; ++j)
                    umma_bf16(tmem, ahi | alo[j], bhi | blo[j], IDESC, (first && j == 0) ? 0u : 1u);
                umma_commit(accfull);
                umma_commit(mmadone + (s & 3));
                *last_commit = s;
                return true;
            });
        }
        __syncwarp();
    } else if (warp < 4) {   // loader warps without work (TMA rows) take no role
        for_steps(t_begin, t_end, ny, nz, [&](int s, int x0, int zz, int r, bool, bool emit) {
            if (*abort_flag) return false;
            if (!mbar_wait_fast(accfull, (unsigned)s & 1u)) {
                give_up();
                return false;
            }
            tc_fence_after();
            const int yo = r - 1;   // the output row this step completes
            const uint32_t col = (uint32_t)((((yo % 3) + 3) % 3) * COUT);
            const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + col;
            float acc[COUT];
            if (emit) tmem_ld<COUT>(ta, acc);
            tmem_st_zero<COUT>(ta);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(accempty);
            if (!emit) return true;
            const int m = warp * 32 + lane;
            const bool own = x0 + m < nx;   // for nx < 128 the tile repeats the row's period
            const size_t vox = ((size_t)zz * ny + yo) * nx + (own ? x0 + m : 0);
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
            return true;
        });
    }
    // every MMA has completed once the epilogue has seen its last accumulator;
    // after an abort, wait (bounded) for the last issued step's MMAs before
    // freeing TMEM
    __syncthreads();
    if (*abort_flag && tid == 0 && *last_commit >= 0) {
        const int jl = *last_commit;
        mbar_wait_fast(mmadone + (jl & 3), (unsigned)(jl >> 2) & 1u);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::NCOL));
}

// ---------------------------------------------------------------------------
// Weight gradient on the tensor cores.
//
// dW[n][tap(dx,dy,dz)*CIN+ci] = sum_v dY[v][n] X[v + (dx-1, dy-1, dz-1)][ci]
// is a GEMM whose K runs over voxels.  For an x segment of WT=64 voxels
// (x0..x0+63) of one (y, z) row, with u = 0..KT-1 indexing x0-1+u:
//
//   A[(dx, n)][u]   = dY[x0 + u - dx][n]  (zero outside the segment's own
//                     voxels; rows 3*COUT..127 zero)           M = 128
//   B_dy[(dz,ci)][u] = X[x0-1+u, y+dy-1, z+dz-1][ci] (periodic in x, y; zero
//                     outside z and for u >= WT+2)             N = 3*CIN
//   D_dy[(dx,n)][(dz,ci)] += sum_u A B_dy                      K = KT = 80
//
// so one segment is 3 (y taps) x 5 (K steps of 16) MMAs of M=128, N=3*CIN,
// both operands K-major in the canonical no-swizzle layout, staged by the
// CTA's threads: A from a transposed copy of the segment's dY (the x tap is
// a shift by 0..2 elements, formed with byte permutes), B by 8x8 transposes
// of the channels-last input.  Segments alternate between two staging
// buffers, so the MMAs of one overlap the staging of the next.  The three
// accumulators (3*3*CIN columns) stay in TMEM over all of a CTA's segments
// (a fixed set, in a fixed order); each CTA writes its partial sums to a
// workspace row and a second kernel adds the rows to dW in CTA order, so the
// result does not depend on timing.
constexpr int WT = 64;               // voxels of an x segment
constexpr int KT = 80;               // K of a segment: WT + 2 halo voxels, padded to 16
constexpr int WG_NTH = 256;          // threads of a weight-gradient CTA
constexpr int DYW = 8 + KT + 8;      // row of the transposed dY: 8 zeros, the segment, zeros

template <int CIN, int COUT>
struct WgLay {
    static constexpr int N = 3 * CIN;                         // columns of one y-tap accumulator
    static constexpr uint32_t NCOL = 3 * N <= 256 ? 256 : 512;
    static constexpr size_t A_B = (size_t)(KT / 8) * 128 * 16;    // one A buffer
    static constexpr size_t BD_B = (size_t)(KT / 8) * N * 16;     // one y tap of a B buffer
    static constexpr size_t B_B = 3 * BD_B;
    static constexpr size_t BUF_B = A_B + B_B;
    static constexpr size_t DYT_OFF = 2 * BUF_B;
    static constexpr size_t DYT_B = (size_t)COUT * DYW * 2;
    static constexpr size_t RED_OFF = (DYT_OFF + DYT_B + 15) / 16 * 16;
    static constexpr size_t RED_B = (size_t)WG_NTH * 8 * 4;
    static constexpr size_t BAR_OFF = RED_OFF + RED_B;
    static constexpr size_t BYTES = BAR_OFF + 2 * 8 + 16 + 1024;   // + alignment of the base to 1024 bytes
};

// 8x8 transpose of BF16: v[a] holds 8 channels of voxel a (word w: channels
// 2w, 2w+1); r[i] receives voxels 0..7 of channel i
__device__ __forceinline__ void transpose8(const uint4 (&v)[8], uint4 (&r)[8])
{
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t sel = (i & 1) ? 0x7632u : 0x5410u;
        uint32_t o[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const uint4& a = v[2 * w];
            const uint4& b = v[2 * w + 1];
            const uint32_t wa = (i >> 1) == 0 ? a.x : (i >> 1) == 1 ? a.y : (i >> 1) == 2 ? a.z : a.w;
            const uint32_t wb = (i >> 1) == 0 ? b.x : (i >> 1) == 1 ? b.y : (i >> 1) == 2 ? b.z : b.w;
            o[w] = __byte_perm(wa, wb, sel);
        }
        r[i] = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(WG_NTH, 1) k_conv3d_wgrad_tc(const __nv_bfloat16* __restrict__ x,
                                                               const __nv_bfloat16* __restrict__ dy,
                                                               float* __restrict__ ws, int nx, int ny, int nz,
                                                               int* __restrict__ err)
{
    using L = WgLay<CIN, COUT>;
    constexpr int N = L::N, K = 27 * CIN, NCC = CIN / 8, NNC = COUT / 8;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* const sb = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    __nv_bfloat16* const dyt = reinterpret_cast<__nv_bfloat16*>(sb + L::DYT_OFF);
    float* const red = reinterpret_cast<float*>(sb + L::RED_OFF);
    unsigned long long* const mmadone = reinterpret_cast<unsigned long long*>(sb + L::BAR_OFF);
    uint32_t* const tslot = reinterpret_cast<uint32_t*>(sb + L::BAR_OFF + 16);
    volatile int* const abort_flag = reinterpret_cast<volatile int*>(sb + L::BAR_OFF + 20);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // A rows 3*COUT..127 stay zero in both buffers; the dY padding is rewritten per segment
    for (int q = tid; q < 2 * (KT / 8) * 128; q += WG_NTH) {
        const int b = q / ((KT / 8) * 128), r = q % ((KT / 8) * 128);
        const int row = r % 128, kc = r / 128;
        if (row >= 3 * COUT)
            *reinterpret_cast<uint4*>(sb + b * L::BUF_B + (size_t)kc * 2048 + row * 16) = make_uint4(0, 0, 0, 0);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(L::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(mmadone + 0, 1);
        mbar_init(mmadone + 1, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const int nseg = (nx + WT - 1) / WT;
    const int ntile = nseg * ny * nz;
    float dbacc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};   // dY sums of this thread's 8 channels
    int i = 0;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x, ++i) {
        const int seg = t % nseg, yy = (t / nseg) % ny, zz = t / (nseg * ny);
        const int x0 = seg * WT;
        const int mlim = nx - x0 < WT ? nx - x0 : WT;   // the segment's own voxels (nx < 64: one period)
        const int b = i & 1;
        unsigned char* const sa = sb + b * L::BUF_B;
        unsigned char* const sbb = sa + L::A_B;
        // the buffer was last read by the MMAs of segment i-2
        if (i >= 2) {
            bool ok = true;
            if (tid == 0) ok = mbar_wait(mmadone + b, (unsigned)((i - 2) >> 1) & 1u);
            if (!ok) *abort_flag = 1;
        }
        __syncthreads();
        if (*abort_flag) break;
        // ---- dY of the segment, transposed: dyt[n][8 + j], zeros around it
        {
            const size_t row = ((size_t)zz * ny + yy) * nx + x0;
            for (int q = tid; q < WT * NNC; q += WG_NTH) {
                const int nc = q % NNC, j = q / NNC;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (j < mlim) v = __ldg(reinterpret_cast<const uint4*>(dy + (row + j) * COUT + nc * 8));
                const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    dyt[(nc * 8 + e) * DYW + 8 + j] = h[e];
                    dbacc[e] += __bfloat162float(h[e]);
                }
            }
            for (int q = tid; q < COUT * 16; q += WG_NTH) {
                const int n = q / 16, e = q % 16;
                dyt[n * DYW + (e < 8 ? e : 8 + WT + (e - 8))] = __float2bfloat16_rn(0.f);
            }
            for (int q = tid; q < COUT * (KT - WT); q += WG_NTH) {   // beyond the segment up to KT
                const int n = q / (KT - WT), e = q % (KT - WT);
                if (8 + WT + 8 + e < DYW) dyt[n * DYW + 8 + WT + 8 + e] = __float2bfloat16_rn(0.f);
            }
        }
        __syncthreads();
        // ---- A[(dx, n)][u] = dyt[n][8 + u - dx]: 16-byte rows (kc, row)
        for (int q = tid; q < (KT / 8) * 3 * COUT; q += WG_NTH) {
            const int kc = q / (3 * COUT), m = q % (3 * COUT);
            const int dxs = m / COUT, n = m % COUT;
            const uint4 c0 = *reinterpret_cast<const uint4*>(dyt + n * DYW + kc * 8);       // elements 8kc-8 ..
            const uint4 c1 = *reinterpret_cast<const uint4*>(dyt + n * DYW + kc * 8 + 8);   // elements 8kc ..
            uint4 o;
            if (dxs == 0) o = c1;
            else if (dxs == 2) o = make_uint4(c0.w, c1.x, c1.y, c1.z);
            else o = make_uint4(__byte_perm(c0.w, c1.x, 0x5432), __byte_perm(c1.x, c1.y, 0x5432),
                                __byte_perm(c1.y, c1.z, 0x5432), __byte_perm(c1.z, c1.w, 0x5432));
            *reinterpret_cast<uint4*>(sa + (size_t)kc * 2048 + m * 16) = o;
        }
        // ---- B_dy[(dz, ci)][u]: 8x8 transposes of the input rows
        for (int q = tid; q < 9 * NCC * (KT / 8); q += WG_NTH) {
            const int kc = q % (KT / 8), c = (q / (KT / 8)) % NCC, rz = q / ((KT / 8) * NCC);
            const int dys = rz / 3, dzs = rz % 3;
            int gy = yy + dys - 1;
            gy = gy < 0 ? gy + ny : (gy >= ny ? gy - ny : gy);
            const int gz = zz + dzs - 1;
            uint4 v[8];
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const int u = kc * 8 + a;
                v[a] = make_uint4(0, 0, 0, 0);
                if (gz >= 0 && gz < nz && u < WT + 2) {
                    int gx = x0 - 1 + u;
                    if (nx >= WT) gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
                    else gx = (gx + nx) % nx;
                    v[a] = __ldg(reinterpret_cast<const uint4*>(x + (((size_t)gz * ny + gy) * nx + gx) * CIN + c * 8));
                }
            }
            uint4 r[8];
            transpose8(v, r);
            unsigned char* dst = sbb + (size_t)dys * L::BD_B + (size_t)kc * (N * 16) + (size_t)(dzs * CIN + c * 8) * 16;
#pragma unroll
            for (int e = 0; e < 8; ++e) *reinterpret_cast<uint4*>(dst + e * 16) = r[e];
        }
        fence_proxy_async();   // plain stores above are read by the tensor cores
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            constexpr uint32_t IDESC = idesc_bf16(128, N);
            const uint32_t aaddr = smem_u32(sa), baddr = smem_u32(sbb);
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int k2 = 0; k2 < KT / 16; ++k2) {
                    const uint64_t da = smem_desc(aaddr + (uint32_t)(2 * k2) * 2048u, 2048u, 128u);
                    const uint64_t db = smem_desc(baddr + (uint32_t)(d * L::BD_B + (size_t)(2 * k2) * N * 16),
                                                  (uint32_t)(N * 16), 128u);
                    umma_bf16(tmem + (uint32_t)(d * N), da, db, IDESC, (i == 0 && k2 == 0) ? 0u : 1u);
                }
            umma_commit(mmadone + b);
        }
    }
    // every MMA issued has completed once the last commit of each buffer has
    const int nmine = i;
    if (tid == 0) {
        for (int j = nmine - 2 < 0 ? 0 : nmine - 2; j < nmine; ++j)
            if (!mbar_wait(mmadone + (j & 1), (unsigned)(j >> 1) & 1u)) *abort_flag = 1;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    float* const wrow = ws + (size_t)blockIdx.x * ((size_t)COUT * K + COUT);
    if (*abort_flag) {
        if (tid == 0) atomicExch(err, 1);
    } else if (nmine > 0 && warp < 4) {
        // accumulator lane m = (dx, n); columns (dz, ci) of y tap d
        const int m = warp * 32 + lane;
        const int dxs = m / COUT, n = m % COUT;
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tmem_ld<16>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d * N + c0), v);
                if (dxs < 3) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const int col = c0 + e, dzs = col / CIN, ci = col % CIN;
                        wrow[(size_t)n * K + (dxs + 3 * d + 9 * dzs) * CIN + ci] = v[e];
                    }
                }
            }
    } else if (nmine == 0 && warp < 4) {
        // a CTA without segments contributes zeros
        for (int q = tid; q < COUT * K; q += 128) wrow[q] = 0.f;
    }
    // bias gradient: this thread's 8 channel sums, added up over the threads
    // that hold the same channels, in thread order
#pragma unroll
    for (int e = 0; e < 8; ++e) red[tid * 8 + e] = dbacc[e];
    __syncthreads();
    if (tid < COUT) {
        const int nc = tid / 8, e = tid % 8;
        float sacc = 0.f;
        for (int t2 = nc; t2 < WG_NTH; t2 += NNC) sacc += red[t2 * 8 + e];
        wrow[(size_t)COUT * K + tid] = sacc;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::NCOL));
}

// dW += sum over CTAs of their rows of the workspace, in CTA order (and db);
// NaN everywhere when a CTA of the gradient kernel gave up a wait
__global__ void k_wgrad_reduce(const float* __restrict__ ws, int rows, int nw, int nb, float* __restrict__ dw,
                               float* __restrict__ db, const int* __restrict__ err)
{
    const int stride = nw + nb;
    const bool bad = *err != 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < stride; q += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int r = 0; r < rows; ++r) acc += ws[(size_t)r * stride + q];
        if (bad) acc = __int_as_float(0x7fc00000);
        if (q < nw) dw[q] += acc;
        else if (db) db[q - nw] += acc;
    }
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

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// tiled TMA map of a BF16 array of the given rank, zeros outside
cudaError_t encode_bf16(CUtensorMap* map, int rank, void* base, const cuuint64_t* dims, const cuuint64_t* strides,
                        const cuuint32_t* box, CUtensorMapSwizzle swz)
{
    static EncodeTiledFn enc = nullptr;
    if (!enc) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return cudaErrorInvalidValue;
        enc = reinterpret_cast<EncodeTiledFn>(fn);
    }
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN, int COUT>
cudaError_t launch_conv_t(const void* x, const void* w, const float* bias, const void* mask, int relu, void* y,
                          float* yf, int nx, int ny, int nz, int* err, cudaStream_t st)
{
    using L = ConvLay<CIN, COUT>;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t ae = smem_attr_once(attr, reinterpret_cast<const void*>(k_conv3d<CIN, COUT>), L::BYTES);
    if (ae != cudaSuccess) return ae;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntile = ((nx + MT - 1) / MT) * ny * nz;
    const int grid = ntile < sms ? ntile : sms;
    // rows of x segments of 128 by TMA: (8 channels, chunk, x, y, z) boxes
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    const int use_tma = nx % MT == 0 ? 1 : 0;
    if (use_tma && CIN == 32) {
        // (channel, x, y, z) boxes of 32 channels x 128 voxels, 64-byte swizzled rows
        const cuuint64_t dims[4] = {(cuuint64_t)CIN, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
        const cuuint64_t strides[3] = {(cuuint64_t)CIN * 2, (cuuint64_t)nx * CIN * 2, (cuuint64_t)nx * ny * CIN * 2};
        const cuuint32_t box[4] = {(cuuint32_t)CIN, (cuuint32_t)MT, 1, 1};
        if (encode_bf16(&map, 4, const_cast<void*>(x), dims, strides, box, CU_TENSOR_MAP_SWIZZLE_64B) != cudaSuccess)
            return cudaErrorInvalidValue;
    } else if (use_tma) {
        // (8 channels, chunk, x, y, z) boxes, 16-byte rows
        const cuuint64_t dims[5] = {8, (cuuint64_t)CIN / 8, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
        const cuuint64_t strides[4] = {16, (cuuint64_t)CIN * 2, (cuuint64_t)nx * CIN * 2,
                                       (cuuint64_t)nx * ny * CIN * 2};
        const cuuint32_t box[5] = {8, 1, (cuuint32_t)MT, 1, 1};
        if (encode_bf16(&map, 5, const_cast<void*>(x), dims, strides, box, CU_TENSOR_MAP_SWIZZLE_NONE) != cudaSuccess)
            return cudaErrorInvalidValue;
    }
    k_conv3d<CIN, COUT><<<grid, CT, L::BYTES, st>>>(
        map, use_tma, static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), bias,
        static_cast<const __nv_bfloat16*>(mask), relu, static_cast<__nv_bfloat16*>(y), yf, nx, ny, nz, err);
    return cudaGetLastError();
}

// the tensor-core weight gradient: one CTA per SM (a fixed grid of at most
// the SM count over the segments), its partial rows in a stream-ordered
// workspace, then the ordered reduction into dw, db
template <int CIN, int COUT>
cudaError_t launch_wgrad_tc_t(const void* x, const void* dy, float* dw, float* db, int nx, int ny, int nz,
                              cudaStream_t st)
{
    using L = WgLay<CIN, COUT>;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t ae = smem_attr_once(attr, reinterpret_cast<const void*>(k_conv3d_wgrad_tc<CIN, COUT>), L::BYTES);
    if (ae != cudaSuccess) return ae;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntile = ((nx + WT - 1) / WT) * ny * nz;
    const int grid = ntile < sms ? ntile : sms;
    const size_t stride = (size_t)COUT * 27 * CIN + COUT;
    const size_t bytes = (size_t)grid * stride * sizeof(float) + 16;
    void* buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, bytes, st);
    if (e != cudaSuccess) return e;
    int* err = reinterpret_cast<int*>(static_cast<char*>(buf) + (size_t)grid * stride * sizeof(float));
    e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        k_conv3d_wgrad_tc<CIN, COUT><<<grid, WG_NTH, L::BYTES, st>>>(
            static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), static_cast<float*>(buf),
            nx, ny, nz, err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        const int nw = COUT * 27 * CIN;
        k_wgrad_reduce<<<(int)((stride + 255) / 256), 256, 0, st>>>(static_cast<const float*>(buf), grid, nw, COUT,
                                                                    dw, db, err);
        e = cudaGetLastError();
    }
    const cudaError_t f = cudaFreeAsync(buf, st);
    return e != cudaSuccess ? e : f;
}

}  // namespace clo
}  // namespace mhd3d

using namespace mhd3d::clo;

// activations and weights move as 16-byte vectors
static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

extern "C" {

int mhd3d_conv3d(int32_t cin, int32_t cout, const void* x, const void* w, const float* bias, const void* mask,
                 int32_t relu, void* y, float* yf, int32_t nx, int32_t ny, int32_t nz, int32_t* err, void* stream)
{
    if (!x || !w || !err || nx <= 0 || ny <= 0 || nz <= 0 || (!y && !yf))
        return MHD3D_ERR_ARG;
    if (!aligned16(x) || !aligned16(w) || !aligned16(mask) || !aligned16(y) || !aligned16(yf)) return MHD3D_ERR_ARG;
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
    if (!x || !dy || !dw || nx <= 0 || ny <= 0 || nz <= 0) return MHD3D_ERR_ARG;
    if (!aligned16(x) || !aligned16(dy)) return MHD3D_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (cin == 16 && cout == 32) e = launch_wgrad_tc_t<16, 32>(x, dy, dw, db, nx, ny, nz, st);
    else if (cin == 32 && cout == 32) e = launch_wgrad_tc_t<32, 32>(x, dy, dw, db, nx, ny, nz, st);
    else if (cin == 32 && cout == 16) e = launch_wgrad_tc_t<32, 16>(x, dy, dw, db, nx, ny, nz, st);
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
