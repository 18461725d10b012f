// stage_impl.cuh -- the fused RK3 stage kernel (RHS + update + BCON +
// ghost-plane toggle + CFL reduction) and the standalone CFL/BCON kernels.
//
// Included twice: by stage_exact.cu (compiled with -fmad=false, so every
// product and sum is rounded separately, as gfortran -O2 evaluates the
// reference) and by stage_fast.cu (FMA contraction allowed).  MHD3D_NS names
// the namespace of each copy.
//
// Work decomposition: a CTA owns a TX x TY tile of (x,y) columns and a
// chunk of z planes and marches down the chunk.  The raw fields of each
// plane arrive by TMA (cp.async.bulk.tensor, one 4-D box per plane: x with
// the periodic halo, y with the halo, one plane, all fields) into a
// four-slot ring two planes ahead of the plane being computed; 1/RO of
// planes k-1, k, k+1 sits in a three-slot ring next to it.  Velocities and
// pressure are formed where they are used, from the same two operands
// FLUXES multiplies (3dmhdsub.f:1386-1425), so every right-hand-side term
// (1249-2634), including the 19-point cross terms, reads shared memory.
// The Z tile of the plane (stages 2, 3) arrives by its own TMA box while
// the right-hand side is computed.  The wall planes take BCON (2751-2955)
// in the same pass: the thread owning a column keeps the new values of the
// two planes next to each wall in registers.  No TMA load uses cluster
// multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cfloat>

#include "../../include/mhd3d.h"
#include "mhd3d_dev.cuh"
#include "smem_attr.cuh"
#include "cfl_cell.cuh"
#include "ring.cuh"

namespace mhd3d {
namespace MHD3D_NS {

enum Q { Q_RU = 0, Q_RV, Q_RW, Q_RO, Q_TT, Q_RI, Q_UU, Q_VV, Q_WW, Q_P, Q_BX, Q_BY, Q_BZ };

#ifndef MHD3D_NRAW
#define MHD3D_NRAW 4
#endif
// raw-plane ring slots: planes k-1, k, k+1 in use and, with 4, plane k+2 in
// flight (with 3 the next plane is issued when plane k-1's slot frees)
constexpr int NRAW = MHD3D_NRAW;
static_assert(NRAW >= 3 && NRAW <= 6, "three to six ring slots (NRAW+2 mbarriers)");
constexpr int NRI = 3;    // 1/RO ring slots (planes k-1, k, k+1)

template <bool MAG>
struct Lay {
    static constexpr int NF = MAG ? 8 : 5;
    static constexpr int RAW_SLOT = (NF * BSLOT * 8 + 127) / 128 * 128 / 8;   // doubles, 128-B aligned
    static constexpr int ZT = NF * TY * TX;                                   // Z tile doubles
    static constexpr int RI_OFF = NRAW * RAW_SLOT;
    static constexpr int Z_OFF = ((RI_OFF + NRI * BSLOT) * 8 + 127) / 128 * 128 / 8;
    static constexpr int BAR_OFF = Z_OFF + 2 * ZT;       // two Z slots; NRAW+2 <= 8 mbarriers (8 B each)
    static constexpr int RED_OFF = BAR_OFF + 8;          // CFL block reduction
    static constexpr int FLAG_OFF = RED_OFF + (NT / 32) * 8;   // 3 keys + a 40-byte screening record per warp
    static constexpr int TOTAL = FLAG_OFF + 2;
    static constexpr size_t BYTES = (size_t)TOTAL * 8 + 128;   // + alignment slack
};

#ifndef MHD3D_FASTRCP
#define MHD3D_FASTRCP 1
#endif
#if MHD3D_FAST_BODY && MHD3D_FASTRCP
// 1/x by two Newton-Raphson steps y <- y + y(1 - xy) from the approximate
// reciprocal rcp.approx.ftz.f64 (each step squares the relative error, so
// two reach the rounding level): within an ulp or so of the correctly rounded
// 1/x for the positive normal densities it is used on.  The derive step of
// every arriving plane runs between a copy wait and a CTA barrier, where a
// full division's latency shows.  FMA build only; the reference-rounding
// build divides.
__device__ __forceinline__ double recip(double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
#else
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }
#endif

// value of quantity QQ at offset off of a plane slot: raw fields, 1/RO, and the
// products FLUXES forms on the whole array (UU=RU*RO' with RO'=1/RO, WW1=RO*TT)
template <int QQ>
__device__ __forceinline__ double qv(const double* __restrict__ raw, const double* __restrict__ ri, int off)
{
    if constexpr (QQ == Q_RU) return raw[F_RU * BSLOT + off];
    else if constexpr (QQ == Q_RV) return raw[F_RV * BSLOT + off];
    else if constexpr (QQ == Q_RW) return raw[F_RW * BSLOT + off];
    else if constexpr (QQ == Q_RO) return raw[F_RO * BSLOT + off];
    else if constexpr (QQ == Q_TT) return raw[F_TT * BSLOT + off];
    else if constexpr (QQ == Q_BX) return raw[F_BX * BSLOT + off];
    else if constexpr (QQ == Q_BY) return raw[F_BY * BSLOT + off];
    else if constexpr (QQ == Q_BZ) return raw[F_BZ * BSLOT + off];
    else if constexpr (QQ == Q_RI) return ri[off];
    else if constexpr (QQ == Q_UU) return raw[F_RU * BSLOT + off] * ri[off];
    else if constexpr (QQ == Q_VV) return raw[F_RV * BSLOT + off] * ri[off];
    else if constexpr (QQ == Q_WW) return raw[F_RW * BSLOT + off] * ri[off];
    else return raw[F_RO * BSLOT + off] * raw[F_TT * BSLOT + off];
}

// store a cell of U and the periodic halo copies COMMUNICATE would make of it
__device__ __forceinline__ void store_u(double* __restrict__ u, size_t fofs, const StageArgs& a, int gi, int gj,
                                        int kz, double v)
{
    const int npx = a.s.npx, npy = a.s.npy;
    const size_t base = fofs + (size_t)kz * a.uz;
    const int ix = gi + 1, jy = gj + 1;
    u[base + (size_t)jy * a.upitch + ix] = v;
    const int hx = (gi == 0) ? npx + 1 : (gi == npx - 1) ? 0 : -1;
    const int hy = (gj == 0) ? npy + 1 : (gj == npy - 1) ? 0 : -1;
    if (hx >= 0) u[base + (size_t)jy * a.upitch + hx] = v;
    if (hy >= 0) u[base + (size_t)hy * a.upitch + ix] = v;
    if (hx >= 0 && hy >= 0) u[base + (size_t)hy * a.upitch + hx] = v;
}

#include "cfl_acc.cuh"

// Block-wide reduction of the CFL parts into the global accumulators.
__device__ __forceinline__ void cfl_commit(Accum* acc, unsigned long long k1, unsigned long long k2,
                                           unsigned long long k3, unsigned long long k4, unsigned long long km,
                                           unsigned int bad, unsigned long long* red)
{
    for (int o = 16; o > 0; o >>= 1) {
        k1 = min(k1, __shfl_xor_sync(0xffffffffu, k1, o));
        k2 = min(k2, __shfl_xor_sync(0xffffffffu, k2, o));
        k3 = min(k3, __shfl_xor_sync(0xffffffffu, k3, o));
        k4 = min(k4, __shfl_xor_sync(0xffffffffu, k4, o));
        km = max(km, __shfl_xor_sync(0xffffffffu, km, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        red[w * 6 + 0] = k1;
        red[w * 6 + 1] = k2;
        red[w * 6 + 2] = k3;
        red[w * 6 + 3] = k4;
        red[w * 6 + 4] = km;
        red[w * 6 + 5] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < NT / 32; ++i) {
            k1 = min(k1, red[i * 6 + 0]);
            k2 = min(k2, red[i * 6 + 1]);
            k3 = min(k3, red[i * 6 + 2]);
            k4 = min(k4, red[i * 6 + 3]);
            km = max(km, red[i * 6 + 4]);
            bad |= (unsigned int)red[i * 6 + 5];
        }
        atomicMin(&acc->wmin[0], k1);
        atomicMin(&acc->wmin[1], k2);
        atomicMin(&acc->wmin[2], k3);
        atomicMin(&acc->wmin[3], k4);
        atomicMax(&acc->umax, km);
        if (bad) atomicOr(&acc->bad, 1u);
    }
}

// ---------------------------------------------------------------------------
// The stage kernel.  STAGE 0: right-hand side only (written to f_out);
// STAGE 1..3: the RK3 substeps of STEP (3dmhdsub.f:874-1169).
// ---------------------------------------------------------------------------
template <bool MAG, bool ROT, int STAGE>
#ifndef MHD3D_MINB
#define MHD3D_MINB 3   // CTAs per SM: 3 x 128 threads x 168 registers, 3 x 72 KB shared
#endif
__global__ void __launch_bounds__(NT, MHD3D_MINB) k_stage(const __grid_constant__ StageArgs a)
{
    using L = Lay<MAG>;
    constexpr int NF = L::NF;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // 128-byte aligned base, formed by pointer arithmetic on the shared array
    // so that every access below stays a shared-window (32-bit) access
    double* const sbase = reinterpret_cast<double*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
    double* const sraw = sbase;
    double* const sri = sbase + L::RI_OFF;
    double* const sz = sbase + L::Z_OFF;
    unsigned long long* const bars = reinterpret_cast<unsigned long long*>(sbase + L::BAR_OFF);
    unsigned long long* const red = reinterpret_cast<unsigned long long*>(sbase + L::RED_OFF);
    int* const sflag = reinterpret_cast<int*>(sbase + L::FLAG_OFF);

    const Control* ctl = a.ctl;

    const Scalars& s = a.s;
    const Metrics& m = a.m;
    const int npx = s.npx, npy = s.npy, npz = s.npz;
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int tile = blockIdx.x;
    const int x0 = (tile % a.ntx) * TX, y0 = (tile / a.ntx) * TY;
    const int chunk = blockIdx.y;
    const int k0 = chunk * a.zlen;
    const int k1 = (chunk == a.nchunks - 1) ? npz : k0 + a.zlen;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool active = gi < npx && gj < npy;
    const int lx = tx + 1, ly = ty + 1;

    const double DT = ctl->dt;
    const double cu = STAGE == 1 ? s.gam1 * DT : STAGE == 2 ? s.gam2 * DT : s.gam3 * DT;   // COEF for U
    const double cz = STAGE == 1 ? s.zeta1 * DT : s.zeta2 * DT;                            // COEF for Z

    const double dxi = active ? m.dxxdx[gi + 1] : 0.0, d2xi = active ? m.d2xxdx2[gi + 1] : 0.0;
    const double dyj = active ? m.dyydy[gj + 1] : 0.0, d2yj = active ? m.d2yydy2[gj + 1] : 0.0;
    const double HX = s.hx, H2X = s.h2x, HY = s.hy, H2Y = s.h2y, HZ = s.hz, H2Z = s.h2z;
    const double C13 = s.c13, C23 = s.c23, C43 = s.c43, OCV = s.ocv, ORE = s.ore;
#if MHD3D_FAST_BODY
    // d/dx ~ (f+ - f-)*ax, d2/dx2 ~ (f+ - f-)*bxq + (f+ + f- - 2f)*cxq, likewise in y and z
    const double ax = active ? m.fax[gi + 1] : 0.0, bxq = active ? m.fbx[gi + 1] : 0.0, cxq = active ? m.fcx[gi + 1] : 0.0;
    const double ay = active ? m.fay[gj + 1] : 0.0, byq = active ? m.fby[gj + 1] : 0.0, cyq = active ? m.fcy[gj + 1] : 0.0;
    (void)HX; (void)H2X; (void)HY; (void)H2Y; (void)HZ; (void)H2Z; (void)OCV; (void)ORE; (void)dxi; (void)d2xi; (void)dyj; (void)d2yj;
#endif

    const unsigned raw_bytes = (unsigned)(NF * BSLOT * 8);
    const unsigned z_bytes = (unsigned)(NF * TY * TX * 8);
    // own column in the U layout (periodic halo at index 0 and NPX+1 / NPY+1,
    // ghost planes at 0 and NPZ+1) and in the compact Z/F layout
    const size_t ucol = (size_t)(gj + 1) * a.upitch + (gi + 1);
    const size_t zcol = (size_t)gj * a.zpitch + gi;
    const HaloCols hc = halo_cols(npx, npy, a.upitch, gi, gj);

    // the stop flag is read once, by one thread, so the CTA takes one path
    if (tid == 0) {
        const bool stopped = STAGE != 0 && ctl->stop;
        *sflag = stopped ? -1 : 0;
        if (!stopped) {
            for (int i = 0; i < NRAW + 2; ++i) mbar_init(&bars[i], 1);
            fence_mbar_init();
        }
    }
    if (STAGE == 3 && (tid & 31) == 0) {
        unsigned long long* r = red + (tid >> 5) * 3;
        r[0] = ~0ull;
        r[1] = 0ull;
        r[2] = 0ull;
    }
    if (STAGE == 3) cfl_screen_init(red, a.acc, a.s, MAG);
    __syncthreads();
    if (*sflag < 0) return;

    // plane kp (-1 .. npz) lives in raw slot (kp+1)&3 and 1/RO slot (kp+1)%3;
    // it is the ((kp-(k0-1))>>2)-th fill of its slot
    int hi_issued = k0 - 2;   // thread 0: highest plane issued so far
    auto issue_plane = [&](int kp) {
        const int sl = (kp + 1) % NRAW;
        fence_proxy_async();
        mbar_expect_tx(&bars[sl], raw_bytes);
        tma_load4(sraw + (size_t)sl * L::RAW_SLOT, &a.map_u, &bars[sl], x0, y0, kp + 1, 0);
        hi_issued = kp;
    };
    auto parity_of = [&](int kp) -> unsigned { return (unsigned)(((kp - (k0 - 1)) / NRAW) & 1); };
    auto derive_ri = [&](int kp) {
        const double* r = sraw + (size_t)((kp + 1) % NRAW) * L::RAW_SLOT + F_RO * BSLOT;
        double* d = sri + (size_t)((kp + 1) % 3) * BSLOT;
        for (int p = tid; p < BSLOT; p += NT) d[p] = recip(r[p]);
    };

    // Z of plane kp (stages 2, 3) goes to slot (kp-k0)&1, a plane ahead of its
    // use; it is the ((kp-k0)>>1)-th fill of that slot's barrier
    int z_hi = k0 - 1;   // thread 0: highest Z plane issued so far
    auto issue_z = [&](int kp) {
        const int zs = (kp - k0) & 1;
        fence_proxy_async();
        mbar_expect_tx(&bars[NRAW + zs], z_bytes);
        tma_load4(sz + (size_t)zs * L::ZT, &a.map_z, &bars[NRAW + zs], x0, y0, kp, 0);
        z_hi = kp;
    };
    auto wait_z = [&](int kp) -> bool {
        return mbar_wait(&bars[NRAW + ((kp - k0) & 1)], (unsigned)(((kp - k0) >> 1) & 1));
    };
    if (tid == 0) {
        for (int kp = k0 - 1; kp <= k0 - 2 + NRAW && kp <= k1; ++kp) issue_plane(kp);
        if (STAGE >= 2) issue_z(k0);
    }
    // the first wait's limit is a launch argument (a test lowers it to make
    // the wait give up); every other wait, the drain's included, is bounded
    // by WAIT_LIMIT
    bool ok = mbar_wait(&bars[(k0 + 0) % NRAW], parity_of(k0 - 1), (long)a.wait_first) &&
              mbar_wait(&bars[(k0 + 1) % NRAW], parity_of(k0));
    if (ok) {
        derive_ri(k0 - 1);
        derive_ri(k0);
    } else {
        atomicOr(sflag, 1);
    }
    CflAcc cfa;              // stage-3 CFL parts of this thread's cells
    const CflCol ccol = cfl_col(m, gi, gj, active);

    for (int k = k0; k < k1; ++k) {
        // Z of the next plane goes to the slot plane k-1's Z has left
        if (STAGE >= 2 && tid == 0 && !*sflag && k + 1 < k1) issue_z(k + 1);
        if (!mbar_wait(&bars[(k + 2) % NRAW], parity_of(k + 1))) atomicOr(sflag, 1);
        else derive_ri(k + 1);
        __syncthreads();
        if (*sflag) break;
        bool zok = true;
        if (active) {
            const double* Rm = sraw + (size_t)((k + 0) % NRAW) * L::RAW_SLOT;   // plane k-1
            const double* Rc = sraw + (size_t)((k + 1) % NRAW) * L::RAW_SLOT;   // plane k
            const double* Rp = sraw + (size_t)((k + 2) % NRAW) * L::RAW_SLOT;   // plane k+1
            const double* Im = sri + (size_t)((k + 0) % 3) * BSLOT;
            const double* Ic = sri + (size_t)((k + 1) % 3) * BSLOT;
            const double* Ip = sri + (size_t)((k + 2) % 3) * BSLOT;
#define C_(q, dx, dy) qv<q>(Rc, Ic, (ly + (dy)) * BW + (lx + (dx)))
#define M_(q, dx, dy) qv<q>(Rm, Im, (ly + (dy)) * BW + (lx + (dx)))
#define P_(q, dx, dy) qv<q>(Rp, Ip, (ly + (dy)) * BW + (lx + (dx)))
#define WALL_LOADS                                                                                   \
    double rw2 = 0, ww2 = 0, bx2 = 0, bx3 = 0, by2 = 0, by3 = 0;                                     \
    if (top || bot) {                                                                                \
        /* own column two and three planes inside the wall (one-sided stencils) */                  \
        const int kk2 = top ? 2 : npz - 3, kk3 = top ? 3 : npz - 4;                                  \
        const size_t c2 = (size_t)(kk2 + 1) * a.uz + ucol, c3 = (size_t)(kk3 + 1) * a.uz + ucol;     \
        rw2 = a.u_in[c2 + F_RW * a.uf];                                                              \
        const double ro2 = a.u_in[c2 + F_RO * a.uf];                                                 \
        ww2 = rw2 * (1.0 / ro2);                                                                     \
        if (MAG) {                                                                                   \
            bx2 = a.u_in[c2 + F_BX * a.uf];                                                          \
            bx3 = a.u_in[c3 + F_BX * a.uf];                                                          \
            by2 = a.u_in[c2 + F_BY * a.uf];                                                          \
            by3 = a.u_in[c3 + F_BY * a.uf];                                                          \
        }                                                                                            \
    }
#if MHD3D_FAST_BODY
            const bool top = (k == 0), bot = (k == npz - 1);
            const double az = m.faz[k + 1], bzq = m.fbz[k + 1], czq = m.fcz[k + 1];
            const double rka = m.rkapa[k + 1], dka = m.dkapa[k + 1];
            WALL_LOADS

            // center
            const double RIc = C_(Q_RI, 0, 0), ROc = C_(Q_RO, 0, 0), TTc = C_(Q_TT, 0, 0);
            const double RUc = C_(Q_RU, 0, 0), RVc = C_(Q_RV, 0, 0), RWc = C_(Q_RW, 0, 0);
            const double BXc0 = MAG ? C_(Q_BX, 0, 0) : 0.0, BYc0 = MAG ? C_(Q_BY, 0, 0) : 0.0;
            const double BZc0 = MAG ? C_(Q_BZ, 0, 0) : 0.0;
            const double uc = RUc * RIc, vc = RVc * RIc, wc = RWc * RIc;
            // face neighbours: velocities (the products FLUXES forms) and momenta
            const double u_xp = C_(Q_UU, 1, 0), u_xm = C_(Q_UU, -1, 0), u_yp = C_(Q_UU, 0, 1), u_ym = C_(Q_UU, 0, -1);
            const double v_xp = C_(Q_VV, 1, 0), v_xm = C_(Q_VV, -1, 0), v_yp = C_(Q_VV, 0, 1), v_ym = C_(Q_VV, 0, -1);
            const double w_xp = C_(Q_WW, 1, 0), w_xm = C_(Q_WW, -1, 0), w_yp = C_(Q_WW, 0, 1), w_ym = C_(Q_WW, 0, -1);
            const double u_zp = P_(Q_UU, 0, 0), u_zm = M_(Q_UU, 0, 0);
            const double v_zp = P_(Q_VV, 0, 0), v_zm = M_(Q_VV, 0, 0);
            const double w_zp = P_(Q_WW, 0, 0), w_zm = M_(Q_WW, 0, 0);

            // ---- continuity (3dmhdsub.f:1258-1295), one-sided d(RW)/dz on the walls
            double dzrw;
            if (top) dzrw = (4.0 * P_(Q_RW, 0, 0) - rw2) * az;
            else if (bot) dzrw = (rw2 - 4.0 * M_(Q_RW, 0, 0)) * az;
            else dzrw = (P_(Q_RW, 0, 0) - M_(Q_RW, 0, 0)) * az;
            double fr = -((C_(Q_RU, 1, 0) - C_(Q_RU, -1, 0)) * ax + (C_(Q_RV, 0, 1) - C_(Q_RV, 0, -1)) * ay) - dzrw;
            // ---- buoyancy, pressure gradient, advection (1376-1482)
            double fu = -((C_(Q_P, 1, 0) - C_(Q_P, -1, 0)) * ax
                          + (C_(Q_RU, 1, 0) * u_xp - C_(Q_RU, -1, 0) * u_xm) * ax
                          + (C_(Q_RU, 0, 1) * v_yp - C_(Q_RU, 0, -1) * v_ym) * ay
                          + (P_(Q_RU, 0, 0) * w_zp - M_(Q_RU, 0, 0) * w_zm) * az);
            double fv = -((C_(Q_P, 0, 1) - C_(Q_P, 0, -1)) * ay
                          + (C_(Q_RV, 1, 0) * u_xp - C_(Q_RV, -1, 0) * u_xm) * ax
                          + (C_(Q_RV, 0, 1) * v_yp - C_(Q_RV, 0, -1) * v_ym) * ay
                          + (P_(Q_RV, 0, 0) * w_zp - M_(Q_RV, 0, 0) * w_zm) * az);
            double fw = s.grav * ROc
                      - ((P_(Q_P, 0, 0) - M_(Q_P, 0, 0)) * az
                         + (C_(Q_RW, 1, 0) * u_xp - C_(Q_RW, -1, 0) * u_xm) * ax
                         + (C_(Q_RW, 0, 1) * v_yp - C_(Q_RW, 0, -1) * v_ym) * ay
                         + (P_(Q_RW, 0, 0) * w_zp - M_(Q_RW, 0, 0) * w_zm) * az);
            // ---- temperature advection and conduction (1495-1506, 1583-1611)
            double ft;
            {
                const double txp = C_(Q_TT, 1, 0), txm = C_(Q_TT, -1, 0);
                const double typ = C_(Q_TT, 0, 1), tym = C_(Q_TT, 0, -1);
                const double tzp = P_(Q_TT, 0, 0), tzm = M_(Q_TT, 0, 0);
                const double dtx = txp - txm, dty = typ - tym, dtz = tzp - tzm;
                const double lap = dtx * bxq + (txp + txm - 2.0 * TTc) * cxq + dty * byq + (typ + tym - 2.0 * TTc) * cyq
                                 + dtz * bzq + (tzp + tzm - 2.0 * TTc) * czq;
                ft = -(uc * dtx * ax + vc * dty * ay + wc * dtz * az) + RIc * s.tmp_cond * (rka * lap + dka * dtz * az);
            }
            // ---- viscous stress (1818-1886)
            {
                const double lxu = (u_xp - u_xm) * bxq + (u_xp + u_xm - 2.0 * uc) * cxq;
                const double lyu = (u_yp - u_ym) * byq + (u_yp + u_ym - 2.0 * uc) * cyq;
                const double lzu = (u_zp - u_zm) * bzq + (u_zp + u_zm - 2.0 * uc) * czq;
                const double lxv = (v_xp - v_xm) * bxq + (v_xp + v_xm - 2.0 * vc) * cxq;
                const double lyv = (v_yp - v_ym) * byq + (v_yp + v_ym - 2.0 * vc) * cyq;
                const double lzv = (v_zp - v_zm) * bzq + (v_zp + v_zm - 2.0 * vc) * czq;
                const double lxw = (w_xp - w_xm) * bxq + (w_xp + w_xm - 2.0 * wc) * cxq;
                const double lyw = (w_yp - w_ym) * byq + (w_yp + w_ym - 2.0 * wc) * cyq;
                const double lzw = (w_zp - w_zm) * bzq + (w_zp + w_zm - 2.0 * wc) * czq;
                fu += s.ore * (s.c43 * lxu + lyu + lzu);
                fv += s.ore * (lxv + s.c43 * lyv + lzv);
                fw += s.ore * (lxw + lyw + s.c43 * lzw);
            }
            // ---- velocity gradients, the 19-point cross terms, heating (1891-2101)
            const double ux = (u_xp - u_xm) * ax, vx = (v_xp - v_xm) * ax, wx = (w_xp - w_xm) * ax;
            const double uy = (u_yp - u_ym) * ay, vy = (v_yp - v_ym) * ay, wy = (w_yp - w_ym) * ay;
            const double uz = (u_zp - u_zm) * az, vz = (v_zp - v_zm) * az, wz = (w_zp - w_zm) * az;
            {
                const double axy = ax * ay, axz = ax * az, ayz = ay * az;
                const double dyvx = ((C_(Q_VV, 1, 1) - C_(Q_VV, -1, 1)) - (C_(Q_VV, 1, -1) - C_(Q_VV, -1, -1))) * axy;
                const double dyux = ((C_(Q_UU, 1, 1) - C_(Q_UU, -1, 1)) - (C_(Q_UU, 1, -1) - C_(Q_UU, -1, -1))) * axy;
                const double dxwz = ((P_(Q_WW, 1, 0) - M_(Q_WW, 1, 0)) - (P_(Q_WW, -1, 0) - M_(Q_WW, -1, 0))) * axz;
                const double dywz = ((P_(Q_WW, 0, 1) - M_(Q_WW, 0, 1)) - (P_(Q_WW, 0, -1) - M_(Q_WW, 0, -1))) * ayz;
                const double dxuz = ((P_(Q_UU, 1, 0) - M_(Q_UU, 1, 0)) - (P_(Q_UU, -1, 0) - M_(Q_UU, -1, 0))) * axz;
                const double dyvz = ((P_(Q_VV, 0, 1) - M_(Q_VV, 0, 1)) - (P_(Q_VV, 0, -1) - M_(Q_VV, 0, -1))) * ayz;
                fu += s.tmp_13 * (dyvx + dxwz);
                fv += s.tmp_13 * (dyux + dywz);
                fw += s.tmp_13 * (dxuz + dyvz);
            }
            double heat = s.tmp_a * (s.c43 * ux * ux + vx * vx + wx * wx + uy * uy + 2.0 * uy * vx + uz * uz + vz * vz
                                     + wy * wy + 2.0 * vz * wy + 2.0 * uz * wx)
                        + s.tmp_b * (vy * vy + wz * wz - ux * wz - ux * vy - vy * wz);
            ft -= s.ocv * TTc * (ux + vy + wz);
            // ---- Coriolis (2106-2125)
            if (ROT) {
                fu += s.omz * RVc;
                fv += s.omx * RWc - s.omz * RUc;
                fw -= s.omx * RVc;
            }
            // ---- induction, Lorentz force, Ohmic heating (2129-2634)
            double w1 = 0, w2 = 0, w3 = 0;
            if (MAG) {
                const double BXc = BXc0, BYc = BYc0, BZc = BZc0;
                const double bxxp = C_(Q_BX, 1, 0), bxxm = C_(Q_BX, -1, 0), bxyp = C_(Q_BX, 0, 1), bxym = C_(Q_BX, 0, -1);
                const double byxp = C_(Q_BY, 1, 0), byxm = C_(Q_BY, -1, 0), byyp = C_(Q_BY, 0, 1), byym = C_(Q_BY, 0, -1);
                const double bzxp = C_(Q_BZ, 1, 0), bzxm = C_(Q_BZ, -1, 0), bzyp = C_(Q_BZ, 0, 1), bzym = C_(Q_BZ, 0, -1);
                const double bxzp = P_(Q_BX, 0, 0), bxzm = M_(Q_BX, 0, 0);
                const double byzp = P_(Q_BY, 0, 0), byzm = M_(Q_BY, 0, 0);
                const double bzzp = P_(Q_BZ, 0, 0), bzzm = M_(Q_BZ, 0, 0);
                const double bxx = (bxxp - bxxm) * ax, byx = (byxp - byxm) * ax, bzx = (bzxp - bzxm) * ax;
                const double bxy = (bxyp - bxym) * ay, byy = (byyp - byym) * ay, bzy = (bzyp - bzym) * ay;
                const double bxz = (bxzp - bxzm) * az, byz = (byzp - byzm) * az, bzz = (bzzp - bzzm) * az;
                double wzm = wz, lzbx, lzby;
                if (top) {
                    wzm = (4.0 * w_zp - ww2) * az;
                    lzbx = (-3.0 * BXc + 4.0 * bxzp - bx2) * bzq + (2.0 * BXc - 5.0 * bxzp + 4.0 * bx2 - bx3) * czq;
                    lzby = (-3.0 * BYc + 4.0 * byzp - by2) * bzq + (2.0 * BYc - 5.0 * byzp + 4.0 * by2 - by3) * czq;
                } else if (bot) {
                    wzm = (ww2 - 4.0 * w_zm) * az;
                    lzbx = (3.0 * BXc - 4.0 * bxzm + bx2) * bzq + (2.0 * BXc - 5.0 * bxzm + 4.0 * bx2 - bx3) * czq;
                    lzby = (3.0 * BYc - 4.0 * byzm + by2) * bzq + (2.0 * BYc - 5.0 * byzm + 4.0 * by2 - by3) * czq;
                } else {
                    lzbx = (bxzp - bxzm) * bzq + (bxzp + bxzm - 2.0 * BXc) * czq;
                    lzby = (byzp - byzm) * bzq + (byzp + byzm - 2.0 * BYc) * czq;
                }
                const double lbx = (bxxp - bxxm) * bxq + (bxxp + bxxm - 2.0 * BXc) * cxq
                                 + (bxyp - bxym) * byq + (bxyp + bxym - 2.0 * BXc) * cyq + lzbx;
                const double lby = (byxp - byxm) * bxq + (byxp + byxm - 2.0 * BYc) * cxq
                                 + (byyp - byym) * byq + (byyp + byym - 2.0 * BYc) * cyq + lzby;
                const double lbz = (bzxp - bzxm) * bxq + (bzxp + bzxm - 2.0 * BZc) * cxq
                                 + (bzyp - bzym) * byq + (bzyp + bzym - 2.0 * BZc) * cyq
                                 + (bzzp - bzzm) * bzq + (bzzp + bzzm - 2.0 * BZc) * czq;
                w1 = BYc * uy - BXc * vy + BZc * uz - BXc * wzm - (uc * bxx + vc * bxy + wc * bxz) + s.orm * lbx;
                w2 = BXc * vx - BYc * ux + BZc * vz - BYc * wzm - (uc * byx + vc * byy + wc * byz) + s.orm * lby;
                w3 = BXc * wx - BZc * ux + BYc * wy - BZc * vy - (uc * bzx + vc * bzy + wc * bzz) + s.orm * lbz;
                const double jz = bxy - byx, jy = bxz - bzx, jx = byz - bzy;
                fu += s.obeta * (BYc * jz + BZc * jy);
                fv += s.obeta * (BZc * jx - BXc * jz);
                fw -= s.obeta * (BXc * jy + BYc * jx);
                heat += s.tmp_m * (jx * jx + jy * jy + jz * jz);
            }
            ft += RIc * heat;
#else
            const bool top = (k == 0), bot = (k == npz - 1);
            const double dzk = m.dzzdz[k + 1], d2zk = m.d2zzdz2[k + 1];
            const double rka = m.rkapa[k + 1], dka = m.dkapa[k + 1];
            const double tmpy = HY * dyj, tmpz = HZ * dzk;
            const double tmpz1 = HZ * d2zk, tmpz2 = H2Z * dzk * dzk;
            const double tmpy1 = HY * d2yj, tmpy2 = H2Y * dyj * dyj;

            WALL_LOADS

            const double RUc = C_(Q_RU, 0, 0), RVc = C_(Q_RV, 0, 0), RWc = C_(Q_RW, 0, 0);
            const double ROc = C_(Q_RO, 0, 0), TTc = C_(Q_TT, 0, 0), RIc = C_(Q_RI, 0, 0);
            const double UUc = C_(Q_UU, 0, 0), VVc = C_(Q_VV, 0, 0), WWc = C_(Q_WW, 0, 0);
            const double BXc0 = MAG ? C_(Q_BX, 0, 0) : 0.0, BYc0 = MAG ? C_(Q_BY, 0, 0) : 0.0;
            const double BZc0 = MAG ? C_(Q_BZ, 0, 0) : 0.0;

            // ---- continuity: loops 10, 40-60, 70 (3dmhdsub.f:1258-1295)
            double fr = (C_(Q_RU, -1, 0) - C_(Q_RU, 1, 0)) * HX * dxi;
            fr = fr - (C_(Q_RV, 0, 1) - C_(Q_RV, 0, -1)) * tmpy;
            double dwz;
            if (top) dwz = (4.0 * P_(Q_RW, 0, 0) - rw2) * tmpz;
            else if (bot) dwz = (rw2 - 4.0 * M_(Q_RW, 0, 0)) * tmpz;
            else dwz = (P_(Q_RW, 0, 0) - M_(Q_RW, 0, 0)) * tmpz;
            fr = fr - dwz;
            // ---- buoyancy and pressure gradient: loops 80, 120 (1376-1404)
            double fw = s.grav * ROc;
            fw = fw - (P_(Q_P, 0, 0) - M_(Q_P, 0, 0)) * tmpz;
            double fv = (C_(Q_P, 0, -1) - C_(Q_P, 0, 1)) * tmpy;
            double fu = (C_(Q_P, -1, 0) - C_(Q_P, 1, 0)) * HX * dxi;
            // ---- momentum advection: loops 210, 280, 330 (1435-1482)
            fu = fu - (C_(Q_RU, 1, 0) * C_(Q_UU, 1, 0) - C_(Q_RU, -1, 0) * C_(Q_UU, -1, 0)) * HX * dxi;
            fu = fu - (C_(Q_RU, 0, 1) * C_(Q_VV, 0, 1) - C_(Q_RU, 0, -1) * C_(Q_VV, 0, -1)) * tmpy;
            fu = fu - (P_(Q_RU, 0, 0) * P_(Q_WW, 0, 0) - M_(Q_RU, 0, 0) * M_(Q_WW, 0, 0)) * tmpz;
            fv = fv - (C_(Q_RV, 1, 0) * C_(Q_UU, 1, 0) - C_(Q_RV, -1, 0) * C_(Q_UU, -1, 0)) * HX * dxi;
            fv = fv - (C_(Q_RV, 0, 1) * C_(Q_VV, 0, 1) - C_(Q_RV, 0, -1) * C_(Q_VV, 0, -1)) * tmpy;
            fv = fv - (P_(Q_RV, 0, 0) * P_(Q_WW, 0, 0) - M_(Q_RV, 0, 0) * M_(Q_WW, 0, 0)) * tmpz;
            fw = fw - (C_(Q_RW, 1, 0) * C_(Q_UU, 1, 0) - C_(Q_RW, -1, 0) * C_(Q_UU, -1, 0)) * HX * dxi;
            fw = fw - (C_(Q_RW, 0, 1) * C_(Q_VV, 0, 1) - C_(Q_RW, 0, -1) * C_(Q_VV, 0, -1)) * tmpy;
            fw = fw - (P_(Q_RW, 0, 0) * P_(Q_WW, 0, 0) - M_(Q_RW, 0, 0) * M_(Q_WW, 0, 0)) * tmpz;
            // ---- temperature advection: loop 450 (1495-1506)
            double ft = -(1.0 * UUc * (C_(Q_TT, 1, 0) - C_(Q_TT, -1, 0)) * HX * dxi);
            ft = ft - VVc * (C_(Q_TT, 0, 1) - C_(Q_TT, 0, -1)) * tmpy;
            ft = ft - WWc * (P_(Q_TT, 0, 0) - M_(Q_TT, 0, 0)) * tmpz;
            // ---- conduction, non-LREM: loop 519 (1583-1611)
            {
                const double TMP = s.tmp_cond;
                const double txp = C_(Q_TT, 1, 0), txm = C_(Q_TT, -1, 0);
                const double typ = C_(Q_TT, 0, 1), tym = C_(Q_TT, 0, -1);
                const double tzp = P_(Q_TT, 0, 0), tzm = M_(Q_TT, 0, 0);
                ft = ft + ((txp - txm) * HX * d2xi + (txp - 2.0 * TTc + txm) * H2X * dxi * dxi) * RIc * TMP * rka;
                ft = ft + ((typ - tym) * tmpy1 + (typ - 2.0 * TTc + tym) * tmpy2) * RIc * TMP * rka;
                ft = ft + ((tzp - tzm) * tmpz1 + (tzp - 2.0 * TTc + tzm) * tmpz2) * RIc * TMP * rka;
                ft = ft + (tzp - tzm) * HZ * dzk * RIc * TMP * dka;
            }
            // ---- viscous momentum terms: loops 530, 540, 550 (1818-1886)
            {
                const double uxp = C_(Q_UU, 1, 0), uxm = C_(Q_UU, -1, 0), uyp = C_(Q_UU, 0, 1), uym = C_(Q_UU, 0, -1);
                const double uzp = P_(Q_UU, 0, 0), uzm = M_(Q_UU, 0, 0);
                fu = fu + ORE * (C43 * ((uxp - uxm) * HX * d2xi + (uxp - 2.0 * UUc + uxm) * H2X * dxi * dxi)
                                 + (uyp - uym) * tmpy1 + (uyp - 2.0 * UUc + uym) * tmpy2
                                 + (uzp - uzm) * tmpz1 + (uzp - 2.0 * UUc + uzm) * tmpz2);
                const double vxp = C_(Q_VV, 1, 0), vxm = C_(Q_VV, -1, 0), vyp = C_(Q_VV, 0, 1), vym = C_(Q_VV, 0, -1);
                const double vzp = P_(Q_VV, 0, 0), vzm = M_(Q_VV, 0, 0);
                fv = fv + ORE * ((vxp - vxm) * HX * d2xi + (vxp - 2.0 * VVc + vxm) * H2X * dxi * dxi
                                 + C43 * ((vyp - vym) * tmpy1 + (vyp - 2.0 * VVc + vym) * tmpy2)
                                 + (vzp - vzm) * tmpz1 + (vzp - 2.0 * VVc + vzm) * tmpz2);
                const double wxp = C_(Q_WW, 1, 0), wxm = C_(Q_WW, -1, 0), wyp = C_(Q_WW, 0, 1), wym = C_(Q_WW, 0, -1);
                const double wzp = P_(Q_WW, 0, 0), wzm = M_(Q_WW, 0, 0);
                fw = fw + ORE * ((wxp - wxm) * HX * d2xi + (wxp - 2.0 * WWc + wxm) * H2X * dxi * dxi
                                 + (wyp - wym) * tmpy1 + (wyp - 2.0 * WWc + wym) * tmpy2
                                 + C43 * ((wzp - wzm) * tmpz1 + (wzp - 2.0 * WWc + wzm) * tmpz2));
            }
            // ---- viscous and compressional heating, (1/3)grad(div u): loops 650-940 (1891-2101)
            const double TA = s.tmp_a, TB = s.tmp_b, T13 = s.tmp_13;
            const double ux = (C_(Q_UU, 1, 0) - C_(Q_UU, -1, 0)) * HX * dxi;
            const double ux_p = (C_(Q_UU, 1, 1) - C_(Q_UU, -1, 1)) * HX * dxi;
            const double ux_m = (C_(Q_UU, 1, -1) - C_(Q_UU, -1, -1)) * HX * dxi;
            const double vx = (C_(Q_VV, 1, 0) - C_(Q_VV, -1, 0)) * HX * dxi;
            const double vx_p = (C_(Q_VV, 1, 1) - C_(Q_VV, -1, 1)) * HX * dxi;
            const double vx_m = (C_(Q_VV, 1, -1) - C_(Q_VV, -1, -1)) * HX * dxi;
            const double wx = (C_(Q_WW, 1, 0) - C_(Q_WW, -1, 0)) * HX * dxi;
            ft = ft + (C43 * ux * ux + vx * vx + wx * wx) * RIc * TA;             // 700
            ft = ft - OCV * ux * TTc;                                            // 710
            fu = fu + T13 * (vx_p - vx_m) * HY * dyj;                            // 720
            fv = fv + T13 * (ux_p - ux_m) * HY * dyj;                            // 730
            const double uy = (C_(Q_UU, 0, 1) - C_(Q_UU, 0, -1)) * HY * dyj;     // 740
            ft = ft + (uy * uy + 2.0 * uy * vx) * RIc * TA;                      // 750
            const double vy = (C_(Q_VV, 0, 1) - C_(Q_VV, 0, -1)) * HY * dyj;     // 755
            ft = ft + vy * vy * RIc * TB;                                        // 760
            ft = ft - OCV * vy * TTc;                                            // 770
            const double wz = (P_(Q_WW, 0, 0) - M_(Q_WW, 0, 0)) * HZ * dzk;      // 790
            const double wz_xp = (P_(Q_WW, 1, 0) - M_(Q_WW, 1, 0)) * HZ * dzk;
            const double wz_xm = (P_(Q_WW, -1, 0) - M_(Q_WW, -1, 0)) * HZ * dzk;
            const double wz_yp = (P_(Q_WW, 0, 1) - M_(Q_WW, 0, 1)) * HZ * dzk;
            const double wz_ym = (P_(Q_WW, 0, -1) - M_(Q_WW, 0, -1)) * HZ * dzk;
            ft = ft + (wz * wz - ux * wz - ux * vy - vy * wz) * RIc * TB;        // 820
            ft = ft - OCV * wz * TTc;                                            // 830
            fu = fu + T13 * (wz_xp - wz_xm) * HX * dxi;                          // 840
            fv = fv + T13 * (wz_yp - wz_ym) * HY * dyj;                          // 850
            const double uz = (P_(Q_UU, 0, 0) - M_(Q_UU, 0, 0)) * HZ * dzk;      // 860
            const double uz_xp = (P_(Q_UU, 1, 0) - M_(Q_UU, 1, 0)) * HZ * dzk;
            const double uz_xm = (P_(Q_UU, -1, 0) - M_(Q_UU, -1, 0)) * HZ * dzk;
            const double vz = (P_(Q_VV, 0, 0) - M_(Q_VV, 0, 0)) * HZ * dzk;      // 880
            const double vz_yp = (P_(Q_VV, 0, 1) - M_(Q_VV, 0, 1)) * HZ * dzk;
            const double vz_ym = (P_(Q_VV, 0, -1) - M_(Q_VV, 0, -1)) * HZ * dzk;
            const double wy = (C_(Q_WW, 0, 1) - C_(Q_WW, 0, -1)) * HY * dyj;     // 900
            ft = ft + (uz * uz + vz * vz + wy * wy + 2.0 * vz * wy) * RIc * TA;  // 910
            fw = fw + T13 * ((uz_xp - uz_xm) * HX * dxi + (vz_yp - vz_ym) * HY * dyj);  // 920
            ft = ft + 2.0 * uz * wx * RIc * TA;                                  // 940
            // ---- Coriolis: loops 950-970 (2106-2125)
            if (ROT) {
                fu = fu + s.omz * RVc;
                fv = fv - s.omz * RUc + s.omx * RWc;
                fw = fw - s.omx * RVc;
            }
            // ---- induction, Lorentz force, Ohmic heating: 2129-2634
            double w1 = 0, w2 = 0, w3 = 0;
            if (MAG) {
                const double OBETA = s.obeta, ORM = s.orm, TM = s.tmp_m;
                const double BXc = C_(Q_BX, 0, 0), BYc = C_(Q_BY, 0, 0), BZc = C_(Q_BZ, 0, 0);
                w2 = BXc * vx - BYc * ux;                                        // 1030
                w3 = BXc * wx - BZc * ux;                                        // 1040
                w1 = BYc * uy - BXc * vy;                                        // 1080
                w3 = w3 + BYc * wy - BZc * vy;                                   // 1090
                double wzm = wz;                                                 // 1120
                if (top) wzm = (4.0 * P_(Q_WW, 0, 0) - ww2) * HZ * dzk;          // 1125
                else if (bot) wzm = (ww2 - 4.0 * M_(Q_WW, 0, 0)) * HZ * dzk;     // 1126
                w1 = w1 + BZc * uz - BXc * wzm;                                  // 1130
                w2 = w2 + BZc * vz - BYc * wzm;                                  // 1140
                const double bxxp = C_(Q_BX, 1, 0), bxxm = C_(Q_BX, -1, 0);
                const double byxp = C_(Q_BY, 1, 0), byxm = C_(Q_BY, -1, 0);
                const double bzxp = C_(Q_BZ, 1, 0), bzxm = C_(Q_BZ, -1, 0);
                const double bxyp = C_(Q_BX, 0, 1), bxym = C_(Q_BX, 0, -1);
                const double byyp = C_(Q_BY, 0, 1), byym = C_(Q_BY, 0, -1);
                const double bzyp = C_(Q_BZ, 0, 1), bzym = C_(Q_BZ, 0, -1);
                const double bxzp = P_(Q_BX, 0, 0), bxzm = M_(Q_BX, 0, 0);
                const double byzp = P_(Q_BY, 0, 0), byzm = M_(Q_BY, 0, 0);
                const double bzzp = P_(Q_BZ, 0, 0), bzzm = M_(Q_BZ, 0, 0);
                const double bxx = (bxxp - bxxm) * HX * dxi;                     // 1150
                const double byx = (byxp - byxm) * HX * dxi;                     // 1160
                const double bzx = (bzxp - bzxm) * HX * dxi;                     // 1170
                const double bxy = (bxyp - bxym) * HY * dyj;                     // 1180
                fu = fu + OBETA * BYc * (bxy - byx) - OBETA * BZc * bzx;         // 1190
                fv = fv + OBETA * BXc * (byx - bxy);                             // 1200
                fw = fw + OBETA * BXc * bzx;                                     // 1210
                ft = ft + (bxy * bxy + byx * byx + bzx * bzx - 2.0 * byx * bxy) * RIc * TM;  // 1220
                w1 = w1 - UUc * bxx - VVc * bxy;                                 // 1230
                w2 = w2 - UUc * byx;                                             // 1240
                w3 = w3 - UUc * bzx;                                             // 1250
                const double bxx2 = (bxxp - bxxm) * HX * d2xi + (bxxp - 2.0 * BXc + bxxm) * H2X * dxi * dxi;  // 1260
                const double byx2 = (byxp - byxm) * HX * d2xi + (byxp - 2.0 * BYc + byxm) * H2X * dxi * dxi;  // 1265
                const double bxy2 = (bxyp - bxym) * HY * d2yj + (bxyp - 2.0 * BXc + bxym) * H2Y * dyj * dyj;  // 1270
                w1 = w1 + ORM * (bxx2 + bxy2);                                   // 1280
                w2 = w2 + ORM * byx2;                                            // 1290
                const double bzx2 = (bzxp - bzxm) * HX * d2xi + (bzxp - 2.0 * BZc + bzxm) * H2X * dxi * dxi;  // 1300
                w3 = w3 + ORM * bzx2;                                            // 1310
                const double bxz = (bxzp - bxzm) * HZ * dzk;                     // 1320
                const double byy = (byyp - byym) * HY * dyj;                     // 1330
                fu = fu + OBETA * BZc * bxz;                                     // 1340
                fw = fw - OBETA * BXc * bxz;                                     // 1350
                ft = ft + (bxz * bxz - 2.0 * bxz * bzx) * RIc * TM;              // 1360
                w1 = w1 - WWc * bxz;                                             // 1370
                w2 = w2 - VVc * byy;                                             // 1380
                double bxz2;                                                     // 1390-1392
                if (top)
                    bxz2 = (-3.0 * BXc + 4.0 * bxzp - bx2) * HZ * d2zk
                         + (2.0 * BXc - 5.0 * bxzp + 4.0 * bx2 - bx3) * H2Z * dzk * dzk;
                else if (bot)
                    bxz2 = (3.0 * BXc - 4.0 * bxzm + bx2) * HZ * d2zk
                         + (2.0 * BXc - 5.0 * bxzm + 4.0 * bx2 - bx3) * H2Z * dzk * dzk;
                else
                    bxz2 = (bxzp - bxzm) * HZ * d2zk + (bxzp - 2.0 * BXc + bxzm) * H2Z * dzk * dzk;
                const double byy2 = (byyp - byym) * HY * d2yj + (byyp - 2.0 * BYc + byym) * H2Y * dyj * dyj;  // 1400
                w1 = w1 + ORM * bxz2;                                            // 1410
                w2 = w2 + ORM * byy2;                                            // 1420
                const double byz = (byzp - byzm) * HZ * dzk;                     // 1430
                const double bzy = (bzyp - bzym) * HY * dyj;                     // 1440
                const double cur = byz - bzy;                                    // 1450
                fv = fv + OBETA * BZc * cur;                                     // 1460
                fw = fw - OBETA * BYc * cur;                                     // 1470
                ft = ft + (byz * byz + bzy * bzy - 2.0 * byz * bzy) * RIc * TM;  // 1480
                w2 = w2 - WWc * byz;                                             // 1490
                w3 = w3 - VVc * bzy;                                             // 1500
                double byz2;                                                     // 1510-1513
                if (top)
                    byz2 = (-3.0 * BYc + 4.0 * byzp - by2) * HZ * d2zk
                         + (2.0 * BYc - 5.0 * byzp + 4.0 * by2 - by3) * H2Z * dzk * dzk;
                else if (bot)
                    byz2 = (3.0 * BYc - 4.0 * byzm + by2) * HZ * d2zk
                         + (2.0 * BYc - 5.0 * byzm + 4.0 * by2 - by3) * H2Z * dzk * dzk;
                else
                    byz2 = (byzp - byzm) * HZ * d2zk + (byzp - 2.0 * BYc + byzm) * H2Z * dzk * dzk;
                const double bzy2 = (bzyp - bzym) * HY * d2yj + (bzyp - 2.0 * BZc + bzym) * H2Y * dyj * dyj;  // 1520
                w2 = w2 + ORM * byz2;                                            // 1530
                w3 = w3 + ORM * bzy2;                                            // 1540
                const double bzz = (bzzp - bzzm) * HZ * dzk;                     // 1550
                w3 = w3 - WWc * bzz;                                             // 1560
                const double bzz2 = (bzzp - bzzm) * HZ * d2zk + (bzzp - 2.0 * BZc + bzzm) * H2Z * dzk * dzk;  // 1570
                w3 = w3 + ORM * bzz2;                                            // 1580
            }
#endif
            // ghost RO planes: this FLUXES call leaves 1/RO behind (3dmhdsub.f:1386-1391)
            if (STAGE != 0) {
                if (top) store_cell<1>(a.u_out, a.uf, ucol, hc, {F_RO}, {M_(Q_RI, 0, 0)});
                if (bot) store_cell<1>(a.u_out + (size_t)(npz + 1) * a.uz, a.uf, ucol, hc, {F_RO}, {P_(Q_RI, 0, 0)});
            }
#undef C_
#undef M_
#undef P_
#undef WALL_LOADS
            const bool wall = top || bot;
            const size_t zc = (size_t)k * a.zz + zcol;
            if (STAGE == 0) {
                // right-hand sides; values BCON discards on the walls are reported as 0
                a.f_out[zc + 0 * a.zf] = wall ? 0.0 : fu;
                a.f_out[zc + 1 * a.zf] = wall ? 0.0 : fv;
                a.f_out[zc + 2 * a.zf] = wall ? 0.0 : fw;
                a.f_out[zc + 3 * a.zf] = fr;
                a.f_out[zc + 4 * a.zf] = wall ? 0.0 : ft;
                if (MAG) {
                    a.f_out[zc + 5 * a.zf] = w1;
                    a.f_out[zc + 6 * a.zf] = w2;
                    a.f_out[zc + 7 * a.zf] = wall ? 0.0 : w3;
                }
            } else {
                // ---- RK3 update: U = Z + COEF*F (STEP loops 70-140, 270-340, 470-540);
                //      stage 1 has Z = U (loops 71-141)
                double zu, zv, zw, zr, zt, zbx = 0, zby = 0, zbz = 0;
                if (STAGE == 1) {
                    zu = RUc; zv = RVc; zw = RWc; zr = ROc; zt = TTc;
                    if (MAG) { zbx = BXc0; zby = BYc0; zbz = BZc0; }
                } else {
                    zok = wait_z(k);
                    const double* zt_ = sz + (size_t)((k - k0) & 1) * L::ZT + ty * TX + tx;
                    zu = zt_[F_RU * TY * TX];
                    zv = zt_[F_RV * TY * TX];
                    zw = zt_[F_RW * TY * TX];
                    zt = zt_[F_TT * TY * TX];
                    zr = zt_[F_RO * TY * TX];
                    if (MAG) {
                        zbx = zt_[F_BX * TY * TX];
                        zby = zt_[F_BY * TY * TX];
                        zbz = zt_[F_BZ * TY * TX];
                    }
                }
                const double nu = zu + cu * fu, nv = zv + cu * fv, nw = zw + cu * fw;
                const double nr = zr + cu * fr, nt = zt + cu * ft;
                const double nbx = zbx + cu * w1, nby = zby + cu * w2, nbz = zbz + cu * w3;
                const int kz = k + 1;
                if (zok) {
                    // on the walls RU, RV, RW, TT, BZ are rewritten by BCON below
                    double* const pl = a.u_out + (size_t)kz * a.uz;
                    if (MAG)
                        store_cell<8>(pl, a.uf, ucol, hc, {F_RO, F_BX, F_BY, F_RU, F_RV, F_RW, F_TT, F_BZ},
                                      {nr, nbx, nby, nu, nv, nw, nt, nbz});
                    else
                        store_cell<5>(pl, a.uf, ucol, hc, {F_RO, F_RU, F_RV, F_RW, F_TT}, {nr, nu, nv, nw, nt});
                    // ---- Z for the next stage: Z = U + ZETA*DT*F (loops 190-260, 390-460).
                    //      On the walls only RO, BX, BY are ever read back.
                    if (STAGE < 3) {
                        double* zo = a.z + zc;
                        zo[F_RO * a.zf] = nr + cz * fr;
                        if (MAG) {
                            zo[F_BX * a.zf] = nbx + cz * w1;
                            zo[F_BY * a.zf] = nby + cz * w2;
                        }
                        if (!wall) {
                            zo[F_RU * a.zf] = nu + cz * fu;
                            zo[F_RV * a.zf] = nv + cz * fv;
                            zo[F_RW * a.zf] = nw + cz * fw;
                            zo[F_TT * a.zf] = nt + cz * ft;
                            if (MAG) zo[F_BZ * a.zf] = nbz + cz * w3;
                        }
                    }
                }
                // ---- BCON (3dmhdsub.f:2751-2955) and the CFL parts of the next step
                if (!top && !bot) {
                    if (STAGE == 3) cfl_acc_cell<MAG>(cfa, s, m, cfl_screen_of(red), ccol, gi, gj, k, nu, nv, nw, nr, nt, nbx, nby, nbz);
                }
                if (k == 2 && k0 == 0) {
                    // top wall: new values of planes K=3 (read back) and K=4 (this plane);
                    // this thread wrote planes K=2 and K=3 of u_out itself
                    const double* ub = a.u_out + ucol;
                    const size_t c0 = 1 * a.uz, c1 = 2 * a.uz;
                    const double h1_ru = ub[F_RU * a.uf + c1], h1_rv = ub[F_RV * a.uf + c1];
                    const double h1_ro = ub[F_RO * a.uf + c1], h1_tt = ub[F_TT * a.uf + c1];
                    const double w0_ro = ub[F_RO * a.uf + c0], w0_tt = ub[F_TT * a.uf + c0];
                    const double w0_bx = MAG ? ub[F_BX * a.uf + c0] : 0.0, w0_by = MAG ? ub[F_BY * a.uf + c0] : 0.0;
                    const double w0_bz = MAG ? ub[F_BZ * a.uf + c0] : 0.0;
                    const double ru_w = w0_ro * (C43 * h1_ru / h1_ro - C13 * nu / nr);
                    const double rv_w = w0_ro * (C43 * h1_rv / h1_ro - C13 * nv / nr);
                    double tt_w = w0_tt;
                    if (s.plume) {
                        const double tpr = (s.tc != 0.0) ? s.tp + (1.0 - s.tp) * exp(-ctl->timt / s.tc) : s.tp;
                        const double gx = m.plume_gx[gi + 1], gy = m.plume_gy[gj + 1];
                        if (s.itcon == 0) tt_w = 1.0 - (1.0 - tpr) * gx / s.hh * gy / s.hh;
                        else tt_w = C43 * h1_tt - C13 * nt - C23 * s.top_dz * (s.theta - (s.theta - tpr) * gx / s.hh * gy / s.hh);
                    } else if (s.itcon == 0 || s.itcon == 2 || s.itcon == 4) {
                        tt_w = 1.0;
                        if (s.itcon == 4 && gi + 2 <= (npx + 2) / 2) tt_w = 1.0 - s.tp;
                    } else if (s.itcon == 1) {
                        tt_w = C43 * h1_tt - C13 * nt - s.top_flux;
                    }
                    const double bz_w = (MAG && s.ibcon == 0) ? 0.0 : w0_bz;
                    if (zok) {
                        double* const pl = a.u_out + a.uz;
                        if (MAG)
                            store_cell<5>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT, F_BZ}, {ru_w, rv_w, 0.0, tt_w, bz_w});
                        else
                            store_cell<4>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT}, {ru_w, rv_w, 0.0, tt_w});
                    }
                    if (STAGE == 3)
                        cfl_acc_direct<MAG>(cfa, s, m, cfl_screen_of(red), ccol, gi, gj, 0, ru_w, rv_w, 0.0, w0_ro, tt_w, w0_bx, w0_by, bz_w);
                }
                if (bot) {
                    // bottom wall: new values of planes K=NZ-2 and K=NZ-3, read back
                    const double* ub = a.u_out + ucol;
                    const size_t c1 = (size_t)(npz - 1) * a.uz, c2 = (size_t)(npz - 2) * a.uz;
                    const double h1_ru = ub[F_RU * a.uf + c1], h1_rv = ub[F_RV * a.uf + c1];
                    const double h1_ro = ub[F_RO * a.uf + c1], h1_tt = ub[F_TT * a.uf + c1];
                    const double h2_ru = ub[F_RU * a.uf + c2], h2_rv = ub[F_RV * a.uf + c2];
                    const double h2_ro = ub[F_RO * a.uf + c2], h2_tt = ub[F_TT * a.uf + c2];
                    const double ru_w = nr * (C43 * h1_ru / h1_ro - C13 * h2_ru / h2_ro);
                    const double rv_w = nr * (C43 * h1_rv / h1_ro - C13 * h2_rv / h2_ro);
                    const double tt_w = (s.izcon == 0) ? s.tb : C43 * h1_tt - C13 * h2_tt + s.bot_flux;
                    const double bz_w = (MAG && s.ibcon == 0) ? 0.0 : nbz;
                    if (zok) {
                        double* const pl = a.u_out + (size_t)kz * a.uz;
                        if (MAG)
                            store_cell<5>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT, F_BZ}, {ru_w, rv_w, 0.0, tt_w, bz_w});
                        else
                            store_cell<4>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT}, {ru_w, rv_w, 0.0, tt_w});
                    }
                    if (STAGE == 3) cfl_acc_cell<MAG>(cfa, s, m, cfl_screen_of(red), ccol, gi, gj, k, ru_w, rv_w, 0.0, nr, tt_w, nbx, nby, bz_w);
                }
            }
        } else if (STAGE >= 2) {
            // columns outside the domain still see the Z fill of this plane land
            zok = wait_z(k);
        }
        if (!zok) atomicOr(sflag, 1);
        if (STAGE == 3) cfl_fold_plane(red, cfa, m.rkapa[k + 1], s);
        __syncthreads();
        if (*sflag) break;
        // refill: plane k+NRAW-1 goes to the slot plane k-1 has left
        if (tid == 0 && k + NRAW - 1 <= k1) issue_plane(k + NRAW - 1);
    }
    if (*sflag) {
        // a bounded wait gave up: let every fill still in flight land (again
        // bounded), report, and leave without touching the reduction
        if (tid == 0) {
            // the last fill of each slot is one of the NRAW highest planes issued
            for (int kp = hi_issued - (NRAW - 1); kp <= hi_issued; ++kp)
                if (kp >= k0 - 1) mbar_wait(&bars[(kp + 1) % NRAW], parity_of(kp));
            // and the last fill of each Z slot is one of the two highest Z planes issued
            for (int kp = z_hi - 1; kp <= z_hi; ++kp)
                if (kp >= k0) wait_z(kp);
            atomicExch(&a.ctl->status, MHD3D_ERR_TIMEOUT);
            atomicExch(&a.ctl->stop, 1);
        }
        return;
    }
    if (STAGE == 3) cfl_commit_acc(a.acc, red, cfa);
}

// Standalone CFL reduction over the current state (STEP 3dmhdsub.f:741-873),
// used before the first step and after a state change.
template <bool MAG>
__global__ void __launch_bounds__(NT) k_cfl(const __grid_constant__ StageArgs a)
{
    const Scalars& s = a.s;
    const int npx = s.npx, npy = s.npy, npz = s.npz;
    const size_t ncell = (size_t)npx * npy * npz;
    unsigned long long kw1 = ~0ull, kw2 = ~0ull, kw3 = ~0ull, kw4 = ~0ull, kmu = 0ull;
    unsigned int bad = 0;
    for (size_t q = (size_t)blockIdx.x * NT + threadIdx.x; q < ncell; q += (size_t)gridDim.x * NT) {
        const int gi = (int)(q % npx);
        const int gj = (int)((q / npx) % npy);
        const int k = (int)(q / ((size_t)npx * npy));
        const double* u = a.u_in + (size_t)(k + 1) * a.uz + (size_t)(gj + 1) * a.upitch + (gi + 1);
        CflPart cp;
        cfl_cell<MAG>(s, u[F_RU * a.uf], u[F_RV * a.uf], u[F_RW * a.uf], u[F_RO * a.uf], u[F_TT * a.uf],
                      MAG ? u[F_BX * a.uf] : 0.0, MAG ? u[F_BY * a.uf] : 0.0, MAG ? u[F_BZ * a.uf] : 0.0,
                      cell_dd(a.m, gi, gj, k), a.m.rkapa[k + 1], cp);
        kw1 = min(kw1, key_of(cp.w1)); kw2 = min(kw2, key_of(cp.w2));
        kw3 = min(kw3, key_of(cp.w3)); kw4 = min(kw4, key_of(cp.w4));
        kmu = max(kmu, key_of(cp.mach2)); bad |= cp.bad;
    }
    __shared__ unsigned long long red[(NT / 32) * 6];
    cfl_commit(a.acc, kw1, kw2, kw3, kw4, kmu, bad, red);
}

// Standalone BCON on the current state, in place (test entry point).
template <bool MAG>
__global__ void __launch_bounds__(NT) k_bcon(const __grid_constant__ StageArgs a)
{
    const Scalars& s = a.s;
    const int npx = s.npx, npy = s.npy, npz = s.npz;
    const int q = blockIdx.x * NT + threadIdx.x;
    if (q >= npx * npy) return;
    const int gi = q % npx, gj = q / npx;
    double* u = const_cast<double*>(a.u_in);
    const size_t col = (size_t)(gj + 1) * a.upitch + (gi + 1);
    auto at = [&](int f, int k) -> double { return u[(size_t)f * a.uf + (size_t)(k + 1) * a.uz + col]; };
    auto put = [&](int f, int k, double v) { store_u(u, (size_t)f * a.uf, a, gi, gj, k + 1, v); };
    const double C13 = s.c13, C23 = s.c23, C43 = s.c43;
    // top
    {
        const double ro0 = at(F_RO, 0), ro1 = at(F_RO, 1), ro2 = at(F_RO, 2);
        const double ru_w = ro0 * (C43 * at(F_RU, 1) / ro1 - C13 * at(F_RU, 2) / ro2);
        const double rv_w = ro0 * (C43 * at(F_RV, 1) / ro1 - C13 * at(F_RV, 2) / ro2);
        double tt_w = at(F_TT, 0);
        const double t1 = at(F_TT, 1), t2 = at(F_TT, 2);
        if (s.plume) {
            const double tpr = (s.tc != 0.0) ? s.tp + (1.0 - s.tp) * exp(-a.ctl->timt / s.tc) : s.tp;
            const double gx = a.m.plume_gx[gi + 1], gy = a.m.plume_gy[gj + 1];
            if (s.itcon == 0) tt_w = 1.0 - (1.0 - tpr) * gx / s.hh * gy / s.hh;
            else tt_w = C43 * t1 - C13 * t2 - C23 * s.top_dz * (s.theta - (s.theta - tpr) * gx / s.hh * gy / s.hh);
        } else if (s.itcon == 0 || s.itcon == 2 || s.itcon == 4) {
            tt_w = 1.0;
            if (s.itcon == 4 && gi + 2 <= (npx + 2) / 2) tt_w = 1.0 - s.tp;
        } else if (s.itcon == 1) {
            tt_w = C43 * t1 - C13 * t2 - s.top_flux;
        }
        put(F_RU, 0, ru_w);
        put(F_RV, 0, rv_w);
        put(F_RW, 0, 0.0);
        put(F_TT, 0, tt_w);
        if (MAG && s.ibcon == 0) put(F_BZ, 0, 0.0);
    }
    // bottom
    {
        const int kb = npz - 1;
        const double ro0 = at(F_RO, kb), ro1 = at(F_RO, kb - 1), ro2 = at(F_RO, kb - 2);
        const double ru_w = ro0 * (C43 * at(F_RU, kb - 1) / ro1 - C13 * at(F_RU, kb - 2) / ro2);
        const double rv_w = ro0 * (C43 * at(F_RV, kb - 1) / ro1 - C13 * at(F_RV, kb - 2) / ro2);
        const double tt_w = (s.izcon == 0) ? s.tb : C43 * at(F_TT, kb - 1) - C13 * at(F_TT, kb - 2) + s.bot_flux;
        put(F_RU, kb, ru_w);
        put(F_RV, kb, rv_w);
        put(F_RW, kb, 0.0);
        put(F_TT, kb, tt_w);
        if (MAG && s.ibcon == 0) put(F_BZ, kb, 0.0);
    }
}

template <bool MAG, bool ROT>
static cudaError_t launch_stage_t(int stage, const StageArgs& a, cudaStream_t st)
{
    const size_t smem = Lay<MAG>::BYTES;
    const int nty = (a.s.npy + TY - 1) / TY;
    dim3 grid(a.ntx * nty, a.nchunks);
    switch (stage) {
#define L_(S)                                                                                              \
    case S: {                                                                                              \
        static std::atomic<unsigned long long> attr_set{0};                                                \
        cudaError_t ae = smem_attr_once(attr_set, reinterpret_cast<const void*>(k_stage<MAG, ROT, S>), smem); \
        if (ae != cudaSuccess) return ae;                                                                  \
        k_stage<MAG, ROT, S><<<grid, NT, smem, st>>>(a);                                                  \
        break;                                                                                             \
    }
        L_(0) L_(1) L_(2) L_(3)
#undef L_
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_stage(int stage, const StageArgs& a, cudaStream_t st)
{
    if (a.s.lmag) return a.s.lrot ? launch_stage_t<true, true>(stage, a, st) : launch_stage_t<true, false>(stage, a, st);
    return a.s.lrot ? launch_stage_t<false, true>(stage, a, st) : launch_stage_t<false, false>(stage, a, st);
}

size_t stage_smem_bytes(int lmag) { return lmag ? Lay<true>::BYTES : Lay<false>::BYTES; }

cudaError_t launch_cfl(const StageArgs& a, cudaStream_t st)
{
    const size_t ncell = (size_t)a.s.npx * a.s.npy * a.s.npz;
    size_t nb = (ncell + NT - 1) / NT;
    if (nb > 148 * 8) nb = 148 * 8;
    if (a.s.lmag) k_cfl<true><<<(unsigned)nb, NT, 0, st>>>(a);
    else k_cfl<false><<<(unsigned)nb, NT, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_bcon(const StageArgs& a, cudaStream_t st)
{
    const int n = a.s.npx * a.s.npy;
    const int nb = (n + NT - 1) / NT;
    if (a.s.lmag) k_bcon<true><<<nb, NT, 0, st>>>(a);
    else k_bcon<false><<<nb, NT, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace MHD3D_NS
}  // namespace mhd3d
