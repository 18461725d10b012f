// stage_f32.cu -- the FP32 form of the fused RK3 stage kernel (RHS + update +
// BCON + ghost-plane toggle + CFL reduction), for the same equations as
// stage_impl.cuh (FLUXES 3dmhdsub.f:1249-2634, STEP 874-1173, BCON 2751-2955).
//
// Storage: U and Z in FP32 as perturbations from the background profiles of
// StageArgs32 (TT, RO, BX, BY, BZ; the momenta are stored whole).  The
// arithmetic is FP32 with FMA contraction.  Differences in x and y of a
// perturbation equal those of the field; differences in z add the
// background's difference, formed on the host in FP64 (PlaneBg), so no FP32
// operation cancels two background-sized numbers.  The pressure enters as
// P' = RHOb*T' + RO'*(Tb + T') and the gravity/pressure balance of the
// background as one FP64-formed number per plane.  The step's CFL limits and
// Mach number are formed per cell in FP32 and reduced through FP64 keys; the
// standalone CFL pass (first step, state changes) forms them in FP64.
//
// Work decomposition and plane ring as in the FP64 kernel: a CTA owns a
// 32 x TY32 tile of columns and a chunk of z planes; planes arrive by TMA
// (box 36 x (TY32+2) x 1 x nf floats) into a four-slot ring, Z by its own box;
// every wait is bounded.  No TMA load uses cluster multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cfloat>

#include "../../include/mhd3d.h"
#include "mhd3d_dev.cuh"
#include "ring.cuh"
#include "smem_attr.cuh"

#define MHD3D_NS f32
#define MHD3D_FAST_BODY 1
#include "cfl_cell.cuh"

namespace mhd3d {
namespace f32 {

#include "cfl_acc.cuh"

constexpr int NRAW = 4;
constexpr int NRI = 3;

constexpr size_t al128(size_t b) { return (b + 127) / 128 * 128; }

// shared-memory layout of a CTA with TYV tile rows (TX x TYV threads)
template <bool MAG, int TYV = TY32>
struct Lay32 {
    static constexpr int NF = MAG ? 8 : 5;
    static constexpr int NTV = TX * TYV;                  // threads
    static constexpr int BSV = BW32 * (TYV + 2);          // floats of one field in one plane box
    static constexpr size_t RAW_SLOT_B = al128((size_t)NF * BSV * 4);
    static constexpr size_t RI_OFF_B = NRAW * RAW_SLOT_B;
    static constexpr size_t Z_OFF_B = al128(RI_OFF_B + (size_t)NRI * BSV * 4);
    static constexpr size_t BAR_OFF_B = al128(Z_OFF_B + (size_t)NF * TYV * TX * 4);
    static constexpr size_t RED_OFF_B = BAR_OFF_B + 8 * 8;
    static constexpr size_t FLAG_OFF_B = RED_OFF_B + (size_t)(NTV / 32) * 3 * 8;
    static constexpr size_t BYTES = FLAG_OFF_B + 16 + 128;   // + alignment slack
};

enum Q32 { P_RU = 0, P_RV, P_RW, P_RO, P_TT, P_RI, P_UU, P_VV, P_WW, P_PP, P_BX, P_BY, P_BZ };

// quantity QQ at offset off of a plane slot whose background is (rob, ttb):
// stored fields, 1/RO, velocities, and the pressure perturbation
template <int QQ, int BS = BSLOT32>
__device__ __forceinline__ float qf(const float* __restrict__ raw, const float* __restrict__ ri, int off, float rob,
                                    float ttb)
{
    if constexpr (QQ == P_RU) return raw[F_RU * BS + off];
    else if constexpr (QQ == P_RV) return raw[F_RV * BS + off];
    else if constexpr (QQ == P_RW) return raw[F_RW * BS + off];
    else if constexpr (QQ == P_RO) return raw[F_RO * BS + off];
    else if constexpr (QQ == P_TT) return raw[F_TT * BS + off];
    else if constexpr (QQ == P_BX) return raw[F_BX * BS + off];
    else if constexpr (QQ == P_BY) return raw[F_BY * BS + off];
    else if constexpr (QQ == P_BZ) return raw[F_BZ * BS + off];
    else if constexpr (QQ == P_RI) return ri[off];
    else if constexpr (QQ == P_UU) return raw[F_RU * BS + off] * ri[off];
    else if constexpr (QQ == P_VV) return raw[F_RV * BS + off] * ri[off];
    else if constexpr (QQ == P_WW) return raw[F_RW * BS + off] * ri[off];
    else {
        const float t = raw[F_TT * BS + off];
        return rob * t + raw[F_RO * BS + off] * (ttb + t);
    }
}

// Stage-3 CFL limits of the FP32 form: formed per cell in FP32 (the
// contracted form of the FP64 FMA build: W1 = DD/(|u|+c_f), W2 and W3 from
// Y=DD*DD*RO), reduced per warp in FP32 and across warps and CTAs as FP64
// keys.  One FP64 reduction per step; DT carries FP32's relative precision.
struct CflAcc32 {
    float smax = 0.f;                          // max over cells of (|u|+c_f)/DD
    float wmin = __builtin_huge_valf();        // min of W2, W3
    float m2 = -__builtin_huge_valf();         // max of MACH**2
    unsigned bad = 0;
};

template <bool MAG>
__device__ __forceinline__ void cfl32_cell(CflAcc32& c, float ogamma, float gamma, float obeta, float cw3, float rdd,
                                           float dd, float fw2, float ru, float rv, float rw, float ro, float tt,
                                           float bx, float by, float bz)
{
    const float r = __frcp_rn(ro);
    const float uu = (ru * ru + rv * rv + rw * rw) * (r * r);
    const float mach2 = ogamma * uu * __frcp_rn(tt);
    float a2 = gamma * tt;
    if (MAG) a2 += (bx * bx + by * by + bz * bz) * obeta * r;
    const float sp = sqrtf(uu) + sqrtf(a2);
    const float sr = sp * rdd;
    const float y = dd * dd * ro;
    const float w = fminf(cw3 * y, fw2 * y);
    c.smax = fmaxf(c.smax, sr);
    c.wmin = fminf(c.wmin, w);
    c.m2 = fmaxf(c.m2, mach2);
    c.bad |= (unsigned)(!(sr > 0.f && sr <= FLT_MAX) || !(fabsf(w) <= FLT_MAX) || !(fabsf(mach2) <= FLT_MAX));
}

__device__ __forceinline__ void cfl32_commit(Accum* acc, unsigned long long* red, const CflAcc32& c)
{
    float smax = c.smax, wmin = c.wmin, m2 = c.m2;
    unsigned bad = c.bad;
    for (int o = 16; o > 0; o >>= 1) {
        smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        wmin = fminf(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        m2 = fmaxf(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    unsigned long long* r = red + (threadIdx.x >> 5) * 3;
    if ((threadIdx.x & 31) == 0) {
        double w = (double)wmin;
        if (smax > 0.f) w = fmin(w, 1.0 / (double)smax);
        r[0] = key_of(w);
        r[1] = key_of((double)m2);
        r[2] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long kmin = ~0ull, kmu = 0ull, b = 0ull;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            kmin = min(kmin, red[i * 3 + 0]);
            kmu = max(kmu, red[i * 3 + 1]);
            b |= red[i * 3 + 2];
        }
        atomicMin(&acc->wmin[0], kmin);
        atomicMax(&acc->umax, kmu);
        if (b) atomicOr(&acc->bad, 1u);
    }
}


// One work item: the z chunk `chunk` of tile `tile` of the grid described by
// `a`, on the CTA's shared memory `sb` (128-byte aligned).  On return every
// TMA copy the item issued has landed and its mbarriers are invalidated, so
// a persistent CTA can take the next item.
template <bool MAG, bool ROT, int STAGE, int TYV = TY32>
__device__ __forceinline__ void stage32_item(const StageArgs32& a, const int tile, const int chunk,
                                             unsigned char* const sb)
{
    using L = Lay32<MAG, TYV>;
    constexpr int TYL = TYV, NTL = L::NTV, BSL = L::BSV;
    constexpr int NF = L::NF;
    float* const sraw = reinterpret_cast<float*>(sb);
    float* const sri = reinterpret_cast<float*>(sb + L::RI_OFF_B);
    float* const sz = reinterpret_cast<float*>(sb + L::Z_OFF_B);
    unsigned long long* const bars = reinterpret_cast<unsigned long long*>(sb + L::BAR_OFF_B);
    unsigned long long* const red = reinterpret_cast<unsigned long long*>(sb + L::RED_OFF_B);
    int* const sflag = reinterpret_cast<int*>(sb + L::FLAG_OFF_B);

    const Control* ctl = a.ctl;
    const Scalars& s = a.s;
    const Metrics& m = a.m;
    const int npx = s.npx, npy = s.npy, npz = s.npz;
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x0 = (tile % a.ntx) * TX, y0 = (tile / a.ntx) * TYL;
    const int k0 = chunk * a.zlen;
    const int k1 = (chunk == a.nchunks - 1) ? npz : k0 + a.zlen;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool active = gi < npx && gj < npy;
    const int lx = tx + 1, ly = ty + 1;

    const double DT = ctl->dt;
    const float cu = (float)(STAGE == 1 ? s.gam1 * DT : STAGE == 2 ? s.gam2 * DT : s.gam3 * DT);
    const float cz = (float)(STAGE == 1 ? s.zeta1 * DT : s.zeta2 * DT);
    const Scalars32& f = a.s32;
    const float C13 = f.c13, C43 = f.c43;

    const ColC cxc = a.cx[active ? gi + 1 : 0], cyc = a.cy[active ? gj + 1 : 0];
    const float ax = cxc.a, bxq = cxc.b, cxq = cxc.c;
    const float ay = cyc.a, byq = cyc.b, cyq = cyc.c;
    // stage-3 CFL: per-column 1/DD and DD parts
    const float rddxy = fmaxf(cxc.rdd, cyc.rdd);
    const float ddxy = fminf(cxc.dd, cyc.dd);

    const unsigned raw_bytes = (unsigned)(NF * BSL * 4);
    const unsigned z_bytes = (unsigned)(NF * TYL * TX * 4);
    const size_t ucol = (size_t)(gj + 1) * a.upitch + (gi + 1);
    const size_t zcol = (size_t)gj * a.zpitch + gi;
    const HaloCols hc = halo_cols(npx, npy, a.upitch, gi, gj);
    const bool use_fcl = STAGE != 0 && a.fcl != nullptr && *a.fcl_flag == 0;

    // the stop flag is read once, by one thread, so the CTA takes one path
    if (tid == 0) {
        const bool stopped = STAGE != 0 && ctl->stop;
        *sflag = stopped ? -1 : 0;
        if (!stopped) {
            for (int i = 0; i < NRAW + 1; ++i) mbar_init(&bars[i], 1);
            fence_mbar_init();
        }
    }
    if (STAGE == 3 && (tid & 31) == 0) {
        unsigned long long* r = red + (tid >> 5) * 3;
        r[0] = ~0ull;
        r[1] = 0ull;
        r[2] = 0ull;
    }
    __syncthreads();
    if (*sflag < 0) return;

    int hi_issued = k0 - 2;
    auto issue_plane = [&](int kp) {
        const int sl = (kp + 1) & 3;
        fence_proxy_async();
        mbar_expect_tx(&bars[sl], raw_bytes);
        tma_load4(reinterpret_cast<unsigned char*>(sraw) + (size_t)sl * L::RAW_SLOT_B, &a.map_u, &bars[sl], x0, y0,
                  kp + 1, 0);
        hi_issued = kp;
    };
    auto parity_of = [&](int kp) -> unsigned { return (unsigned)(((kp - (k0 - 1)) >> 2) & 1); };
    auto slot = [&](int kp) -> const float* {
        return reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(sraw) +
                                              (size_t)((kp + 1) & 3) * L::RAW_SLOT_B);
    };
    auto derive_ri = [&](int kp) {
        const float* r = slot(kp) + F_RO * BSL;
        float* d = sri + (size_t)((kp + 1) % 3) * BSL;
        const float rb = a.rob[kp + 1];
        for (int p = tid; p < BSL; p += NTL) d[p] = __frcp_rn(rb + r[p]);
    };

    if (tid == 0)
        for (int kp = k0 - 1; kp <= k0 + 2 && kp <= k1; ++kp) issue_plane(kp);
    bool ok = mbar_wait(&bars[(k0 + 0) & 3], parity_of(k0 - 1)) && mbar_wait(&bars[(k0 + 1) & 3], parity_of(k0));
    if (ok) {
        derive_ri(k0 - 1);
        derive_ri(k0);
    } else {
        atomicOr(sflag, 1);
    }
    bool zpending = false;
    int zfill = 0;
    CflAcc32 cfa;
    auto cfl_at = [&](const PlaneBg& q, float ru, float rv, float rw, float ro, float tt, float bx, float by, float bz) {
        cfl32_cell<MAG>(cfa, f.ogamma, f.gamma, f.obeta, f.cw3, fmaxf(rddxy, q.rddz), fminf(ddxy, q.ddz), q.fw2z, ru,
                        rv, rw, ro, tt, bx, by, bz);
    };

    for (int k = k0; k < k1; ++k) {
        if (STAGE >= 2 && tid == 0 && !*sflag) {
            fence_proxy_async();
            mbar_expect_tx(&bars[NRAW], z_bytes);
            tma_load4(sz, &a.map_z, &bars[NRAW], x0, y0, k, 0);
            zpending = true;
        }
        if (!mbar_wait(&bars[(k + 2) & 3], parity_of(k + 1))) atomicOr(sflag, 1);
        else derive_ri(k + 1);
        __syncthreads();
        if (*sflag) break;
        bool zok = true;
        if (active) {
            const float* Rm = slot(k - 1);
            const float* Rc = slot(k);
            const float* Rp = slot(k + 1);
            const float* Im = sri + (size_t)((k + 0) % 3) * BSL;
            const float* Ic = sri + (size_t)((k + 1) % 3) * BSL;
            const float* Ip = sri + (size_t)((k + 2) % 3) * BSL;
            const PlaneBg& pb = a.pb[k];
            const float robm = pb.robm, robc = pb.robc, robp = pb.robp;
            const float ttbm = pb.ttbm, ttbc = pb.ttbc, ttbp = pb.ttbp;
#define C_(q, dx, dy) qf<q, BSL>(Rc, Ic, (ly + (dy)) * BW32 + (lx + (dx)), robc, ttbc)
#define M_(q, dx, dy) qf<q, BSL>(Rm, Im, (ly + (dy)) * BW32 + (lx + (dx)), robm, ttbm)
#define P_(q, dx, dy) qf<q, BSL>(Rp, Ip, (ly + (dy)) * BW32 + (lx + (dx)), robp, ttbp)
            const bool top = (k == 0), bot = (k == npz - 1);
            const float az = pb.az, bzq = pb.bzq, czq = pb.czq, rka = pb.rka, dka = pb.dka;
            // own column two and three planes inside the wall (one-sided stencils)
            float rw2 = 0.f, ww2 = 0.f, bx2 = 0.f, bx3 = 0.f, by2 = 0.f, by3 = 0.f;
            if (top || bot) {
                const int kk2 = top ? 2 : npz - 3, kk3 = top ? 3 : npz - 4;
                const size_t c2 = (size_t)(kk2 + 1) * a.uz + ucol, c3 = (size_t)(kk3 + 1) * a.uz + ucol;
                rw2 = a.u_in[c2 + F_RW * a.uf];
                ww2 = rw2 / (a.rob[kk2 + 1] + a.u_in[c2 + F_RO * a.uf]);
                if (MAG) {
                    bx2 = a.u_in[c2 + F_BX * a.uf];
                    bx3 = a.u_in[c3 + F_BX * a.uf];
                    by2 = a.u_in[c2 + F_BY * a.uf];
                    by3 = a.u_in[c3 + F_BY * a.uf];
                }
            }

            const float RIc = C_(P_RI, 0, 0), ROp = C_(P_RO, 0, 0), TTp = C_(P_TT, 0, 0);
            const float RUc = C_(P_RU, 0, 0), RVc = C_(P_RV, 0, 0), RWc = C_(P_RW, 0, 0);
            const float BXp = MAG ? C_(P_BX, 0, 0) : 0.f, BYp = MAG ? C_(P_BY, 0, 0) : 0.f;
            const float BZp = MAG ? C_(P_BZ, 0, 0) : 0.f;
            const float uc = RUc * RIc, vc = RVc * RIc, wc = RWc * RIc;
            const float u_xp = C_(P_UU, 1, 0), u_xm = C_(P_UU, -1, 0), u_yp = C_(P_UU, 0, 1), u_ym = C_(P_UU, 0, -1);
            const float v_xp = C_(P_VV, 1, 0), v_xm = C_(P_VV, -1, 0), v_yp = C_(P_VV, 0, 1), v_ym = C_(P_VV, 0, -1);
            const float w_xp = C_(P_WW, 1, 0), w_xm = C_(P_WW, -1, 0), w_yp = C_(P_WW, 0, 1), w_ym = C_(P_WW, 0, -1);
            const float u_zp = P_(P_UU, 0, 0), u_zm = M_(P_UU, 0, 0);
            const float v_zp = P_(P_VV, 0, 0), v_zm = M_(P_VV, 0, 0);
            const float w_zp = P_(P_WW, 0, 0), w_zm = M_(P_WW, 0, 0);

            // continuity, one-sided d(RW)/dz on the walls
            float dzrw;
            if (top) dzrw = (4.f * P_(P_RW, 0, 0) - rw2) * az;
            else if (bot) dzrw = (rw2 - 4.f * M_(P_RW, 0, 0)) * az;
            else dzrw = (P_(P_RW, 0, 0) - M_(P_RW, 0, 0)) * az;
            float fr = -((C_(P_RU, 1, 0) - C_(P_RU, -1, 0)) * ax + (C_(P_RV, 0, 1) - C_(P_RV, 0, -1)) * ay) - dzrw;
            // buoyancy, pressure gradient (perturbation), advection
            float fu = -((C_(P_PP, 1, 0) - C_(P_PP, -1, 0)) * ax
                         + (C_(P_RU, 1, 0) * u_xp - C_(P_RU, -1, 0) * u_xm) * ax
                         + (C_(P_RU, 0, 1) * v_yp - C_(P_RU, 0, -1) * v_ym) * ay
                         + (P_(P_RU, 0, 0) * w_zp - M_(P_RU, 0, 0) * w_zm) * az);
            float fv = -((C_(P_PP, 0, 1) - C_(P_PP, 0, -1)) * ay
                         + (C_(P_RV, 1, 0) * u_xp - C_(P_RV, -1, 0) * u_xm) * ax
                         + (C_(P_RV, 0, 1) * v_yp - C_(P_RV, 0, -1) * v_ym) * ay
                         + (P_(P_RV, 0, 0) * w_zp - M_(P_RV, 0, 0) * w_zm) * az);
            float fw = f.grav * ROp + pb.fw
                     - ((P_(P_PP, 0, 0) - M_(P_PP, 0, 0)) * az
                        + (C_(P_RW, 1, 0) * u_xp - C_(P_RW, -1, 0) * u_xm) * ax
                        + (C_(P_RW, 0, 1) * v_yp - C_(P_RW, 0, -1) * v_ym) * ay
                        + (P_(P_RW, 0, 0) * w_zp - M_(P_RW, 0, 0) * w_zm) * az);
            // temperature advection and conduction
            float ft;
            {
                const float txp = C_(P_TT, 1, 0), txm = C_(P_TT, -1, 0);
                const float typ = C_(P_TT, 0, 1), tym = C_(P_TT, 0, -1);
                const float tzp = P_(P_TT, 0, 0), tzm = M_(P_TT, 0, 0);
                const float dtx = txp - txm, dty = typ - tym, dtzp = tzp - tzm;
                const float dtz = dtzp + pb.tz;
                const float lap = dtx * bxq + (txp + txm - 2.f * TTp) * cxq + dty * byq + (typ + tym - 2.f * TTp) * cyq
                                + dtzp * bzq + (tzp + tzm - 2.f * TTp) * czq + pb.tlz;
                ft = -(uc * dtx * ax + vc * dty * ay + wc * dtz * az) + RIc * f.tmpc * (rka * lap + dka * dtz * az);
            }
            // viscous stress
            {
                const float lxu = (u_xp - u_xm) * bxq + (u_xp + u_xm - 2.f * uc) * cxq;
                const float lyu = (u_yp - u_ym) * byq + (u_yp + u_ym - 2.f * uc) * cyq;
                const float lzu = (u_zp - u_zm) * bzq + (u_zp + u_zm - 2.f * uc) * czq;
                const float lxv = (v_xp - v_xm) * bxq + (v_xp + v_xm - 2.f * vc) * cxq;
                const float lyv = (v_yp - v_ym) * byq + (v_yp + v_ym - 2.f * vc) * cyq;
                const float lzv = (v_zp - v_zm) * bzq + (v_zp + v_zm - 2.f * vc) * czq;
                const float lxw = (w_xp - w_xm) * bxq + (w_xp + w_xm - 2.f * wc) * cxq;
                const float lyw = (w_yp - w_ym) * byq + (w_yp + w_ym - 2.f * wc) * cyq;
                const float lzw = (w_zp - w_zm) * bzq + (w_zp + w_zm - 2.f * wc) * czq;
                fu += f.ore * (f.c43 * lxu + lyu + lzu);
                fv += f.ore * (lxv + f.c43 * lyv + lzv);
                fw += f.ore * (lxw + lyw + f.c43 * lzw);
            }
            // velocity gradients, the 19-point cross terms, heating
            const float ux = (u_xp - u_xm) * ax, vx = (v_xp - v_xm) * ax, wx = (w_xp - w_xm) * ax;
            const float uy = (u_yp - u_ym) * ay, vy = (v_yp - v_ym) * ay, wy = (w_yp - w_ym) * ay;
            const float uz = (u_zp - u_zm) * az, vz = (v_zp - v_zm) * az, wz = (w_zp - w_zm) * az;
            {
                const float axy = ax * ay, axz = ax * az, ayz = ay * az;
                const float dyvx = ((C_(P_VV, 1, 1) - C_(P_VV, -1, 1)) - (C_(P_VV, 1, -1) - C_(P_VV, -1, -1))) * axy;
                const float dyux = ((C_(P_UU, 1, 1) - C_(P_UU, -1, 1)) - (C_(P_UU, 1, -1) - C_(P_UU, -1, -1))) * axy;
                const float dxwz = ((P_(P_WW, 1, 0) - M_(P_WW, 1, 0)) - (P_(P_WW, -1, 0) - M_(P_WW, -1, 0))) * axz;
                const float dywz = ((P_(P_WW, 0, 1) - M_(P_WW, 0, 1)) - (P_(P_WW, 0, -1) - M_(P_WW, 0, -1))) * ayz;
                const float dxuz = ((P_(P_UU, 1, 0) - M_(P_UU, 1, 0)) - (P_(P_UU, -1, 0) - M_(P_UU, -1, 0))) * axz;
                const float dyvz = ((P_(P_VV, 0, 1) - M_(P_VV, 0, 1)) - (P_(P_VV, 0, -1) - M_(P_VV, 0, -1))) * ayz;
                fu += f.tmp13 * (dyvx + dxwz);
                fv += f.tmp13 * (dyux + dywz);
                fw += f.tmp13 * (dxuz + dyvz);
            }
            float heat = f.tmpa * (f.c43 * ux * ux + vx * vx + wx * wx + uy * uy + 2.f * uy * vx + uz * uz + vz * vz
                                 + wy * wy + 2.f * vz * wy + 2.f * uz * wx)
                       + f.tmpb * (vy * vy + wz * wz - ux * wz - ux * vy - vy * wz);
            ft -= f.ocv * (ttbc + TTp) * (ux + vy + wz);
            if (ROT) {
                fu += f.omz * RVc;
                fv += f.omx * RWc - f.omz * RUc;
                fw -= f.omx * RVc;
            }
            // induction, Lorentz force, Ohmic heating
            float w1 = 0.f, w2 = 0.f, w3 = 0.f;
            if (MAG) {
                const float BXc = pb.bx + BXp, BYc = pb.by + BYp, BZc = pb.bz + BZp;
                const float bxxp = C_(P_BX, 1, 0), bxxm = C_(P_BX, -1, 0), bxyp = C_(P_BX, 0, 1), bxym = C_(P_BX, 0, -1);
                const float byxp = C_(P_BY, 1, 0), byxm = C_(P_BY, -1, 0), byyp = C_(P_BY, 0, 1), byym = C_(P_BY, 0, -1);
                const float bzxp = C_(P_BZ, 1, 0), bzxm = C_(P_BZ, -1, 0), bzyp = C_(P_BZ, 0, 1), bzym = C_(P_BZ, 0, -1);
                const float bxzp = P_(P_BX, 0, 0), bxzm = M_(P_BX, 0, 0);
                const float byzp = P_(P_BY, 0, 0), byzm = M_(P_BY, 0, 0);
                const float bzzp = P_(P_BZ, 0, 0), bzzm = M_(P_BZ, 0, 0);
                const float bxx = (bxxp - bxxm) * ax, byx = (byxp - byxm) * ax, bzx = (bzxp - bzxm) * ax;
                const float bxy = (bxyp - bxym) * ay, byy = (byyp - byym) * ay, bzy = (bzyp - bzym) * ay;
                const float bxz = (bxzp - bxzm + pb.bxz) * az, byz = (byzp - byzm + pb.byz) * az;
                const float bzz = (bzzp - bzzm + pb.bzz) * az;
                float wzm = wz, lzbx, lzby;
                if (top) {
                    wzm = (4.f * w_zp - ww2) * az;
                    lzbx = (-3.f * BXp + 4.f * bxzp - bx2) * bzq + (2.f * BXp - 5.f * bxzp + 4.f * bx2 - bx3) * czq;
                    lzby = (-3.f * BYp + 4.f * byzp - by2) * bzq + (2.f * BYp - 5.f * byzp + 4.f * by2 - by3) * czq;
                } else if (bot) {
                    wzm = (ww2 - 4.f * w_zm) * az;
                    lzbx = (3.f * BXp - 4.f * bxzm + bx2) * bzq + (2.f * BXp - 5.f * bxzm + 4.f * bx2 - bx3) * czq;
                    lzby = (3.f * BYp - 4.f * byzm + by2) * bzq + (2.f * BYp - 5.f * byzm + 4.f * by2 - by3) * czq;
                } else {
                    lzbx = (bxzp - bxzm) * bzq + (bxzp + bxzm - 2.f * BXp) * czq;
                    lzby = (byzp - byzm) * bzq + (byzp + byzm - 2.f * BYp) * czq;
                }
                const float lbx = (bxxp - bxxm) * bxq + (bxxp + bxxm - 2.f * BXp) * cxq
                                + (bxyp - bxym) * byq + (bxyp + bxym - 2.f * BXp) * cyq + lzbx + pb.bxlz;
                const float lby = (byxp - byxm) * bxq + (byxp + byxm - 2.f * BYp) * cxq
                                + (byyp - byym) * byq + (byyp + byym - 2.f * BYp) * cyq + lzby + pb.bylz;
                const float lbz = (bzxp - bzxm) * bxq + (bzxp + bzxm - 2.f * BZp) * cxq
                                + (bzyp - bzym) * byq + (bzyp + bzym - 2.f * BZp) * cyq
                                + (bzzp - bzzm) * bzq + (bzzp + bzzm - 2.f * BZp) * czq + pb.bzlz;
                w1 = BYc * uy - BXc * vy + BZc * uz - BXc * wzm - (uc * bxx + vc * bxy + wc * bxz) + f.orm * lbx;
                w2 = BXc * vx - BYc * ux + BZc * vz - BYc * wzm - (uc * byx + vc * byy + wc * byz) + f.orm * lby;
                w3 = BXc * wx - BZc * ux + BYc * wy - BZc * vy - (uc * bzx + vc * bzy + wc * bzz) + f.orm * lbz;
                const float jz = bxy - byx, jy = bxz - bzx, jx = byz - bzy;
                fu += f.obeta * (BYc * jz + BZc * jy);
                fv += f.obeta * (BZc * jx - BXc * jz);
                fw -= f.obeta * (BXc * jy + BYc * jx);
                heat += f.tmpm * (jx * jx + jy * jy + jz * jz);
            }
            ft += RIc * heat;
            // ghost RO planes: FLUXES leaves 1/RO behind (3dmhdsub.f:1386-1391)
            if (STAGE != 0) {
                if (top) store_cell<1, float>(a.u_out, a.uf, ucol, hc, {F_RO}, {M_(P_RI, 0, 0) - a.rob[0]});
                if (bot)
                    store_cell<1, float>(a.u_out + (size_t)(npz + 1) * a.uz, a.uf, ucol, hc, {F_RO},
                                         {P_(P_RI, 0, 0) - a.rob[npz + 1]});
            }
#undef C_
#undef M_
#undef P_
            const bool wall = top || bot;
            const size_t zc = (size_t)k * a.zz + zcol;
            if (STAGE == 0) {
                a.f_out[zc + 0 * a.zf] = wall ? 0.f : fu;
                a.f_out[zc + 1 * a.zf] = wall ? 0.f : fv;
                a.f_out[zc + 2 * a.zf] = wall ? 0.f : fw;
                a.f_out[zc + 3 * a.zf] = fr;
                a.f_out[zc + 4 * a.zf] = wall ? 0.f : ft;
                if (MAG) {
                    a.f_out[zc + 5 * a.zf] = w1;
                    a.f_out[zc + 6 * a.zf] = w2;
                    a.f_out[zc + 7 * a.zf] = wall ? 0.f : w3;
                }
            } else {
                // learned closure: its tendencies, fixed over the step, join the right-hand side
                if (use_fcl) {
                    const float* fc = a.fcl + zc;
                    fu += fc[0];
                    fv += fc[a.zf];
                    fw += fc[2 * a.zf];
                    ft += fc[3 * a.zf];
                    if (MAG) {
                        w1 += fc[4 * a.zf];
                        w2 += fc[5 * a.zf];
                        w3 += fc[6 * a.zf];
                    }
                }
                // RK3 update of the perturbations (the backgrounds do not change)
                float zu, zv, zw, zr, zt, zbx = 0.f, zby = 0.f, zbz = 0.f;
                if (STAGE == 1) {
                    zu = RUc; zv = RVc; zw = RWc; zr = ROp; zt = TTp;
                    if (MAG) { zbx = BXp; zby = BYp; zbz = BZp; }
                } else {
                    zok = mbar_wait(&bars[NRAW], (unsigned)(zfill & 1));
                    const float* zt_ = sz + ty * TX + tx;
                    zu = zt_[F_RU * TYL * TX];
                    zv = zt_[F_RV * TYL * TX];
                    zw = zt_[F_RW * TYL * TX];
                    zt = zt_[F_TT * TYL * TX];
                    zr = zt_[F_RO * TYL * TX];
                    if (MAG) {
                        zbx = zt_[F_BX * TYL * TX];
                        zby = zt_[F_BY * TYL * TX];
                        zbz = zt_[F_BZ * TYL * TX];
                    }
                }
                const float nu = zu + cu * fu, nv = zv + cu * fv, nw = zw + cu * fw;
                const float nr = zr + cu * fr, nt = zt + cu * ft;
                const float nbx = zbx + cu * w1, nby = zby + cu * w2, nbz = zbz + cu * w3;
                const int kz = k + 1;
                if (zok) {
                    float* const pl = a.u_out + (size_t)kz * a.uz;
                    if (MAG)
                        store_cell<8, float>(pl, a.uf, ucol, hc, {F_RO, F_BX, F_BY, F_RU, F_RV, F_RW, F_TT, F_BZ},
                                             {nr, nbx, nby, nu, nv, nw, nt, nbz});
                    else
                        store_cell<5, float>(pl, a.uf, ucol, hc, {F_RO, F_RU, F_RV, F_RW, F_TT}, {nr, nu, nv, nw, nt});
                    if (STAGE < 3) {
                        float* zo = a.z + zc;
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
                if (!top && !bot && STAGE == 3)
                    cfl_at(pb, nu, nv, nw, robc + nr, ttbc + nt, MAG ? pb.bx + nbx : 0.f, MAG ? pb.by + nby : 0.f,
                           MAG ? pb.bz + nbz : 0.f);
                if (k == 2 && k0 == 0) {
                    // top wall (plane 0) from planes 1 (read back) and 2 (this plane)
                    const float* ub = a.u_out + ucol;
                    const size_t c0 = 1 * a.uz, c1 = 2 * a.uz;
                    const float h1_ru = ub[F_RU * a.uf + c1], h1_rv = ub[F_RV * a.uf + c1];
                    const float h1_ro = a.rob[2] + ub[F_RO * a.uf + c1], h1_tt = ub[F_TT * a.uf + c1];
                    const float w0_rop = ub[F_RO * a.uf + c0], w0_ttp = ub[F_TT * a.uf + c0];
                    const float w0_ro = a.rob[1] + w0_rop, nrf = a.rob[3] + nr;
                    const float w0_bx = MAG ? ub[F_BX * a.uf + c0] : 0.f, w0_by = MAG ? ub[F_BY * a.uf + c0] : 0.f;
                    const float w0_bz = MAG ? ub[F_BZ * a.uf + c0] : 0.f;
                    const float ru_w = w0_ro * (C43 * h1_ru / h1_ro - C13 * nu / nrf);
                    const float rv_w = w0_ro * (C43 * h1_rv / h1_ro - C13 * nv / nrf);
                    float tt_w = w0_ttp;
                    if (s.plume) {
                        const double tpr = (s.tc != 0.0) ? s.tp + (1.0 - s.tp) * exp(-ctl->timt / s.tc) : s.tp;
                        const double gx = m.plume_gx[gi + 1], gy = m.plume_gy[gj + 1];
                        if (s.itcon == 0)
                            tt_w = (float)(1.0 - (1.0 - tpr) * gx / s.hh * gy / s.hh - a.top_tb);
                        else
                            tt_w = C43 * h1_tt - C13 * nt
                                 + (float)(a.top_lin - s.c23 * s.top_dz * (s.theta - (s.theta - tpr) * gx / s.hh * gy / s.hh));
                    } else if (s.itcon == 0 || s.itcon == 2 || s.itcon == 4) {
                        tt_w = (s.itcon == 4 && gi + 2 <= (npx + 2) / 2) ? a.t_top_fix4 : a.t_top_fix;
                    } else if (s.itcon == 1) {
                        tt_w = C43 * h1_tt - C13 * nt + a.t_top_flux;
                    }
                    const float bz_w = (MAG && s.ibcon == 0) ? -a.pb[0].bz : w0_bz;
                    if (zok) {
                        float* const pl = a.u_out + a.uz;
                        if (MAG)
                            store_cell<5, float>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT, F_BZ},
                                                 {ru_w, rv_w, 0.f, tt_w, bz_w});
                        else
                            store_cell<4, float>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT}, {ru_w, rv_w, 0.f, tt_w});
                    }
                    if (STAGE == 3) {
                        const PlaneBg& p0 = a.pb[0];
                        cfl_at(p0, ru_w, rv_w, 0.f, w0_ro, p0.ttbc + tt_w, MAG ? p0.bx + w0_bx : 0.f,
                               MAG ? p0.by + w0_by : 0.f, MAG ? p0.bz + bz_w : 0.f);
                    }
                }
                if (bot) {
                    // bottom wall (this plane) from planes npz-2 and npz-3, read back
                    const float* ub = a.u_out + ucol;
                    const size_t c1 = (size_t)(npz - 1) * a.uz, c2 = (size_t)(npz - 2) * a.uz;
                    const float h1_ru = ub[F_RU * a.uf + c1], h1_rv = ub[F_RV * a.uf + c1];
                    const float h1_ro = a.rob[npz - 1] + ub[F_RO * a.uf + c1], h1_tt = ub[F_TT * a.uf + c1];
                    const float h2_ru = ub[F_RU * a.uf + c2], h2_rv = ub[F_RV * a.uf + c2];
                    const float h2_ro = a.rob[npz - 2] + ub[F_RO * a.uf + c2], h2_tt = ub[F_TT * a.uf + c2];
                    const float nrf = a.rob[npz] + nr;
                    const float ru_w = nrf * (C43 * h1_ru / h1_ro - C13 * h2_ru / h2_ro);
                    const float rv_w = nrf * (C43 * h1_rv / h1_ro - C13 * h2_rv / h2_ro);
                    const float tt_w = (s.izcon == 0) ? a.t_bot : C43 * h1_tt - C13 * h2_tt + a.t_bot;
                    const float bz_w = (MAG && s.ibcon == 0) ? -pb.bz : nbz;
                    if (zok) {
                        float* const pl = a.u_out + (size_t)kz * a.uz;
                        if (MAG)
                            store_cell<5, float>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT, F_BZ},
                                                 {ru_w, rv_w, 0.f, tt_w, bz_w});
                        else
                            store_cell<4, float>(pl, a.uf, ucol, hc, {F_RU, F_RV, F_RW, F_TT}, {ru_w, rv_w, 0.f, tt_w});
                    }
                    if (STAGE == 3)
                        cfl_at(pb, ru_w, rv_w, 0.f, nrf, ttbc + tt_w, MAG ? pb.bx + nbx : 0.f, MAG ? pb.by + nby : 0.f,
                               MAG ? pb.bz + bz_w : 0.f);
                }
            }
        } else if (STAGE >= 2) {
            zok = mbar_wait(&bars[NRAW], (unsigned)(zfill & 1));
        }
        if (!zok) atomicOr(sflag, 1);
        if (STAGE >= 2) {
            ++zfill;
            if (tid == 0) zpending = false;
        }
        __syncthreads();
        if (*sflag) break;
        if (tid == 0 && k + 3 <= k1) issue_plane(k + 3);
    }
    if (*sflag) {
        if (tid == 0) {
            for (int kp = hi_issued - 3; kp <= hi_issued; ++kp)
                if (kp >= k0 - 1) mbar_wait(&bars[(kp + 1) & 3], parity_of(kp));
            if (zpending) mbar_wait(&bars[NRAW], (unsigned)(zfill & 1));
            atomicExch(&a.ctl->status, MHD3D_ERR_TIMEOUT);
            atomicExch(&a.ctl->stop, 1);
        }
    } else if (STAGE == 3) {
        cfl32_commit(a.acc, red, cfa);
    }
    __syncthreads();
    if (tid == 0)
        for (int i = 0; i < NRAW + 1; ++i) mbar_inval(&bars[i]);
}

template <bool MAG, bool ROT, int STAGE>
__global__ void __launch_bounds__(NT32, MHD3D_MINB32) k_stage32(const __grid_constant__ StageArgs32 a)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    stage32_item<MAG, ROT, STAGE>(a, blockIdx.x, blockIdx.y, sb);
}

// Persistent form for an ensemble of grids: one launch per RK3 stage for all
// members.  Work items (member, tile, z chunk) are numbered member by member
// in `order` (largest members first); item_base[i] is the first item of the
// i-th member in that order.  CTAs take items from a global counter until
// none is left, so members of uneven size share the SMs.
#ifndef MHD3D_MINB32M
#define MHD3D_MINB32M 4   // the persistent form carries its loop state as well: 128 registers, no spills
#endif
// CTAs per SM the register budget of each tile height is sized for (128
// registers a thread in each case)
template <int TYV>
struct MultiMinB {
    static constexpr int v = TYV == 2 ? 8 : TYV == 4 ? MHD3D_MINB32M : 2;
};
template <bool MAG, bool ROT, int STAGE, int TYV>
__global__ void __launch_bounds__(TX * TYV, MultiMinB<TYV>::v) k_stage32_multi(const StageArgs32* __restrict__ args,
                                                                      const int* __restrict__ order,
                                                                      const int* __restrict__ item_base, int nmem,
                                                                      unsigned* counter)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    __shared__ int s_item;
    const int nitems = item_base[nmem];
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= nitems) break;
        int lo = 0, hi = nmem - 1;   // last i with item_base[i] <= it
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (item_base[mid] <= it) lo = mid;
            else hi = mid - 1;
        }
        const StageArgs32& a = args[order[lo]];
        const int ntiles = a.ntx * ((a.s.npy + TYV - 1) / TYV);
        const int local = it - item_base[lo];
        stage32_item<MAG, ROT, STAGE, TYV>(a, local % ntiles, local / ntiles, sb);
        __syncthreads();
    }
}

// CFL reduction over the current FP32 state, formed in FP64 (first step,
// after a state change): every limit as STEP forms it, from the full values.
template <bool MAG>
__global__ void __launch_bounds__(256) k_cfl32(const __grid_constant__ StageArgs32 a)
{
    const Scalars& s = a.s;
    const int npx = s.npx, npy = s.npy, npz = s.npz;
    const size_t NZ = (size_t)npz + 2;
    const size_t ncell = (size_t)npx * npy * npz;
    unsigned long long kmin = ~0ull, kmu = 0ull;
    unsigned bad = 0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < ncell; q += (size_t)gridDim.x * blockDim.x) {
        const int gi = (int)(q % npx);
        const int gj = (int)((q / npx) % npy);
        const int k = (int)(q / ((size_t)npx * npy));
        const float* u = a.u_in + (size_t)(k + 1) * a.uz + (size_t)(gj + 1) * a.upitch + (gi + 1);
        auto full = [&](int which, int f) -> double { return a.bgd[which * NZ + k + 1] + (double)u[(size_t)f * a.uf]; };
        CflPart cp;
        cfl_cell<MAG>(s, (double)u[F_RU * a.uf], (double)u[F_RV * a.uf], (double)u[F_RW * a.uf], full(0, F_RO),
                      full(1, F_TT), MAG ? full(2, F_BX) : 0.0, MAG ? full(3, F_BY) : 0.0, MAG ? full(4, F_BZ) : 0.0,
                      cell_dd(a.m, gi, gj, k), a.m.rkapa[k + 1], cp);
        // W4 depends on the grid alone: its minimum is the accumulator's start value
        kmin = min(kmin, min(min(key_of(cp.w1), key_of(cp.w2)), key_of(cp.w3)));
        kmu = max(kmu, key_of(cp.mach2));
        bad |= cp.bad ? 1u : 0u;
    }
    __shared__ unsigned long long red[(256 / 32) * 3];
    if ((threadIdx.x & 31) == 0) {
        red[(threadIdx.x >> 5) * 3 + 0] = ~0ull;
        red[(threadIdx.x >> 5) * 3 + 1] = 0ull;
        red[(threadIdx.x >> 5) * 3 + 2] = 0ull;
    }
    __syncwarp();
    kmin = warp_min_u64(kmin);
    kmu = warp_max_u64(kmu);
    for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0) {
        red[(threadIdx.x >> 5) * 3 + 0] = kmin;
        red[(threadIdx.x >> 5) * 3 + 1] = kmu;
        red[(threadIdx.x >> 5) * 3 + 2] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long k1 = ~0ull, km = 0ull, b = 0ull;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            k1 = min(k1, red[i * 3 + 0]);
            km = max(km, red[i * 3 + 1]);
            b |= red[i * 3 + 2];
        }
        atomicMin(&a.acc->wmin[0], k1);
        atomicMax(&a.acc->umax, km);
        if (b) atomicOr(&a.acc->bad, 1u);
    }
}

template <bool MAG, bool ROT>
static cudaError_t launch_stage_t(int stage, const StageArgs32& a, cudaStream_t st)
{
    const size_t smem = Lay32<MAG>::BYTES;
    const int nty = (a.s.npy + TY32 - 1) / TY32;
    dim3 grid(a.ntx * nty, a.nchunks);
    switch (stage) {
#define L_(S)                                                                                              \
    case S: {                                                                                              \
        static std::atomic<unsigned long long> attr_set{0};                                                \
        cudaError_t ae = smem_attr_once(attr_set, reinterpret_cast<const void*>(k_stage32<MAG, ROT, S>), smem); \
        if (ae != cudaSuccess) return ae;                                                                  \
        k_stage32<MAG, ROT, S><<<grid, NT32, smem, st>>>(a);                                              \
        break;                                                                                             \
    }
        L_(0) L_(1) L_(2) L_(3)
#undef L_
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_stage(int stage, const StageArgs32& a, cudaStream_t st)
{
    if (a.s.lmag) return a.s.lrot ? launch_stage_t<true, true>(stage, a, st) : launch_stage_t<true, false>(stage, a, st);
    return a.s.lrot ? launch_stage_t<false, true>(stage, a, st) : launch_stage_t<false, false>(stage, a, st);
}

size_t stage_smem_bytes(int lmag) { return lmag ? Lay32<true>::BYTES : Lay32<false>::BYTES; }

template <bool MAG, bool ROT, int TYV>
static cudaError_t launch_multi_t(int stage, const StageArgs32* args, const int* order, const int* item_base,
                                  int nmem, unsigned* counter, int nblocks, cudaStream_t st)
{
    const size_t smem = Lay32<MAG, TYV>::BYTES;
    switch (stage) {
#define L_(S)                                                                                              \
    case S: {                                                                                              \
        static std::atomic<unsigned long long> attr_set{0};                                                \
        cudaError_t ae = smem_attr_once(attr_set, reinterpret_cast<const void*>(k_stage32_multi<MAG, ROT, S, TYV>), \
                                        smem);                                                             \
        if (ae != cudaSuccess) return ae;                                                                  \
        if (nblocks > 0)                                                                                   \
            k_stage32_multi<MAG, ROT, S, TYV><<<nblocks, TX * TYV, smem, st>>>(args, order, item_base, nmem, counter); \
        break;                                                                                             \
    }
        L_(1) L_(2) L_(3)
#undef L_
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int TYV>
static cudaError_t launch_multi_ty(int stage, int lmag, int lrot, const StageArgs32* args, const int* order,
                                   const int* item_base, int nmem, unsigned* counter, int nblocks, cudaStream_t st)
{
    if (lmag)
        return lrot ? launch_multi_t<true, true, TYV>(stage, args, order, item_base, nmem, counter, nblocks, st)
                    : launch_multi_t<true, false, TYV>(stage, args, order, item_base, nmem, counter, nblocks, st);
    return lrot ? launch_multi_t<false, true, TYV>(stage, args, order, item_base, nmem, counter, nblocks, st)
                : launch_multi_t<false, false, TYV>(stage, args, order, item_base, nmem, counter, nblocks, st);
}

bool multi_tile_rows_ok(int ty) { return ty == 2 || ty == 4 || ty == 8; }

size_t multi_smem_bytes(int lmag, int ty)
{
    if (ty == 2) return lmag ? Lay32<true, 2>::BYTES : Lay32<false, 2>::BYTES;
    if (ty == 8) return lmag ? Lay32<true, 8>::BYTES : Lay32<false, 8>::BYTES;
    return lmag ? Lay32<true, 4>::BYTES : Lay32<false, 4>::BYTES;
}

cudaError_t launch_stage_multi(int stage, int lmag, int lrot, int ty, const StageArgs32* args, const int* order,
                               const int* item_base, int nmem, unsigned* counter, int nblocks, cudaStream_t st)
{
    switch (ty) {
    case 2: return launch_multi_ty<2>(stage, lmag, lrot, args, order, item_base, nmem, counter, nblocks, st);
    case 4: return launch_multi_ty<4>(stage, lmag, lrot, args, order, item_base, nmem, counter, nblocks, st);
    case 8: return launch_multi_ty<8>(stage, lmag, lrot, args, order, item_base, nmem, counter, nblocks, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cfl(const StageArgs32& a, cudaStream_t st)
{
    const size_t ncell = (size_t)a.s.npx * a.s.npy * a.s.npz;
    size_t nb = (ncell + 255) / 256;
    if (nb > 148 * 8) nb = 148 * 8;
    if (a.s.lmag) k_cfl32<true><<<(unsigned)nb, 256, 0, st>>>(a);
    else k_cfl32<false><<<(unsigned)nb, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace f32
}  // namespace mhd3d
