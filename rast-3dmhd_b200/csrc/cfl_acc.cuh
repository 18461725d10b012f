// cfl_acc.cuh -- stage-3 accumulation of the next step's CFL limits and
// Mach number, included inside the namespace of a stage-kernel build.
// MHD3D_FAST_BODY selects the contracted form; otherwise every limit is
// formed as STEP forms it.
#pragma once

// ---- stage-3 CFL accumulation (STEP 3dmhdsub.f:741-873) ----
// DT=SF*MIN(W1,W2,W3,W4) needs only the minimum over all cells of the four
// limits together, and UMACH the maximum of MACH**2.  W4=0.5*DD*DD*RM depends
// on the grid alone: the host folds its minimum into the accumulator's start
// value.  Each warp keeps one slot of three words in shared memory: the
// limits' minimum key, MACH**2's maximum key and the non-finite flag.
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Per-column CFL factors, formed once per thread instead of once per cell:
// MIN(DDX(I), DDY(J)) and, for the screening, MAX(1/DDX, 1/DDY) in FP32.
struct CflCol {
    double dd;
    float rdd;
};
__device__ __forceinline__ CflCol cfl_col(const Metrics& m, int gi, int gj, bool active)
{
    CflCol c;
    c.dd = active ? dmin(m.ddx[gi + 1], m.ddy[gj + 1]) : 0.0;
    c.rdd = active ? fmaxf(m.rddx_f[gi + 1], m.rddy_f[gj + 1]) : 0.0f;
    return c;
}

#if MHD3D_FAST_BODY
// Contracted form: W1=DD/(|u|+c_f) (SQRT(FAST2) of the reference is |u|+c_f
// exactly, c_f**2=GAMMA*TT+B**2*OBETA/RO), reduced as max((|u|+c_f)/DD);
// W3 and W2 are 0.375*RE*Y and (0.5*REPR*CV/RKAPA(K))*Y with Y=DD*DD*RO; one
// reciprocal of RO*TT serves 1/RO and 1/TT.
//
// Screening: each cell first asks whether it can reach the extremes its warp
// already knows (the accumulators of the CTAs that have finished, read when
// the CTA starts, and the warp's own results of earlier planes), with a
// margin of 1e-5 -- MACH**2 >= M(1-1e-5), W2/W3 <= W(1+1e-5) and
// (|u|+c_f)/DD >= (1-1e-5)/W -- without a division or a square root of its
// own: |m|**2 >= M*GAMMA*TT*RO**2, DD*DD*RO*MIN(0.375*RE, 0.5*REPR*CV/RKAPA)
// <= W, and (SQRT(|m|**2) + SQRT(RO*(GAMMA*TT*RO + B**2*OBETA)))/DD >= RO/W,
// the last with FP32 square roots of FP64 products (relative error below
// 1e-6).  Only a warp with a cell that passes forms the FP64 limits, and only
// for those cells.  The cell holding an extreme always passes, so the FP64
// minimum and maximum equal those over all cells; a non-finite value always
// passes, so the non-finite flag is exact too.
constexpr double CFL_SCREEN_LO = 1.0 - 1e-5;
constexpr double CFL_SCREEN_HI = 1.0 + 1e-5;

struct CflAcc {
    // this plane's screened-in cells (folded and reset by cfl_fold_plane)
    double smax = 0.0;                     // max of (|u|+c_f)/DD
    double wmin = __builtin_huge_val();    // min of W2, W3
    double m2 = -__builtin_huge_val();     // max of MACH**2
    unsigned bad = 0;
};

// per-warp screening record in shared memory
struct CflScreen {
    double w_best, m_best;   // the warp's best W (min of the limits) and MACH**2 so far
    double w_hi, mg_lo;      // W*(1+1e-5), M*GAMMA*(1-1e-5)
    float s_lo, pad;         // (1-1e-5)/W
};

__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void screen_set(CflScreen* t, double w, double mm, double gamma)
{
    t->w_best = w;
    t->m_best = mm;
    t->w_hi = w * CFL_SCREEN_HI;
    t->mg_lo = mm * gamma * CFL_SCREEN_LO;
    t->s_lo = (w < __builtin_huge_val()) ? (float)(CFL_SCREEN_LO / w) : 0.0f;
}

__device__ __forceinline__ CflScreen* cfl_screen_rec(unsigned long long* red)
{
    return reinterpret_cast<CflScreen*>(red + (NT / 32) * 3) + (threadIdx.x >> 5);
}
__device__ __forceinline__ const CflScreen* cfl_screen_of(const unsigned long long* red)
{
    return reinterpret_cast<const CflScreen*>(red + (NT / 32) * 3) + (threadIdx.x >> 5);
}

// start of the CTA: one lane per warp seeds its record from the global
// accumulators (keys ~0 / 0 mean nothing reduced yet)
__device__ __forceinline__ void cfl_screen_init(unsigned long long* red, const Accum* acc, const Scalars& s, int lmag)
{
    if ((threadIdx.x & 31) == 0) {
        const unsigned long long kw = __ldcg(&acc->wmin[0]), kw4 = __ldcg(&acc->wmin[3]);
        const unsigned long long km = __ldcg(&acc->umax);
        double w = kw != ~0ull ? of_key(kw) : __builtin_huge_val();
        if (lmag && kw4 != ~0ull) w = fmin(w, of_key(kw4));
        double mm = km ? of_key(km) : 0.0;
        if (!(mm >= 0.0)) mm = 0.0;
        if (!(w > 0.0)) w = __builtin_huge_val();
        screen_set(cfl_screen_rec(red), w, mm, s.gamma);
    }
}

template <bool MAG>
__device__ __forceinline__ void cfl_acc_cell(CflAcc& c, const Scalars& s, const Metrics& m, const CflScreen* scr,
                                             const CflCol& col, int gi, int gj, int kd, double ru, double rv,
                                             double rw, double ro, double tt, double bx, double by, double bz)
{
    const double mm = ru * ru + rv * rv + rw * rw;
    const double a2r = MAG ? s.gamma * tt * ro + (bx * bx + by * by + bz * bz) * s.obeta : s.gamma * tt * ro;
    const double dd = dmin(col.dd, m.ddz[kd + 1]);
    const double wv = dd * dd * ro * fmin(s.cw3, m.fw2z[kd + 1]);
    const float rddf = fmaxf(col.rdd, m.rddz_f[kd + 1]);
    const float sf = (sqrt_approx((float)mm) + sqrt_approx((float)(ro * a2r))) * rddf;
    const double w_hi = scr->w_hi, mg_lo = scr->mg_lo;
    const float s_lo = scr->s_lo;
    const bool cand = !(wv > w_hi) || !(mm < mg_lo * tt * ro * ro) || !(sf < (float)ro * s_lo);
    if (__any_sync(__activemask(), cand)) {
        if (cand) {
            const double rp = 1.0 / (ro * tt);
            const double r = tt * rp;
            const double uu = mm * (r * r);
            const double mach2 = s.ogamma * uu * (ro * rp);
            const double a2 = a2r * r;
            const double sp = (uu > 0.0 ? uu * rsqrt(uu) : 0.0) + a2 * rsqrt(a2);
            const double rdd = fmax(fmax(m.rddx[gi + 1], m.rddy[gj + 1]), m.rddz[kd + 1]);
            const double sr = sp * rdd;
            const double y = dd * dd * ro;
            const double w = fmin(s.cw3 * y, m.fw2z[kd + 1] * y);
            c.smax = fmax(c.smax, sr);
            c.wmin = fmin(c.wmin, w);
            c.m2 = fmax(c.m2, mach2);
            c.bad |= (unsigned)(!(sr > 0.0 && sr <= DBL_MAX) || !(fabs(w) <= DBL_MAX) || !(fabs(mach2) <= DBL_MAX));
        }
    }
}

// the top wall's cells (formed in the pass of plane 3): nothing plane-bound
template <bool MAG>
__device__ __forceinline__ void cfl_acc_direct(CflAcc& c, const Scalars& s, const Metrics& m, const CflScreen* scr,
                                               const CflCol& col, int gi, int gj, int kd, double ru, double rv,
                                               double rw, double ro, double tt, double bx, double by, double bz)
{
    cfl_acc_cell<MAG>(c, s, m, scr, col, gi, gj, kd, ru, rv, rw, ro, tt, bx, by, bz);
}

// end of a plane (all lanes): when a cell of the warp was formed in FP64,
// fold the warp's extremes into its keys and its screening record
__device__ __forceinline__ void cfl_fold_plane(unsigned long long* red, CflAcc& c, double, const Scalars& s)
{
    const double gamma = s.gamma;
    double smax = c.smax, wmin = c.wmin, m2 = c.m2;
    if (__any_sync(0xffffffffu, smax > 0.0 || wmin < __builtin_huge_val() || m2 > -__builtin_huge_val())) {
        for (int o = 16; o > 0; o >>= 1) {
            smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
            wmin = fmin(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
            m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        if ((threadIdx.x & 31) == 0) {
            if (smax > 0.0) wmin = fmin(wmin, 1.0 / smax);
            unsigned long long* r = red + (threadIdx.x >> 5) * 3;
            r[0] = min(r[0], key_of(wmin));
            if (m2 > -__builtin_huge_val()) r[1] = max(r[1], key_of(m2));
            CflScreen* t = cfl_screen_rec(red);
            const double w = (wmin > 0.0) ? fmin(t->w_best, wmin) : t->w_best;
            const double mm = (m2 >= 0.0) ? fmax(t->m_best, m2) : t->m_best;
            screen_set(t, w, mm, gamma);
        }
        c.smax = 0.0;
        c.wmin = __builtin_huge_val();
        c.m2 = -__builtin_huge_val();
    }
}

__device__ __forceinline__ void cfl_commit_acc(Accum* acc, unsigned long long* red, CflAcc& c)
{
    unsigned bad = c.bad;
    for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    unsigned long long* r = red + (threadIdx.x >> 5) * 3;
    if ((threadIdx.x & 31) == 0) r[2] |= bad;
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
#else
// Reference rounding: every limit as STEP forms it.  W2=X/RKAPA(K) with
// X=0.5*DD*DD*REPR*CV*RO is reduced per plane: RKAPA(K) is one value over a
// plane and X->X/RKAPA(K) is monotone (correctly rounded), so the plane's
// minimum of W2 is min(Xmin/RKAPA(K), Xmax/RKAPA(K)) bit for bit, and W2 is
// non-finite somewhere on the plane exactly when X is or one of those two is.
struct CflAcc {
    unsigned long long kmin = ~0ull, kmu = 0ull;    // W1, W3 (and direct W2); MACH**2
    unsigned long long kxmin = ~0ull, kxmax = 0ull; // X over this plane
    unsigned bad = 0;
};
struct CflScreen {};   // every cell is formed as STEP forms it: no screening
__device__ __forceinline__ void cfl_screen_init(unsigned long long*, const Accum*, const Scalars&, int) {}
__device__ __forceinline__ const CflScreen* cfl_screen_of(const unsigned long long*) { return nullptr; }

template <bool MAG>
__device__ __forceinline__ void cfl_acc_cell(CflAcc& c, const Scalars& s, const Metrics& m, const CflScreen*,
                                             const CflCol&, int gi, int gj, int kd, double ru, double rv, double rw,
                                             double ro, double tt, double bx, double by, double bz)
{
    double w1, x, w3, mach2;
    cfl_terms<MAG>(s, ru, rv, rw, ro, tt, bx, by, bz, cell_dd(m, gi, gj, kd), w1, x, w3, mach2);
    c.kmin = min(c.kmin, min(key_of(w1), key_of(w3)));
    c.kxmin = min(c.kxmin, key_of(x));
    c.kxmax = max(c.kxmax, key_of(x));
    c.kmu = max(c.kmu, key_of(mach2));
    c.bad |= (unsigned)!(isfinite(w1) && isfinite(x) && isfinite(w3) && isfinite(mach2));
}

// a cell whose RKAPA is not that of the plane being folded (the top wall's,
// formed in the pass of plane 3)
template <bool MAG>
__device__ __forceinline__ void cfl_acc_direct(CflAcc& c, const Scalars& s, const Metrics& m, const CflScreen*,
                                               const CflCol&, int gi, int gj, int kd, double ru, double rv, double rw,
                                               double ro, double tt, double bx, double by, double bz)
{
    CflPart cp;
    cfl_cell<MAG>(s, ru, rv, rw, ro, tt, bx, by, bz, cell_dd(m, gi, gj, kd), m.rkapa[kd + 1], cp);
    c.kmin = min(c.kmin, min(min(key_of(cp.w1), key_of(cp.w2)), key_of(cp.w3)));
    c.kmu = max(c.kmu, key_of(cp.mach2));
    c.bad |= (unsigned)cp.bad;
}

// end of a plane: W2 of the plane's cells from the warp's X range
__device__ __forceinline__ void cfl_fold_plane(unsigned long long* red, CflAcc& c, double rk, const Scalars&)
{
    const unsigned long long xlo = warp_min_u64(c.kxmin), xhi = warp_max_u64(c.kxmax);
    c.kxmin = ~0ull;
    c.kxmax = 0ull;
    if ((threadIdx.x & 31) == 0 && xlo != ~0ull) {
        const double a = of_key(xlo) / rk, b = of_key(xhi) / rk;
        unsigned long long* r = red + (threadIdx.x >> 5) * 3;
        r[0] = min(r[0], min(key_of(a), key_of(b)));
        if (!(isfinite(a) && isfinite(b))) r[2] = 1ull;
    }
}

__device__ __forceinline__ void cfl_commit_acc(Accum* acc, unsigned long long* red, CflAcc& c)
{
    const unsigned long long kmin = warp_min_u64(c.kmin), kmu = warp_max_u64(c.kmu);
    unsigned bad = c.bad;
    for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    unsigned long long* r = red + (threadIdx.x >> 5) * 3;
    if ((threadIdx.x & 31) == 0) {
        r[0] = min(r[0], kmin);
        r[1] = max(r[1], kmu);
        r[2] |= bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long k1 = ~0ull, km = 0ull, b = 0ull;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            k1 = min(k1, red[i * 3 + 0]);
            km = max(km, red[i * 3 + 1]);
            b |= red[i * 3 + 2];
        }
        atomicMin(&acc->wmin[0], k1);
        atomicMax(&acc->umax, km);
        if (b) atomicOr(&acc->bad, 1u);
    }
}
#endif

