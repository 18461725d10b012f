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

#if MHD3D_FAST_BODY
// Contracted form: W1=DD/(|u|+c_f) (SQRT(FAST2) of the reference is |u|+c_f
// exactly, c_f**2=GAMMA*TT+B**2*OBETA/RO), reduced as max((|u|+c_f)/DD);
// W3 and W2 are 0.375*RE*Y and (0.5*REPR*CV/RKAPA(K))*Y with Y=DD*DD*RO; one
// reciprocal of RO*TT serves 1/RO and 1/TT.
struct CflAcc {
    double smax = 0.0;        // max over cells of (|u|+c_f)/DD
    double wmin = __builtin_huge_val();   // min of W2, W3
    double m2 = -__builtin_huge_val();    // max of MACH**2
    unsigned bad = 0;
};

template <bool MAG>
__device__ __forceinline__ void cfl_acc_cell(CflAcc& c, const Scalars& s, const Metrics& m, int gi, int gj, int kd,
                                             double ru, double rv, double rw, double ro, double tt, double bx,
                                             double by, double bz)
{
    const double rp = 1.0 / (ro * tt);
    const double r = tt * rp;
    const double uu = (ru * ru + rv * rv + rw * rw) * (r * r);
    const double mach2 = s.ogamma * uu * (ro * rp);
    double a2 = s.gamma * tt;
    if (MAG) a2 += (bx * bx + by * by + bz * bz) * s.obeta * r;
    const double sp = (uu > 0.0 ? uu * rsqrt(uu) : 0.0) + a2 * rsqrt(a2);
    const double rdd = fmax(fmax(m.rddx[gi + 1], m.rddy[gj + 1]), m.rddz[kd + 1]);
    const double dd = dmin(dmin(m.ddx[gi + 1], m.ddy[gj + 1]), m.ddz[kd + 1]);
    const double sr = sp * rdd;
    const double y = dd * dd * ro;
    const double w = fmin(s.cw3 * y, m.fw2z[kd + 1] * y);
    c.smax = fmax(c.smax, sr);
    c.wmin = fmin(c.wmin, w);
    c.m2 = fmax(c.m2, mach2);
    c.bad |= (unsigned)(!(sr > 0.0 && sr <= DBL_MAX) || !(fabs(w) <= DBL_MAX) || !(fabs(mach2) <= DBL_MAX));
}

// the top wall's cells (formed in the pass of plane 3): nothing plane-bound
template <bool MAG>
__device__ __forceinline__ void cfl_acc_direct(CflAcc& c, const Scalars& s, const Metrics& m, int gi, int gj, int kd,
                                               double ru, double rv, double rw, double ro, double tt, double bx,
                                               double by, double bz)
{
    cfl_acc_cell<MAG>(c, s, m, gi, gj, kd, ru, rv, rw, ro, tt, bx, by, bz);
}

__device__ __forceinline__ void cfl_fold_plane(unsigned long long*, CflAcc&, double) {}

__device__ __forceinline__ void cfl_commit_acc(Accum* acc, unsigned long long* red, CflAcc& c)
{
    double smax = c.smax, wmin = c.wmin, m2 = c.m2;
    unsigned bad = c.bad;
    for (int o = 16; o > 0; o >>= 1) {
        smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        wmin = fmin(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    unsigned long long* r = red + (threadIdx.x >> 5) * 3;
    if ((threadIdx.x & 31) == 0) {
        if (smax > 0.0) wmin = fmin(wmin, 1.0 / smax);
        r[0] = min(r[0], key_of(wmin));
        r[1] = max(r[1], key_of(m2));
        r[2] |= bad;
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

template <bool MAG>
__device__ __forceinline__ void cfl_acc_cell(CflAcc& c, const Scalars& s, const Metrics& m, int gi, int gj, int kd,
                                             double ru, double rv, double rw, double ro, double tt, double bx,
                                             double by, double bz)
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
__device__ __forceinline__ void cfl_acc_direct(CflAcc& c, const Scalars& s, const Metrics& m, int gi, int gj, int kd,
                                               double ru, double rv, double rw, double ro, double tt, double bx,
                                               double by, double bz)
{
    CflPart cp;
    cfl_cell<MAG>(s, ru, rv, rw, ro, tt, bx, by, bz, cell_dd(m, gi, gj, kd), m.rkapa[kd + 1], cp);
    c.kmin = min(c.kmin, min(min(key_of(cp.w1), key_of(cp.w2)), key_of(cp.w3)));
    c.kmu = max(c.kmu, key_of(cp.mach2));
    c.bad |= (unsigned)cp.bad;
}

// end of a plane: W2 of the plane's cells from the warp's X range
__device__ __forceinline__ void cfl_fold_plane(unsigned long long* red, CflAcc& c, double rk)
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

