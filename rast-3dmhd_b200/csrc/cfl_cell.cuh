// cfl_cell.cuh -- the per-cell CFL and Mach-number terms of STEP
// (3dmhdsub.f:749-857, ISW=1), shared by the step kernels and the
// allocation-free reduction.  The arithmetic mode (FMA contraction or not)
// is that of the translation unit including it.
#pragma once
#include "mhd3d_dev.cuh"

namespace mhd3d {
namespace MHD3D_NS {

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

// CFL limits of one cell (STEP loops 10-50 and 2, 3dmhdsub.f:749-857).
struct CflPart {
    double w1, w2, w3, w4, mach2;
    bool bad;
};

// The limits of one cell before the division of W2 by RKAPA(K):
// X=0.5*DD*DD*REPR*CV*RO, so that W2=X/RKAPA(K) in the reference's order.
template <bool MAG>
__device__ __forceinline__ void cfl_terms(const Scalars& s, double ru, double rv, double rw, double ro, double tt,
                                          double bx, double by, double bz, double dd, double& w1, double& x,
                                          double& w3, double& mach2)
{
    const double r = 1.0 / ro;
    const double uu = (ru * ru + rv * rv + rw * rw) * (r * r);
    mach2 = s.ogamma * uu / tt;
    double fast2;
    if (MAG) {
        const double b2o = (bx * bx + by * by + bz * bz) * s.obeta / ro;
        fast2 = uu + s.gamma * tt + b2o + 2.0 * sqrt(uu * (s.gamma * tt + b2o));
    } else {
        fast2 = uu + s.gamma * tt + 2.0 * sqrt(uu * s.gamma * tt);
    }
    w1 = dd / sqrt(fast2);
    x = 0.5 * dd * dd * s.repr * s.cv * ro;
    w3 = 0.375 * dd * dd * s.re * ro;
}

template <bool MAG>
__device__ __forceinline__ void cfl_cell(const Scalars& s, double ru, double rv, double rw, double ro, double tt,
                                         double bx, double by, double bz, double dd, double rkapa, CflPart& c)
{
    double x;
    cfl_terms<MAG>(s, ru, rv, rw, ro, tt, bx, by, bz, dd, c.w1, x, c.w3, c.mach2);
    c.w2 = x / rkapa;
    c.w4 = MAG ? 0.5 * dd * dd * s.rm : 0.0;
    c.bad = !(isfinite(c.w1) && isfinite(c.w2) && isfinite(c.w3) && isfinite(c.mach2));
}

__device__ __forceinline__ double cell_dd(const Metrics& m, int gi, int gj, int k)
{
    // DD=MIN(DDX(I),DDY(J),DDZ(K))
    return dmin(dmin(m.ddx[gi + 1], m.ddy[gj + 1]), m.ddz[k + 1]);
}

}  // namespace MHD3D_NS
}  // namespace mhd3d
