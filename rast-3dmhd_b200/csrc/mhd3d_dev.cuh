// mhd3d_dev.cuh -- device-side data structures shared by the step kernels.
//
// Layout in HBM (one handle):
//   U, U', Z : nf fields x npz planes x npy rows x pitch doubles, interior
//              cells only (Fortran I=2..NX-1, J=2..NY-1, K=2..NZ-1 map to
//              i=I-2, j=J-2, k=K-2).  Field-major, x fastest.  The periodic
//              x/y halos of the reference are not stored: every load wraps.
//   ghost    : the reference's z ghost planes K=1 and K=NZ for RU,RV,RW,TT,
//              BX,BY,BZ (never refreshed by the reference).
//   gro      : two copies of the RO ghost planes; FLUXES inverts RO there on
//              every call (3dmhdsub.f:1386-1391), the copies ping-pong.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>

namespace mhd3d {

constexpr int TX = 32;            // tile width (one warp per row)
constexpr int TY = 8;             // tile rows
constexpr int NT = TX * TY;       // threads per CTA
constexpr int SX = TX + 2;        // shared-memory row incl. periodic halo
constexpr int SY = TY + 2;

enum Field { F_RU = 0, F_RV, F_RW, F_TT, F_RO, F_BX, F_BY, F_BZ };

// Run-constant scalars, in the values the reference holds (float-rounded
// REAL(4) literals included) plus products the reference forms once per
// FLUXES call (TMP=OCV/REPR etc.), formed here with the same operations.
struct Scalars {
    double c13, c23, c43;
    double hx, h2x, hy, h2y, hz, h2z;
    double gam1, gam2, gam3, zeta1, zeta2;
    double cv, ocv, ore, re, repr, theta, grav, gamma, ogamma, sf, rm;
    double omx, omz, orm, obeta;
    double tmp_cond;   // OCV/REPR          (3dmhdsub.f:1584)
    double tmp_a;      // OCV*ORE           (1911, 1952, 2059, 2091)
    double tmp_b;      // C43*OCV*ORE       (1968, 2016)
    double tmp_13;     // C13*ORE           (1926, 2031, 2082)
    double tmp_m;      // OBETA*ORM*OCV     (2222, 2420, 2511)
    double tb, tp, tc, hh, theta_tp;
    double top_flux;   // C23*DZ*THETA at the top wall (ITC=1, 2856-2868)
    double top_dz;     // DZ at the top wall
    double bot_flux;   // C23*DZ*THETA/RKAPA at the bottom wall (IZC=1, 2925-2941)
    double dtmin, timi;
    int npx, npy, npz, pitch;
    int lmag, lrot, izcon, itcon, ibcon, plume;
};

// Step bookkeeping kept on the device so that many steps run without a
// host round trip (COMMON/CTIM, ITER, TRACE).
struct Control {
    double dt, umach;             // DT, UMACH of the step about to run
    double last_dt, last_umach;   // of the last completed step
    double timc, timt, timi;
    int nit;
    int stop;                     // nonzero: later stage kernels return at once
    int status;                   // MHD3D_* code behind stop
    int gparity;                  // which gro copy is current at step start
};

// CFL accumulators: order-preserving 64-bit keys of doubles.
struct Accum {
    unsigned long long wmin[4];
    unsigned long long umax;
    unsigned int bad;
    unsigned int pad;
};

struct Metrics {
    // 1-D arrays in Fortran index order (C index = Fortran index - 1)
    const double *dxxdx, *d2xxdx2, *ddx;
    const double *dyydy, *d2yydy2, *ddy;
    const double *dzzdz, *d2zzdz2, *ddz;
    const double *rkapa, *dkapa;
    const double *plume_gx, *plume_gy;   // EXP(CLN*(EXX(I)-XP)**2), EXP(CLN*(WYY(J)-YP)**2)
};

struct StageArgs {
    const double* u_in;     // current state
    double* u_out;          // next state (other ping-pong buffer)
    double* z;              // Z (read in stages 2,3; written in stages 1,2)
    double* f_out;          // RHS output (RHS-only launch)
    const double* ghost;    // [8][2][npy][pitch]
    double* gro;            // [2 copies][2 planes][npy][pitch]
    Control* ctl;
    Accum* acc;
    Metrics m;
    Scalars s;
    size_t fstride;         // doubles per field
    size_t pstride;         // doubles per plane (npy*pitch)
    int ntx;                // tiles along x
    int zlen;               // planes per z chunk
    int nchunks;
};

// order-preserving map double -> uint64 and back
__host__ __device__ inline unsigned long long key_of(double x)
{
    unsigned long long b;
    memcpy(&b, &x, 8);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double of_key(unsigned long long k)
{
    unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    double x;
    memcpy(&x, &b, 8);
    return x;
}

// Launchers, one set per arithmetic mode (compiled from the same source
// with and without FMA contraction).
namespace exact {
cudaError_t launch_stage(int stage, const StageArgs& a, cudaStream_t st);
cudaError_t launch_cfl(const StageArgs& a, cudaStream_t st);
cudaError_t launch_bcon(const StageArgs& a, cudaStream_t st);
}
namespace fast {
cudaError_t launch_stage(int stage, const StageArgs& a, cudaStream_t st);
cudaError_t launch_cfl(const StageArgs& a, cudaStream_t st);
cudaError_t launch_bcon(const StageArgs& a, cudaStream_t st);
}

}  // namespace mhd3d
