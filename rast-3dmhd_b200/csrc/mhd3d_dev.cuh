// mhd3d_dev.cuh -- device-side data structures shared by the step kernels.
//
// Layout in HBM (one handle):
//   U, U' (ping-pong): nf fields x (NPZ+2) planes x (NPY+2) rows x upitch
//              doubles, exactly the reference's (NX,NY,NZ) index space: the
//              periodic x/y halo at index 0 and NPX+1 / NPY+1, the z ghost
//              planes at 0 and NPZ+1 (never refreshed by the reference except
//              RO, which FLUXES inverts there on every call, 3dmhdsub.f:1386-1391
//              -- the two U buffers carry the two values).  upitch = NPX+2
//              rounded up to even, so every row starts on 16 bytes and a tile
//              with its halo is one in-bounds TMA box.  Field-major, x fastest.
//   Z        : nf fields x NPZ x NPY x zpitch, interior cells only.
#pragma once

#ifndef MHD3D_MINB
#define MHD3D_MINB 3   // FP64 stage CTAs per SM: 3 x 128 threads x 168 registers, 3 x 72 KB shared
#endif
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>

namespace mhd3d {

#ifndef MHD3D_TY
#define MHD3D_TY 4
#endif
#ifndef MHD3D_ZCHUNK
#define MHD3D_ZCHUNK 64           // planes a CTA marches through (z chunk length target)
#endif
constexpr int TX = 32;            // tile width (one warp per row)
constexpr int TY = MHD3D_TY;      // tile rows (threads per CTA = 32*TY)
constexpr int NT = TX * TY;       // threads per CTA
constexpr int BW = TX + 2;        // TMA box row: x0-1 .. x0+TX
constexpr int BH = TY + 2;        // TMA box rows: y0-1 .. y0+TY
constexpr int BSLOT = BW * BH;    // doubles of one field in one plane box

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
    double cw3;        // 0.375*RE, the factor of DD*DD*RO in W3 (fast-mode CFL)
    double tb, tp, tc, hh, theta_tp;
    double top_flux;   // C23*DZ*THETA at the top wall (ITC=1, 2856-2868)
    double top_dz;     // DZ at the top wall
    double bot_flux;   // C23*DZ*THETA/RKAPA at the bottom wall (IZC=1, 2925-2941)
    double dtmin, timi;
    float ogamma_f, gamma_f, obeta_f;   // 1/GAMMA, GAMMA, OBETA rounded to FP32 (fast-mode CFL screening)
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
    // fast mode: HX*DXXDX, HX*D2XXDX2, H2X*DXXDX**2 and the same in y and z
    const double *fax, *fbx, *fcx, *fay, *fby, *fcy, *faz, *fbz, *fcz;
    // fast-mode CFL: 1/DDX, 1/DDY, 1/DDZ and 0.5*REPR*CV/RKAPA(K)
    const double *rddx, *rddy, *rddz, *fw2z;
    // the same rounded to FP32 for the CFL screening: 1/DD and DD per axis,
    // MIN(0.375*RE, 0.5*REPR*CV/RKAPA(K)) per plane
    const float *rddx_f, *rddy_f, *rddz_f, *ddx_f, *ddy_f, *ddz_f, *wfz_f;
};

struct StageArgs {
    CUtensorMap map_u;      // TMA map of the input U buffer (x, y, z, field)
    CUtensorMap map_z;      // TMA map of Z (x, y, z, field)
    const double* u_in;     // current state
    double* u_out;          // next state (other ping-pong buffer)
    double* z;              // Z (read in stages 2,3; written in stages 1,2)
    double* f_out;          // RHS output (RHS-only launch), Z layout
    Control* ctl;
    Accum* acc;
    Metrics m;
    Scalars s;
    size_t uf, uz;          // U: doubles per field, per plane
    size_t zf, zz;          // Z: doubles per field, per plane
    int upitch, zpitch;
    int ntx;                // tiles along x
    int zlen;               // planes per z chunk
    int nchunks;
    long long wait_first;   // poll limit of a CTA's first ring wait (WAIT_LIMIT; lowered only by tests)
};

// ---- FP32 form ----------------------------------------------------------
// The state is held in FP32 as perturbations from FP64 background profiles
// (horizontal means of TT, RO, BX, BY, BZ per plane, taken when the state is
// uploaded; the momenta have none).  Every term of the right-hand side that
// involves a z difference of a background is formed on the host in FP64 and
// rounded once to FP32 per plane (PlaneBg); x and y differences of a
// background vanish, so the FP32 arithmetic only ever sees perturbation-sized
// differences.  Metrics stay FP64 in memory; the CFL reduction is FP64.
#ifndef MHD3D_TY32
#define MHD3D_TY32 4
#endif
#ifndef MHD3D_MINB32
#define MHD3D_MINB32 5   // FP32 stage CTAs per SM: 5 x 128 threads x 96 registers, 5 x 34 KB shared
#endif
constexpr int TY32 = MHD3D_TY32;        // tile rows of the FP32 kernel
constexpr int NT32 = TX * TY32;
constexpr int BW32 = 36;                // TMA box row: x0-1 .. x0+34 (36 floats = 144 B, a 16-B multiple)
constexpr int BH32 = TY32 + 2;
constexpr int BSLOT32 = BW32 * BH32;

// Per-plane constants of the FP32 kernel, rounded once from FP64 on the host
// and read as one aligned record per plane.
struct alignas(16) PlaneBg {
    float az, bzq, czq, rka, dka;   // HZ*DZZDZ, HZ*D2ZZDZ2, H2Z*DZZDZ**2, RKAPA, DKAPA
    float rddz, ddz, fw2z;          // 1/DDZ, DDZ, 0.5*REPR*CV/RKAPA (CFL)
    float robm, robc, robp;         // RHOb of planes K-1, K, K+1
    float ttbm, ttbc, ttbp;         // Tb of planes K-1, K, K+1
    float tz;                       // Tb(K+1)-Tb(K-1)
    float tlz;                      // z part of the Laplacian of Tb: tz*BZQ(K) + (Tb(K+1)+Tb(K-1)-2Tb(K))*CZQ(K)
    float fw;                       // GRAV*RHOb(K) - (Pb(K+1)-Pb(K-1))*AZ(K), Pb=RHOb*Tb
    float bx, by, bz;               // Bb(K)
    float bxz, byz, bzz;            // Bb(K+1)-Bb(K-1)
    float bxlz, bylz, bzlz;         // z part of the Laplacian of Bb (one-sided on the walls, like B's)
    float pad[2];
};

// Run constants of the FP32 kernel (Scalars rounded once to FP32).
struct Scalars32 {
    float grav, ore, c13, c43, tmp13, tmpa, tmpb, tmpc, ocv;
    float omx, omz, orm, obeta, tmpm;
    float ogamma, gamma, cw3;
};

// Per-column constants of the FP32 kernel: HX*DXXDX, HX*D2XXDX2,
// H2X*DXXDX**2, 1/DDX, DDX (and the same in y).
struct alignas(16) ColC {
    float a, b, c, rdd;
    float dd, pad[3];
};

struct StageArgs32 {
    CUtensorMap map_u;
    CUtensorMap map_z;
    const float* u_in;
    float* u_out;
    float* z;
    float* f_out;
    Control* ctl;
    Accum* acc;
    Metrics m;
    Scalars s;
    const float* rob;         // RHOb at every U plane (Fortran K=1..NZ)
    const float* ttb;         // Tb at every U plane
    const double* bgd;        // FP64 backgrounds: RHOb, Tb, BXb, BYb, BZb, NZ values each
    const PlaneBg* pb;        // per interior plane
    const ColC* cx;           // per x column (Fortran I=1..NX)
    const ColC* cy;           // per y row (Fortran J=1..NY)
    Scalars32 s32;
    const float* fcl;         // learned-closure tendencies (RU,RV,RW,TT,BX,BY,BZ in the Z layout) or null
    const int* fcl_flag;      // non-zero: the closure's error indicator tripped for this step
    double top_lin, top_tb;   // C43*Tb(3)-C13*Tb(4)-Tb(2) and Tb(2): top-wall temperature in perturbation form
    float t_top_fix, t_top_fix4, t_top_flux, t_bot;   // wall T' constants (ITC 0/2/4, ITC=4 left half, ITC=1; IZC)
    size_t uf, uz, zf, zz;
    int upitch, zpitch;
    int ntx, zlen, nchunks;
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
size_t stage_smem_bytes(int lmag);
cudaError_t launch_stage(int stage, const StageArgs& a, cudaStream_t st);
cudaError_t launch_cfl(const StageArgs& a, cudaStream_t st);
cudaError_t launch_bcon(const StageArgs& a, cudaStream_t st);
}
namespace fast {
size_t stage_smem_bytes(int lmag);
cudaError_t launch_stage(int stage, const StageArgs& a, cudaStream_t st);
cudaError_t launch_cfl(const StageArgs& a, cudaStream_t st);
cudaError_t launch_bcon(const StageArgs& a, cudaStream_t st);
}
// FP32 form (FMA contraction, FP64 CFL reduction)
namespace f32 {
size_t stage_smem_bytes(int lmag);
cudaError_t launch_stage(int stage, const StageArgs32& a, cudaStream_t st);
cudaError_t launch_cfl(const StageArgs32& a, cudaStream_t st);
// persistent multi-grid form (ensembles) with tile rows ty (2, 4 or 8): args,
// order, item_base in device memory; nblocks == 0 only prepares the kernel
// attributes (before a graph capture)
cudaError_t launch_stage_multi(int stage, int lmag, int lrot, int ty, const StageArgs32* args, const int* order,
                               const int* item_base, int nmem, unsigned* counter, int nblocks, cudaStream_t st);
bool multi_tile_rows_ok(int ty);
size_t multi_smem_bytes(int lmag, int ty);
}

}  // namespace mhd3d
