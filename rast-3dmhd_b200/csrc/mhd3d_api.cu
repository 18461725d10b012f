// mhd3d_api.cu -- the C-ABI of include/mhd3d.h: handle life cycle, layout
// conversion between the reference's Fortran arrays and the device layout,
// and the step loop with its device-side bookkeeping.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/mhd3d.h"
#include "mhd3d_dev.cuh"
#include "ring.cuh"
#include "smem_attr.cuh"

namespace mhd3d {
namespace {

struct Handle {
    mhd3d_params p;
    int dev = -1;
    cudaStream_t st = nullptr;
    int nf = 0;
    int upitch = 0, urows = 0, zpitch = 0, zrows = 0;
    size_t uf = 0, uz = 0, zf = 0, zz = 0;
    double* ubuf[2] = {nullptr, nullptr};
    int cur = 0;               // ubuf[cur] holds the current state
    CUtensorMap map_u[2];      // TMA maps of the two U buffers
    CUtensorMap map_z;
    CUtensorMap emap_u[2];     // the same for the tile rows of an ensemble (FP32 members)
    CUtensorMap emap_z;
    int ety = 0;               // tile rows emap_* were made for (0: none)
    double* z = nullptr;
    double* stage = nullptr;   // one Fortran (NX,NY,NZ) field
    double* stage2 = nullptr;  // a second one: upload/download alternate between the two
    cudaStream_t cst = nullptr;             // host<->device copies of upload/download
    cudaEvent_t ev_copy[2] = {nullptr, nullptr}, ev_kern[2] = {nullptr, nullptr};
    double* fout = nullptr;
    double* met = nullptr;     // all 1-D arrays, packed
    float* metf = nullptr;     // FP32 copies for the fast-mode CFL screening, packed
    Control* ctl = nullptr;
    Accum* acc = nullptr;
    Metrics m{};
    Scalars s{};
    int ntx = 0, zlen = 0, nchunks = 0;
    bool dt_valid = false;
    unsigned long long w4key = ~0ull;   // key of min over cells of W4 (MHD), else ~0
    // FP32 form: the buffers above hold floats; background profiles
    bool f32 = false;
    double* bgd = nullptr;        // 5 x NZ: RHOb, Tb, BXb, BYb, BZb (FP64)
    float* bg32 = nullptr;        // 2 x NZ: RHOb, Tb (FP32)
    PlaneBg* pb = nullptr;        // per interior plane
    std::vector<double> faz_h, fbz_h, fcz_h;   // host copies of the z stencil factors
    std::vector<double> rka_h, dka_h, ddz_h;   // and of RKAPA, DKAPA, DDZ
    ColC* cxy = nullptr;                       // FP32 column constants: NX in x, then NY in y
    // learned closure attached to an FP32 handle (mhd3d_closure_set)
    bool clo = false;
    void* cbuf = nullptr;                      // one allocation for everything below
    __nv_bfloat16 *cw[3] = {nullptr, nullptr, nullptr};
    float *cb[3] = {nullptr, nullptr, nullptr}, *cin_scale = nullptr, *cout_scale = nullptr;
    __nv_bfloat16 *cfeat = nullptr, *cact1 = nullptr, *cact2 = nullptr;
    float *cpred = nullptr, *cfcl = nullptr;
    float* cbias = nullptr;   // closure: per-plane bias tendency [7][NPZ] (null: none)
    float* cbtend = nullptr;  // that bias broadcast into the Z layout (7 fields), then a zero flag: the
                              // tendencies a step adds when no network is attached
    double* cmeans = nullptr;                  // 3 x NPZ horizontal means (T, RO, BY)
    double* hpart = nullptr;                   // 3 x NPZ x HM_SPLIT partial sums of those means
    int* cflag = nullptr;                      // [0] trip flag of the current evaluation, [1] trips, [2] evaluations, [3] kernel error
    float ctrip = 1.f;
    Scalars32 s32{};
    double top_lin = 0.0, top_tb = 0.0;
    float t_top_fix = 0.f, t_top_fix4 = 0.f, t_top_flux = 0.f, t_bot = 0.f;
    cudaStream_t own = nullptr;   // the handle's stream; st may be a caller's
    // asynchronous stepping: state at the last sync and steps enqueued since
    int nit_base = 0, cur_base = 0, pending = 0;
    // poll limit of the stage kernels' first ring wait (tests lower it)
    long long wait_first = WAIT_LIMIT;
    // per-stage event timing
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_stage;    // stage of each recorded pair
    size_t ev_used = 0;
};

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) {                                                                 \
            std::fprintf(stderr, "mhd3d: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_),   \
                         __FILE__, __LINE__);                                                     \
            return e_ == cudaErrorMemoryAllocation ? MHD3D_ERR_NOMEM : MHD3D_ERR_CUDA;            \
        }                                                                                        \
    } while (0)

__global__ void k_unpack(const double* __restrict__ fort, double* __restrict__ u0, double* __restrict__ u1,
                         int npx, int npy, int npz, int upitch, size_t uz)
{
    // Fortran (NX,NY,NZ) -> both U buffers, halos refreshed from the interior
    // (COMMUNICATE's periodic copies), ghost planes kept
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t n = (size_t)NX * NY * NZ;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(q % NX), J = (int)((q / NX) % NY), K = (int)(q / ((size_t)NX * NY));
        const int Is = I == 0 ? npx : (I == NX - 1 ? 1 : I);
        const int Js = J == 0 ? npy : (J == NY - 1 ? 1 : J);
        const double v = fort[(size_t)Is + (size_t)NX * ((size_t)Js + (size_t)NY * K)];
        const size_t d = (size_t)K * uz + (size_t)J * upitch + I;
        u0[d] = v;
        u1[d] = v;
    }
}

__global__ void k_pack(const double* __restrict__ u, double* __restrict__ fort, int npx, int npy, int npz,
                       int upitch, size_t uz)
{
    // U layout -> Fortran (NX,NY,NZ): the same index space, halos and ghost planes included
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t n = (size_t)NX * NY * NZ;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(q % NX), J = (int)((q / NX) % NY), K = (int)(q / ((size_t)NX * NY));
        fort[q] = u[(size_t)K * uz + (size_t)J * upitch + I];
    }
}

__global__ void k_pack_interior(const double* __restrict__ f, double* __restrict__ fort, int npx, int npy,
                                int npz, int zpitch, size_t zz)
{
    // Z layout (interior cells) -> Fortran (NX,NY,NZ) with zeros outside the interior
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t n = (size_t)NX * NY * NZ;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(q % NX), J = (int)((q / NX) % NY), K = (int)(q / ((size_t)NX * NY));
        double v = 0.0;
        if (I > 0 && I < NX - 1 && J > 0 && J < NY - 1 && K > 0 && K < NZ - 1)
            v = f[(size_t)(K - 1) * zz + (size_t)(J - 1) * zpitch + (I - 1)];
        fort[q] = v;
    }
}

// horizontal mean of one Fortran (NX,NY,NZ) field per plane K over the
// interior I=2..NX-1, J=2..NY-1, FP64, fixed summation order (one block per K)
__global__ void k_hmean(const double* __restrict__ fort, double* __restrict__ mean, int npx, int npy)
{
    const int NX = npx + 2, NY = npy + 2;
    const int K = blockIdx.x;
    const double* pl = fort + (size_t)K * NX * NY;
    double acc = 0.0;
    for (int q = threadIdx.x; q < npx * npy; q += blockDim.x) {
        const int i = q % npx, j = q / npx;
        acc += pl[(size_t)(j + 1) * NX + (i + 1)];
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) mean[K] = red[0] / ((double)npx * (double)npy);
}

// Fortran (NX,NY,NZ) FP64 -> both FP32 U buffers as perturbations from bg(K)
// (bg may be null: no background), halos refreshed from the interior
__global__ void k_unpack32(const double* __restrict__ fort, const double* __restrict__ bg, float* __restrict__ u0,
                           float* __restrict__ u1, int npx, int npy, int npz, int upitch, size_t uz)
{
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t n = (size_t)NX * NY * NZ;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(q % NX), J = (int)((q / NX) % NY), K = (int)(q / ((size_t)NX * NY));
        const int Is = I == 0 ? npx : (I == NX - 1 ? 1 : I);
        const int Js = J == 0 ? npy : (J == NY - 1 ? 1 : J);
        double v = fort[(size_t)Is + (size_t)NX * ((size_t)Js + (size_t)NY * K)];
        if (bg) v -= bg[K];
        const size_t d = (size_t)K * uz + (size_t)J * upitch + I;
        u0[d] = (float)v;
        u1[d] = (float)v;
    }
}

// FP32 U layout -> Fortran (NX,NY,NZ) FP64 full values
__global__ void k_pack32(const float* __restrict__ u, const double* __restrict__ bg, double* __restrict__ fort,
                         int npx, int npy, int npz, int upitch, size_t uz)
{
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t n = (size_t)NX * NY * NZ;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(q % NX), J = (int)((q / NX) % NY), K = (int)(q / ((size_t)NX * NY));
        const double v = (double)u[(size_t)K * uz + (size_t)J * upitch + I];
        fort[q] = bg ? bg[K] + v : v;
    }
}

// FP32 Z layout (interior) -> Fortran (NX,NY,NZ) FP64, zeros outside
__global__ void k_pack_interior32(const float* __restrict__ f, double* __restrict__ fort, int npx, int npy, int npz,
                                  int zpitch, size_t zz)
{
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t n = (size_t)NX * NY * NZ;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(q % NX), J = (int)((q / NX) % NY), K = (int)(q / ((size_t)NX * NY));
        double v = 0.0;
        if (I > 0 && I < NX - 1 && J > 0 && J < NY - 1 && K > 0 && K < NZ - 1)
            v = (double)f[(size_t)(K - 1) * zz + (size_t)(J - 1) * zpitch + (I - 1)];
        fort[q] = v;
    }
}

// ---- horizontally averaged profiles (HORIZONTAL_MEAN, 3dmhdsub.f:3143-3223) ----
// One block per interior plane; per-thread partial sums in a fixed order, then a
// fixed tree, so the result is deterministic.  Per-cell formulas follow the
// reference's flux diagnostics (1651-1661).
constexpr int PROF_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double* red)
{
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = PROF_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

template <bool F32>
__global__ void __launch_bounds__(PROF_THREADS) k_profiles(const void* __restrict__ ubuf, const double* __restrict__ bgd,
                                                           double* __restrict__ out, int npx, int npy, int npz,
                                                           int upitch, size_t uz, size_t uf, int lmag)
{
    __shared__ double red[PROF_THREADS];
    const int k = blockIdx.x;   // interior plane, Fortran K = k+2
    const int K0 = k + 1;       // U plane index
    const size_t NZ = (size_t)npz + 2;
    auto val = [&](int f, size_t off) -> double {
        if (F32) {
            const double v = (double)reinterpret_cast<const float*>(ubuf)[(size_t)f * uf + off];
            const int bi = f == F_RO ? 0 : f == F_TT ? 1 : f == F_BX ? 2 : f == F_BY ? 3 : f == F_BZ ? 4 : -1;
            return bi >= 0 ? bgd[bi * NZ + K0] + v : v;
        }
        return reinterpret_cast<const double*>(ubuf)[(size_t)f * uf + off];
    };
    const int n = npx * npy;
    double sro = 0.0, stt = 0.0, ske = 0.0, sen = 0.0, sme = 0.0;
    for (int q = threadIdx.x; q < n; q += PROF_THREADS) {
        const int i = q % npx, j = q / npx;
        const size_t off = (size_t)K0 * uz + (size_t)(j + 1) * upitch + (i + 1);
        const double ro = val(F_RO, off), tt = val(F_TT, off);
        const double ri = 1.0 / ro;
        const double u = val(F_RU, off) * ri, v = val(F_RV, off) * ri, w = val(F_RW, off) * ri;
        sro += ro;
        stt += tt;
        ske += 0.5 * ro * (u * u + v * v + w * w);
        sen += 2.5 * ro * tt;
        if (lmag) {
            const double bx = val(F_BX, off), by = val(F_BY, off), bz = val(F_BZ, off);
            sme += 0.5 * (bx * bx + by * by + bz * bz);
        }
    }
    const double cnt = (double)(float)n;   // FLOAT(NPX*NPY)
    const double rom = block_sum(sro, red) / cnt;
    const double ttm = block_sum(stt, red) / cnt;
    const double kem = block_sum(ske, red) / cnt;
    const double enm = block_sum(sen, red) / cnt;
    const double mem = block_sum(sme, red) / cnt;
    double sfc = 0.0;
    for (int q = threadIdx.x; q < n; q += PROF_THREADS) {
        const int i = q % npx, j = q / npx;
        const size_t off = (size_t)K0 * uz + (size_t)(j + 1) * upitch + (i + 1);
        const double ro = val(F_RO, off), tt = val(F_TT, off), rw = val(F_RW, off);
        const double ri = 1.0 / ro;
        const double u = val(F_RU, off) * ri, v = val(F_RV, off) * ri, w = rw * ri;
        sfc += -rw * (2.5 * (tt - ttm) + 0.5 * (u * u + v * v + w * w));
    }
    const double fcm = block_sum(sfc, red) / cnt;
    if (threadIdx.x == 0) {
        out[MHD3D_PROF_RHO * npz + k] = rom;
        out[MHD3D_PROF_T * npz + k] = ttm;
        out[MHD3D_PROF_KE * npz + k] = kem;
        out[MHD3D_PROF_ENTH * npz + k] = enm;
        out[MHD3D_PROF_FCONV * npz + k] = fcm;
        out[MHD3D_PROF_ME * npz + k] = mem;
    }
}

// FRADM from TTM (3dmhdsub.f:1663-1676): centred inside, one-sided at both walls
__global__ void k_frad(double* __restrict__ out, const double* __restrict__ dzzdz, const double* __restrict__ rkapa,
                       double hz, double repr, int npz)
{
    const double* ttm = out + MHD3D_PROF_T * npz;   // ttm[k] is TTM(K=k+2)
    for (int k = threadIdx.x; k < npz; k += blockDim.x) {
        const int K = k + 2;
        double d;
        if (k == 0) d = -3.0 * ttm[0] + 4.0 * ttm[1] - ttm[2];
        else if (k == npz - 1) d = 3.0 * ttm[npz - 1] - 4.0 * ttm[npz - 2] + ttm[npz - 3];
        else d = ttm[k + 1] - ttm[k - 1];
        out[MHD3D_PROF_FRAD * npz + k] = d * hz * dzzdz[K - 1] * rkapa[K - 1] / repr;
    }
}

__global__ void k_reset(Control* ctl, Accum* acc, int clear_stop, unsigned long long w4key)
{
    for (int i = 0; i < 3; ++i) acc->wmin[i] = ~0ull;
    acc->wmin[3] = w4key;
    acc->umax = 0ull;
    acc->bad = 0u;
    if (clear_stop) {
        ctl->stop = 0;
        ctl->status = 0;
    }
}

// End of a step (advance=1: NIT, TIMC, TIMT of STEP 3dmhdsub.f:1171-1173 and
// the driver's DT check 3dmhd.f:924) and DT/UMACH of the next step from the
// CFL accumulators (DT=SF*MIN(...), 3dmhdsub.f:866-873; UMACH=SQRT(...), 761).
// ---- learned closure (no counterpart in the reference) ----------------------
// Reads of a handle's state as full FP64 values, for either precision.
struct UView {
    const void* u;        // U buffer (double, or float perturbations)
    const double* bgd;    // FP32 form: backgrounds (5 x NZ), else null
    size_t uf, uz, NZ;
    int upitch, f32;
};
__device__ __forceinline__ double uget(const UView& v, int f, int i, int j, int K)
{
    // i, j, K: U-layout indices (halo / ghost plane at 0)
    const size_t off = (size_t)f * v.uf + (size_t)K * v.uz + (size_t)j * v.upitch + i;
    if (v.f32) {
        const double x = (double)static_cast<const float*>(v.u)[off];
        const int bi = f == F_RO ? 0 : f == F_TT ? 1 : f == F_BX ? 2 : f == F_BY ? 3 : f == F_BZ ? 4 : -1;
        return bi >= 0 ? v.bgd[bi * v.NZ + K] + x : x;
    }
    return static_cast<const double*>(v.u)[off];
}

// Box filter by fac in every direction (interior cells fac*i..fac*i+fac-1) of a
// fine state: the coarse state (Favre temperature TT = <RO*TT>/<RO>) in
// Fortran (NXc,NYc,NZc) arrays, and the subgrid targets channels-last
// [k][j][i][12]: tau_xx,yy,zz,xy,xz,yz = <RO u_i u_j> - <RU_i><RU_j>/<RO>,
// q_x,y,z = <RU_i TT> - <RU_i><RO TT>/<RO>, eps = <u x B> - (<RU>/<RO>) x <B>.
__global__ void k_coarsen(UView fine, int fac, int npxc, int npyc, int npzc, int lmag, double* __restrict__ cs,
                          float* __restrict__ tg)
{
    const size_t n = (size_t)npxc * npyc * npzc;
    const size_t NXc = npxc + 2, NYc = npyc + 2, NC = NXc * NYc * (npzc + 2);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int ic = (int)(q % npxc), jc = (int)((q / npxc) % npyc), kc = (int)(q / ((size_t)npxc * npyc));
        double R = 0, M[3] = {0, 0, 0}, E = 0, B[3] = {0, 0, 0}, S[6] = {0, 0, 0, 0, 0, 0}, H[3] = {0, 0, 0};
        double X[3] = {0, 0, 0};
        for (int c = 0; c < fac; ++c)
            for (int b = 0; b < fac; ++b)
                for (int a = 0; a < fac; ++a) {
                    const int i = fac * ic + a + 1, j = fac * jc + b + 1, K = fac * kc + c + 1;
                    const double ro = uget(fine, F_RO, i, j, K), tt = uget(fine, F_TT, i, j, K);
                    const double m0 = uget(fine, F_RU, i, j, K), m1 = uget(fine, F_RV, i, j, K),
                                 m2 = uget(fine, F_RW, i, j, K);
                    const double ri = 1.0 / ro, u0 = m0 * ri, u1 = m1 * ri, u2 = m2 * ri;
                    R += ro;
                    M[0] += m0; M[1] += m1; M[2] += m2;
                    E += ro * tt;
                    S[0] += m0 * u0; S[1] += m1 * u1; S[2] += m2 * u2;
                    S[3] += m0 * u1; S[4] += m0 * u2; S[5] += m1 * u2;
                    H[0] += m0 * tt; H[1] += m1 * tt; H[2] += m2 * tt;
                    if (lmag) {
                        const double bx = uget(fine, F_BX, i, j, K), by = uget(fine, F_BY, i, j, K),
                                     bz = uget(fine, F_BZ, i, j, K);
                        B[0] += bx; B[1] += by; B[2] += bz;
                        X[0] += u1 * bz - u2 * by;
                        X[1] += u2 * bx - u0 * bz;
                        X[2] += u0 * by - u1 * bx;
                    }
                }
        const double w = 1.0 / ((double)fac * fac * fac);
        R *= w; E *= w;
        for (int t = 0; t < 3; ++t) { M[t] *= w; B[t] *= w; H[t] *= w; X[t] *= w; }
        for (int t = 0; t < 6; ++t) S[t] *= w;
        const size_t fo = (size_t)(ic + 1) + NXc * ((size_t)(jc + 1) + NYc * (size_t)(kc + 1));
        cs[F_RU * NC + fo] = M[0];
        cs[F_RV * NC + fo] = M[1];
        cs[F_RW * NC + fo] = M[2];
        cs[F_TT * NC + fo] = E / R;
        cs[F_RO * NC + fo] = R;
        if (lmag) {
            cs[F_BX * NC + fo] = B[0];
            cs[F_BY * NC + fo] = B[1];
            cs[F_BZ * NC + fo] = B[2];
        }
        const double ri = 1.0 / R, v0 = M[0] * ri, v1 = M[1] * ri, v2 = M[2] * ri;
        float* o = tg + q * 12;
        o[0] = (float)(S[0] - M[0] * v0);
        o[1] = (float)(S[1] - M[1] * v1);
        o[2] = (float)(S[2] - M[2] * v2);
        o[3] = (float)(S[3] - M[0] * v1);
        o[4] = (float)(S[4] - M[0] * v2);
        o[5] = (float)(S[5] - M[1] * v2);
        o[6] = (float)(H[0] - M[0] * E * ri);
        o[7] = (float)(H[1] - M[1] * E * ri);
        o[8] = (float)(H[2] - M[2] * E * ri);
        o[9] = (float)(X[0] - (v1 * B[2] - v2 * B[1]));
        o[10] = (float)(X[1] - (v2 * B[0] - v0 * B[2]));
        o[11] = (float)(X[2] - (v0 * B[1] - v1 * B[0]));
    }
}

// Fortran (NX,NY,NZ) arrays: periodic halos from the interior, z ghost planes = wall planes
__global__ void k_fort_wrap(double* __restrict__ a, int nf, int npx, int npy, int npz)
{
    const size_t NX = npx + 2, NY = npy + 2, NZ = npz + 2, NC = NX * NY * NZ;
    const size_t n = (size_t)nf * NC;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const size_t f = q / NC, r = q % NC;
        const int I = (int)(r % NX), J = (int)((r / NX) % NY), K = (int)(r / (NX * NY));
        const bool halo = I == 0 || I == (int)NX - 1 || J == 0 || J == (int)NY - 1 || K == 0 || K == (int)NZ - 1;
        if (!halo) continue;
        const int Is = I == 0 ? npx : (I == (int)NX - 1 ? 1 : I);
        const int Js = J == 0 ? npy : (J == (int)NY - 1 ? 1 : J);
        const int Ks = K == 0 ? 1 : (K == (int)NZ - 1 ? npz : K);
        a[q] = a[f * NC + (size_t)Is + NX * ((size_t)Js + NY * (size_t)Ks)];
    }
}

// per-plane horizontal means of TT, RO, BY (network features), in two passes
// with a fixed summation order: HM_SPLIT CTAs per plane write partial sums,
// then one thread per (field, plane) adds them in order; the FP32 form sums
// the perturbations and adds the plane's background once
constexpr int HM_THREADS = 256, HM_SPLIT = 8;
__global__ void __launch_bounds__(HM_THREADS) k_hmeans3(UView v, int npx, int npy, double* __restrict__ part,
                                                        int npz, int lmag)
{
    __shared__ double red[3][HM_THREADS / 32];
    const int k = blockIdx.x, K = k + 1, b = blockIdx.y;
    const size_t fo[3] = {(size_t)F_TT * v.uf, (size_t)F_RO * v.uf, (size_t)F_BY * v.uf};
    const int nf = lmag ? 3 : 2;
    double acc[3] = {0.0, 0.0, 0.0};
    const float* uf32 = static_cast<const float*>(v.u);
    const double* uf64 = static_cast<const double*>(v.u);
    // rows j of this CTA's share, x along the threads
    for (int j = b; j < npy; j += HM_SPLIT)
        for (int i = threadIdx.x; i < npx; i += HM_THREADS) {
            const size_t off = (size_t)K * v.uz + (size_t)(j + 1) * v.upitch + (i + 1);
            for (int t = 0; t < nf; ++t) acc[t] += v.f32 ? (double)uf32[fo[t] + off] : uf64[fo[t] + off];
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int t = 0; t < 3; ++t) {
        double x = acc[t];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[t][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double x = 0.0;
        for (int w = 0; w < HM_THREADS / 32; ++w) x += red[threadIdx.x][w];
        part[((size_t)threadIdx.x * npz + k) * HM_SPLIT + b] = x;
    }
}

__global__ void k_hmeans3_fin(UView v, const double* __restrict__ part, int npx, int npy, int npz, int lmag,
                              double* __restrict__ means)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;   // t * npz + k
    if (q >= 3 * npz) return;
    const int t = q / npz, k = q % npz;
    const int nf = lmag ? 3 : 2;
    double x = 0.0;
    for (int b = 0; b < HM_SPLIT; ++b) x += part[(size_t)q * HM_SPLIT + b];
    // background rows of the FP32 form: RO 0, TT 1, BY 3
    const double bg = v.f32 ? v.bgd[(t == 0 ? 1 : t == 1 ? 0 : 3) * v.NZ + k + 1] : 0.0;
    means[q] = t < nf ? bg + x / ((double)npx * npy) : 0.0;
}

// network input, channels-last BF16 [k][j][i][16]: u, v, w, TT-<TT>, RO-<RO>, BX, BY-<BY>, BZ
// times in_scale, channels 8..15 zero; grid (x blocks, y, z)
__global__ void k_features(UView v, const double* __restrict__ means, const float* __restrict__ sc, int npx, int npy,
                           int npz, int lmag, __nv_bfloat16* __restrict__ feat)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x, j0 = blockIdx.y, k = blockIdx.z;
    if (i0 >= npx) return;
    const int i = i0 + 1, j = j0 + 1;
    const size_t q = ((size_t)k * npy + j0) * npx + i0;
    const double ro = uget(v, F_RO, i, j, k + 1), ri = 1.0 / ro;
    float f[8];
    f[0] = (float)(uget(v, F_RU, i, j, k + 1) * ri);
    f[1] = (float)(uget(v, F_RV, i, j, k + 1) * ri);
    f[2] = (float)(uget(v, F_RW, i, j, k + 1) * ri);
    f[3] = (float)(uget(v, F_TT, i, j, k + 1) - means[k]);
    f[4] = (float)(ro - means[npz + k]);
    f[5] = lmag ? (float)uget(v, F_BX, i, j, k + 1) : 0.f;
    f[6] = lmag ? (float)(uget(v, F_BY, i, j, k + 1) - means[2 * npz + k]) : 0.f;
    f[7] = lmag ? (float)uget(v, F_BZ, i, j, k + 1) : 0.f;
    __align__(16) __nv_bfloat16 h[16];
#pragma unroll
    for (int c = 0; c < 8; ++c) h[c] = __float2bfloat16_rn(f[c] * sc[c]);
#pragma unroll
    for (int c = 8; c < 16; ++c) h[c] = __float2bfloat16_rn(0.f);
    uint4* o = reinterpret_cast<uint4*>(feat + q * 16);
    o[0] = reinterpret_cast<const uint4*>(h)[0];
    o[1] = reinterpret_cast<const uint4*>(h)[1];
}

// features of the handle's current state with the per-plane means (means: 3 x NPZ)
cudaError_t launch_features(Handle* h, const UView& v, const float* in_scale, double* means, __nv_bfloat16* feat,
                            cudaStream_t st)
{
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    if (!h->hpart) {
        const cudaError_t e = cudaMalloc(&h->hpart, sizeof(double) * 3 * npz * HM_SPLIT);
        if (e != cudaSuccess) return e;
    }
    k_hmeans3<<<dim3((unsigned)npz, HM_SPLIT), HM_THREADS, 0, st>>>(v, npx, npy, h->hpart, npz, h->p.lmag);
    k_hmeans3_fin<<<(unsigned)((3 * npz + 127) / 128), 128, 0, st>>>(v, h->hpart, npx, npy, npz, h->p.lmag, means);
    k_features<<<dim3((unsigned)((npx + 127) / 128), (unsigned)npy, (unsigned)npz), 128, 0, st>>>(
        v, means, in_scale, npx, npy, npz, h->p.lmag, feat);
    return cudaGetLastError();
}

// mean-square error over 12 channels and its gradient (BF16, channels 12..15 zero)
__global__ void __launch_bounds__(256) k_closure_loss(const float* __restrict__ pred, const float* __restrict__ tgt,
                                                      size_t nvox, __nv_bfloat16* __restrict__ dy,
                                                      double* __restrict__ loss)
{
    __shared__ double red[256];
    const double nrm = 1.0 / ((double)nvox * 12.0);
    double acc = 0.0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nvox; q += (size_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < 16; ++c) {
            float g = 0.f;
            if (c < 12) {
                const double d = (double)pred[q * 16 + c] - (double)tgt[q * 12 + c];
                acc += d * d * nrm;
                g = (float)(2.0 * d * nrm);
            }
            if (dy) dy[q * 16 + c] = __float2bfloat16_rn(g);
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

// Adam on FP32 master parameters; optional BF16 copy
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       __nv_bfloat16* __restrict__ pb)
{
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float pq = p[q] - lr * (mq / bc1) / (sqrtf(vq / bc2) + eps);
        p[q] = pq;
        if (pb) pb[q] = __float2bfloat16_rn(pq);
    }
}

// Closure tendencies from the network output (normalised targets x out_scale):
// RU_i -= d_j tau_ij, TT -= (1/RO) d_j q_j, B += curl eps, centred differences
// with the grid's metric factors (HX*DXXDX ...), zero on the wall planes.
// Output field f (RU,RV,RW,TT,BX,BY,BZ) at out[f*fstride + k*kstride + j*jstride + i].
// flag[0] is set when an output is not finite or the stress exceeds trip x RO*TT.
// Closure tendencies marching in z: a CTA owns a TTX x TTY column tile and a
// chunk of TZC planes, and keeps four planes of the tile with its one-voxel
// x/y halo (channels 0..11 of the prediction rows) in shared memory, so each
// prediction row is read from L2 about once instead of once per neighbour.
// Plane k+2 is fetched into registers while plane k is formed.
constexpr int TTX = 32, TTY = 8, TZC = 8;
constexpr int TPX = TTX + 2, TPY = TTY + 2, TPV = TPX * TPY;   // voxels of a plane tile with halo
constexpr size_t TEND_SMEM = (size_t)4 * TPV * 12 * sizeof(float);
__global__ void __launch_bounds__(TTX * TTY) k_tendency(UView v, const float* __restrict__ pred,
                                                       const float* __restrict__ osc, const double* __restrict__ fax,
                                                       const double* __restrict__ fay, const double* __restrict__ faz,
                                                       const float* __restrict__ bias, int npx, int npy, int npz,
                                                       float trip, float* __restrict__ out, size_t fstride,
                                                       size_t kstride, size_t jstride, int* flag)
{
    extern __shared__ __align__(16) float tsm[];   // [slot 0..3][TPV][12], plane p in slot p & 3
    const int tid = threadIdx.x, tx = tid % TTX, ty = tid / TTX;
    const int x0 = blockIdx.x * TTX, y0 = blockIdx.y * TTY;
    const int kc0 = blockIdx.z * TZC, kc1 = kc0 + TZC < npz ? kc0 + TZC : npz;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool active = gi < npx && gj < npy;
    constexpr int NL = (TPV * 3 + TTX * TTY - 1) / (TTX * TTY);   // 16-byte loads per thread and plane
    // plane p (clamped to the grid: the wall planes have no tendency): fetch
    // into registers, then store into its slot
    float4 t[NL];
    auto fetch_plane = [&](int p) {
        p = p < 0 ? 0 : (p >= npz ? npz - 1 : p);
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int e = tid + u * TTX * TTY;
            if (e < TPV * 3) {
                const int vox = e / 3, h = e % 3;
                int px = x0 - 1 + vox % TPX, py = y0 - 1 + vox / TPX;
                px %= npx;
                px = px < 0 ? px + npx : px;
                py %= npy;
                py = py < 0 ? py + npy : py;
                t[u] = __ldg(reinterpret_cast<const float4*>(pred + (((size_t)p * npy + py) * npx + px) * 16) + h);
            }
        }
    };
    auto store_plane = [&](int p) {
        const int slot = (p + 4) & 3;
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int e = tid + u * TTX * TTY;
            if (e < TPV * 3) *reinterpret_cast<float4*>(tsm + ((size_t)slot * TPV + e / 3) * 12 + 4 * (e % 3)) = t[u];
        }
    };
    float s[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) s[c] = osc[c];
    const float ax = active ? (float)fax[gi + 1] : 0.f, ay = active ? (float)fay[gj + 1] : 0.f;
    const int lc = (ty + 1) * TPX + (tx + 1);   // own voxel in a plane tile
    for (int p = kc0 - 1; p <= kc0 + 1; ++p) {
        fetch_plane(p);
        store_plane(p);
    }
    for (int k = kc0; k < kc1; ++k) {
        __syncthreads();                     // planes k-1, k, k+1 are in place
        if (k + 2 <= kc1) fetch_plane(k + 2);  // in flight while plane k is formed
        if (active) {
            const float* Pc = tsm + (size_t)(k & 3) * TPV * 12;
            const float* Pp = tsm + (size_t)((k + 1) & 3) * TPV * 12;
            const float* Pm = tsm + (size_t)((k + 3) & 3) * TPV * 12;
            const float* cv = Pc + lc * 12;
            float* o = out + (size_t)k * kstride + (size_t)gj * jstride + gi;
            bool bad = false;
#pragma unroll
            for (int c = 0; c < 12; ++c) bad |= !isfinite(cv[c]);
            const double ro = uget(v, F_RO, gi + 1, gj + 1, k + 1), tt = uget(v, F_TT, gi + 1, gj + 1, k + 1);
            const double tr =
                fabs((double)(cv[0] * s[0])) + fabs((double)(cv[1] * s[1])) + fabs((double)(cv[2] * s[2]));
            if (bad || !(tr <= (double)trip * ro * tt)) atomicOr(flag, 1);
            if (k == 0 || k == npz - 1) {
#pragma unroll
                for (int f = 0; f < 7; ++f) o[f * fstride] = 0.f;
            } else {
                const float az = (float)faz[k + 1];
                const float *xp = cv + 12, *xm = cv - 12, *yp = cv + TPX * 12, *ym = cv - TPX * 12;
                const float *zp = Pp + lc * 12, *zm = Pm + lc * 12;
                auto dx = [&](int c) { return (xp[c] - xm[c]) * s[c] * ax; };
                auto dy = [&](int c) { return (yp[c] - ym[c]) * s[c] * ay; };
                auto dz = [&](int c) { return (zp[c] - zm[c]) * s[c] * az; };
                float bz[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (bias) {
#pragma unroll
                    for (int f = 0; f < 7; ++f) bz[f] = bias[(size_t)f * npz + k];
                }
                o[0 * fstride] = -(dx(0) + dy(3) + dz(4)) + bz[0];
                o[1 * fstride] = -(dx(3) + dy(1) + dz(5)) + bz[1];
                o[2 * fstride] = -(dx(4) + dy(5) + dz(2)) + bz[2];
                o[3 * fstride] = -(dx(6) + dy(7) + dz(8)) / (float)ro + bz[3];
                o[4 * fstride] = dy(11) - dz(10) + bz[4];
                o[5 * fstride] = dz(9) - dx(11) + bz[5];
                o[6 * fstride] = dx(10) - dy(9) + bz[6];
            }
        }
        if (k + 2 <= kc1) store_plane(k + 2);   // slot of plane k-2, read by no thread since the last barrier
    }
}

// The per-plane bias alone, broadcast into the Z layout of the closure's
// tendencies (zero on the wall planes, as k_tendency writes them).
__global__ void __launch_bounds__(256) k_bias_tendency(const float* __restrict__ bias, int npx, int npy, int npz,
                                                       float* __restrict__ out, size_t fstride, size_t kstride,
                                                       size_t jstride)
{
    const size_t n = (size_t)npx * npy * npz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % npx), j = (int)((c / npx) % npy), k = (int)(c / ((size_t)npx * npy));
        float* o = out + (size_t)k * kstride + (size_t)j * jstride + i;
        const bool wall = k == 0 || k == npz - 1;
#pragma unroll
        for (int f = 0; f < 7; ++f) o[f * fstride] = wall ? 0.f : bias[(size_t)f * npz + k];
    }
}

cudaError_t launch_tendency(UView v, const float* pred, const float* osc, const Metrics& m, const float* bias, int npx,
                            int npy, int npz, float trip, float* out, size_t fstride, size_t kstride, size_t jstride,
                            int* flag, cudaStream_t st)
{
    static std::atomic<unsigned long long> attr{0};
    const cudaError_t ae = smem_attr_once(attr, reinterpret_cast<const void*>(k_tendency), TEND_SMEM);
    if (ae != cudaSuccess) return ae;
    const dim3 grid((unsigned)((npx + TTX - 1) / TTX), (unsigned)((npy + TTY - 1) / TTY),
                    (unsigned)((npz + TZC - 1) / TZC));
    k_tendency<<<grid, TTX * TTY, TEND_SMEM, st>>>(v, pred, osc, m.fax, m.fay, m.faz, bias, npx, npy, npz, trip, out,
                                                  fstride, kstride, jstride, flag);
    return cudaGetLastError();
}

// Adjoint of k_tendency's linear map pred -> tendencies: for output g
// [7][nvox] (the loss gradient of each tendency) writes d loss / d pred as
// BF16 [nvox][16] (channels 12..15 zero), the last layer's output gradient.
// A term s * (P[n+1] - P[n-1]) * a[n] of tendency f at cell n hands
// s * (a[m-1] g[m-1] - a[m+1] g[m+1]) to P[m]; TT's terms carry 1/RO of
// cell n; the first and last z planes have no tendency.
__global__ void k_tendency_adj(UView v, const float* __restrict__ g, const float* __restrict__ osc,
                               const double* __restrict__ fax, const double* __restrict__ fay,
                               const double* __restrict__ faz, int npx, int npy, int npz, size_t fstride,
                               __nv_bfloat16* __restrict__ dpred)
{
    // (field, direction, sign) of each output channel, as k_tendency uses them
    constexpr int NT[12] = {1, 1, 1, 2, 2, 2, 1, 1, 1, 2, 2, 2};
    constexpr int TF[12][2] = {{0, 0}, {1, 0}, {2, 0}, {0, 1}, {0, 2}, {1, 2},
                               {3, 0}, {3, 0}, {3, 0}, {5, 6}, {6, 4}, {4, 5}};
    constexpr int TD[12][2] = {{0, 0}, {1, 0}, {2, 0}, {1, 0}, {2, 0}, {2, 1},
                               {0, 0}, {1, 0}, {2, 0}, {2, 1}, {0, 2}, {1, 0}};
    constexpr float TS[12][2] = {{-1, 0}, {-1, 0}, {-1, 0}, {-1, -1}, {-1, -1}, {-1, -1},
                                 {-1, 0}, {-1, 0}, {-1, 0}, {1, -1}, {1, -1}, {1, -1}};
    const size_t n = (size_t)npx * npy * npz;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % npx), j = (int)((q / npx) % npy), k = (int)(q / ((size_t)npx * npy));
        // weighted gradient of field f at the neighbour one cell along d (side -1 or +1)
        auto H = [&](int f, int d, int side) -> double {
            int ii = i, jj = j, kk = k;
            double a;
            if (d == 0) {
                ii = i + side;
                ii = ii < 0 ? npx - 1 : (ii == npx ? 0 : ii);
                a = fax[ii + 1];
            } else if (d == 1) {
                jj = j + side;
                jj = jj < 0 ? npy - 1 : (jj == npy ? 0 : jj);
                a = fay[jj + 1];
            } else {
                kk = k + side;
                if (kk < 1 || kk > npz - 2) return 0.0;
                a = faz[kk + 1];
            }
            if (d < 2 && (kk < 1 || kk > npz - 2)) return 0.0;
            double h = (double)g[f * fstride + ((size_t)kk * npy + jj) * npx + ii] * a;
            if (f == 3) h /= uget(v, F_RO, ii + 1, jj + 1, kk + 1);
            return h;
        };
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            double acc = 0.0;
            for (int t = 0; t < NT[c]; ++t)
                acc += TS[c][t] * (H(TF[c][t], TD[c][t], -1) - H(TF[c][t], TD[c][t], 1));
            o[c] = __float2bfloat16_rn((float)(acc * osc[c]));
        }
#pragma unroll
        for (int c = 12; c < 16; ++c) o[c] = __float2bfloat16_rn(0.f);
        uint4* dst = reinterpret_cast<uint4*>(dpred + q * 16);
        dst[0] = reinterpret_cast<const uint4*>(o)[0];
        dst[1] = reinterpret_cast<const uint4*>(o)[1];
    }
}

// Weighted mean-square loss of the 7 tendencies against a target and its
// gradient: loss += sum_f w_f sum_q (t - r)^2 / (7 nvox), g = d loss / d t.
__global__ void __launch_bounds__(256) k_tendency_loss(const float* __restrict__ t, const float* __restrict__ r,
                                                       const float* __restrict__ w, size_t nvox,
                                                       float* __restrict__ g, double* __restrict__ loss)
{
    __shared__ double red[256];
    const double nrm = 1.0 / ((double)nvox * 7.0);
    double acc = 0.0;
    const size_t n = nvox * 7;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const double wf = w[q / nvox] * nrm;
        const double d = (double)t[q] - (double)r[q];
        acc += wf * d * d;
        g[q] = (float)(2.0 * wf * d);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s2 = 128; s2 > 0; s2 >>= 1) {
        if ((int)threadIdx.x < s2) red[threadIdx.x] += red[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

__global__ void k_trip_count(int* flag)
{
    flag[1] += flag[0] ? 1 : 0;
    flag[2] += 1;
}


__device__ void finalize_one(Control* ctl, Accum* acc, double sf, double dtmin, int lmag, int advance,
                             unsigned long long w4key)
{
    if (advance) {
        if (ctl->stop) return;
        ctl->timc = ctl->timc + ctl->dt;
        ctl->timt = ctl->timi + ctl->timc;
        ctl->nit += 1;
        ctl->last_dt = ctl->dt;
        ctl->last_umach = ctl->umach;
        if (!(ctl->dt >= dtmin)) {
            ctl->stop = 1;
            ctl->status = isfinite(ctl->dt) ? MHD3D_ERR_DT_SMALL : MHD3D_ERR_NONFINITE;
        }
    }
    double w = of_key(acc->wmin[0]);
    const double w2 = of_key(acc->wmin[1]), w3 = of_key(acc->wmin[2]), w4 = of_key(acc->wmin[3]);
    w = w2 < w ? w2 : w;
    w = w3 < w ? w3 : w;
    if (lmag) w = w4 < w ? w4 : w;
    ctl->dt = sf * w;
    ctl->umach = sqrt(of_key(acc->umax));
    if (acc->bad && !ctl->stop) {
        ctl->stop = 1;
        ctl->status = MHD3D_ERR_NONFINITE;
    }
    for (int i = 0; i < 3; ++i) acc->wmin[i] = ~0ull;
    acc->wmin[3] = w4key;
    acc->umax = 0ull;
    acc->bad = 0u;
}

__global__ void k_finalize(Control* ctl, Accum* acc, double sf, double dtmin, int lmag, int advance,
                           unsigned long long w4key)
{
    finalize_one(ctl, acc, sf, dtmin, lmag, advance, w4key);
}

// end of a step of every member of an ensemble (one thread per member)
struct FinArgs {
    Control* ctl;
    Accum* acc;
    double sf, dtmin;
    unsigned long long w4key;
    int lmag, pad;
};
__global__ void k_finalize_multi(const FinArgs* __restrict__ f, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) finalize_one(f[i].ctl, f[i].acc, f[i].sf, f[i].dtmin, f[i].lmag, 1, f[i].w4key);
}

unsigned grid_for(size_t n)
{
    size_t b = (n + 255) / 256;
    return (unsigned)(b > 148 * 16 ? 148 * 16 : (b ? b : 1));
}

StageArgs make_args(Handle* h)
{
    StageArgs a{};
    a.map_u = h->map_u[h->cur];
    a.map_z = h->map_z;
    a.u_in = h->ubuf[h->cur];
    a.u_out = h->ubuf[h->cur ^ 1];
    a.z = h->z;
    a.f_out = h->fout;
    a.ctl = h->ctl;
    a.acc = h->acc;
    a.m = h->m;
    a.s = h->s;
    a.uf = h->uf;
    a.uz = h->uz;
    a.zf = h->zf;
    a.zz = h->zz;
    a.upitch = h->upitch;
    a.zpitch = h->zpitch;
    a.ntx = h->ntx;
    a.zlen = h->zlen;
    a.nchunks = h->nchunks;
    a.wait_first = h->wait_first;
    return a;
}

StageArgs32 make_args32(Handle* h)
{
    StageArgs32 a{};
    a.map_u = h->map_u[h->cur];
    a.map_z = h->map_z;
    a.u_in = reinterpret_cast<const float*>(h->ubuf[h->cur]);
    a.u_out = reinterpret_cast<float*>(h->ubuf[h->cur ^ 1]);
    a.z = reinterpret_cast<float*>(h->z);
    a.f_out = reinterpret_cast<float*>(h->fout);
    a.ctl = h->ctl;
    a.acc = h->acc;
    a.m = h->m;
    a.s = h->s;
    const size_t NZ = (size_t)h->p.npz + 2;
    a.rob = h->bg32;
    a.ttb = h->bg32 + NZ;
    a.bgd = h->bgd;
    a.pb = h->pb;
    a.cx = h->cxy;
    a.cy = h->cxy + (h->p.npx + 2);
    a.s32 = h->s32;
    a.fcl = h->clo ? h->cfcl : h->cbtend;
    a.fcl_flag = h->clo ? h->cflag : (h->cbtend ? reinterpret_cast<const int*>(h->cbtend + 7 * h->zf) : nullptr);
    a.top_lin = h->top_lin;
    a.top_tb = h->top_tb;
    a.t_top_fix = h->t_top_fix;
    a.t_top_fix4 = h->t_top_fix4;
    a.t_top_flux = h->t_top_flux;
    a.t_bot = h->t_bot;
    a.uf = h->uf;
    a.uz = h->uz;
    a.zf = h->zf;
    a.zz = h->zz;
    a.upitch = h->upitch;
    a.zpitch = h->zpitch;
    a.ntx = h->ntx;
    a.zlen = h->zlen;
    a.nchunks = h->nchunks;
    return a;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// 4-D tiled TMA map (x, y, z, field) of a double or float array, no swizzle, zero fill
int make_map(CUtensorMap* map, void* base, const cuuint64_t dims[4], const cuuint32_t box[4], bool f32 = false)
{
    static EncodeTiledFn enc = nullptr;
    if (!enc) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return MHD3D_ERR_CUDA;
        enc = reinterpret_cast<EncodeTiledFn>(fn);
    }
    const cuuint64_t es = f32 ? 4 : 8;
    const cuuint64_t strides[3] = {dims[0] * es, dims[0] * dims[1] * es, dims[0] * dims[1] * dims[2] * es};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims,
                     strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        std::fprintf(stderr, "mhd3d: cuTensorMapEncodeTiled failed (%d)\n", (int)r);
        return MHD3D_ERR_CUDA;
    }
    return MHD3D_OK;
}

cudaError_t launch_stage(Handle* h, int stage, const StageArgs& a)
{
    return h->p.mode == MHD3D_MODE_FAST ? fast::launch_stage(stage, a, h->st) : exact::launch_stage(stage, a, h->st);
}

cudaError_t launch_cfl(Handle* h, const StageArgs& a)
{
    if (h->f32) return f32::launch_cfl(make_args32(h), h->st);
    return h->p.mode == MHD3D_MODE_FAST ? fast::launch_cfl(a, h->st) : exact::launch_cfl(a, h->st);
}

int validate(const mhd3d_params* p)
{
    if (!p) return MHD3D_ERR_ARG;
    if (p->npx < 2 || p->npy < 2 || p->npz < 4) return MHD3D_ERR_ARG;
    if (p->izcon != 0 && p->izcon != 1) return MHD3D_ERR_ARG;
    if (p->itcon < 0 || p->itcon > 4 || p->itcon == 2) return MHD3D_ERR_ARG;
    if (p->mode != MHD3D_MODE_EXACT && p->mode != MHD3D_MODE_FAST && p->mode != MHD3D_MODE_FP32) return MHD3D_ERR_ARG;
    if ((size_t)(p->npx + 2) * (p->npy + 2) * (p->npz + 2) > ((size_t)1 << 40)) return MHD3D_ERR_ARG;
    return MHD3D_OK;
}

int destroy(Handle* h)
{
    if (!h) return MHD3D_OK;
    if (h->dev >= 0) cudaSetDevice(h->dev);
    cudaFree(h->ubuf[0]);
    cudaFree(h->ubuf[1]);
    cudaFree(h->z);
    cudaFree(h->stage);
    cudaFree(h->stage2);
    for (int i = 0; i < 2; ++i) {
        if (h->ev_copy[i]) cudaEventDestroy(h->ev_copy[i]);
        if (h->ev_kern[i]) cudaEventDestroy(h->ev_kern[i]);
    }
    if (h->cst) cudaStreamDestroy(h->cst);
    cudaFree(h->fout);
    cudaFree(h->hpart);
    cudaFree(h->met);
    cudaFree(h->metf);
    cudaFree(h->bgd);
    cudaFree(h->bg32);
    cudaFree(h->pb);
    cudaFree(h->cxy);
    cudaFree(h->cbuf);
    cudaFree(h->cbias);
    cudaFree(h->cbtend);
    cudaFree(h->ctl);
    cudaFree(h->acc);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
    return MHD3D_OK;
}

int create(const mhd3d_params* p, const double* const arrs[14], void** out)
{
    int st = validate(p);
    if (st) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MHD3D_ERR_NO_DEVICE;
    for (int i = 0; i < 14; ++i)
        if (!arrs[i]) return MHD3D_ERR_ARG;
    Handle* h = new (std::nothrow) Handle();
    if (!h) return MHD3D_ERR_NOMEM;
    *out = h;   // released by the caller if anything below fails
    h->p = *p;
    CK(cudaGetDevice(&h->dev));
    CK(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
    h->st = h->own;
    const int npx = p->npx, npy = p->npy, npz = p->npz;
    const int NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    h->nf = p->lmag ? 8 : 5;
    h->f32 = p->mode == MHD3D_MODE_FP32;
    // U: the Fortran index space (halos, ghost planes), rows padded to 16
    // bytes and to at least one TMA box; Z: interior cells only
    const int ealign = h->f32 ? 4 : 2;                 // elements per 16 bytes
    const int bw = h->f32 ? BW32 : BW, bh = h->f32 ? BH32 : BH, ty = h->f32 ? TY32 : TY;
    h->upitch = (NX + ealign - 1) / ealign * ealign;
    if (h->upitch < bw) h->upitch = bw;
    h->urows = NY < bh ? bh : NY;
    h->uz = (size_t)h->urows * h->upitch;
    h->uf = (size_t)NZ * h->uz;
    h->zpitch = (npx + ealign - 1) / ealign * ealign;
    if (h->zpitch < TX) h->zpitch = TX;
    h->zrows = npy < ty ? ty : npy;
    h->zz = (size_t)h->zrows * h->zpitch;
    h->zf = (size_t)npz * h->zz;
    const size_t esize = h->f32 ? sizeof(float) : sizeof(double);
    const size_t ubytes = esize * h->nf * h->uf;
    const size_t zbytes = esize * h->nf * h->zf;
    CK(cudaMalloc(&h->ubuf[0], ubytes));
    CK(cudaMalloc(&h->ubuf[1], ubytes));
    CK(cudaMalloc(&h->z, zbytes));
    CK(cudaMemset(h->ubuf[0], 0, ubytes));
    CK(cudaMemset(h->ubuf[1], 0, ubytes));
    CK(cudaMemset(h->z, 0, zbytes));
    {
        const cuuint64_t du[4] = {(cuuint64_t)h->upitch, (cuuint64_t)h->urows, (cuuint64_t)NZ, (cuuint64_t)h->nf};
        const cuuint32_t bu[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, (cuuint32_t)h->nf};
        for (int b = 0; b < 2; ++b) {
            int st2 = make_map(&h->map_u[b], h->ubuf[b], du, bu, h->f32);
            if (st2) return st2;
        }
        const cuuint64_t dz[4] = {(cuuint64_t)h->zpitch, (cuuint64_t)h->zrows, (cuuint64_t)npz, (cuuint64_t)h->nf};
        const cuuint32_t bz[4] = {TX, (cuuint32_t)ty, 1, (cuuint32_t)h->nf};
        int st3 = make_map(&h->map_z, h->z, dz, bz, h->f32);
        if (st3) return st3;
    }
    if (h->f32) {
        CK(cudaMalloc(&h->bgd, sizeof(double) * 5 * NZ));
        CK(cudaMemset(h->bgd, 0, sizeof(double) * 5 * NZ));
        CK(cudaMalloc(&h->bg32, sizeof(float) * 2 * NZ));
        CK(cudaMemset(h->bg32, 0, sizeof(float) * 2 * NZ));
        CK(cudaMalloc(&h->pb, sizeof(PlaneBg) * npz));
        CK(cudaMemset(h->pb, 0, sizeof(PlaneBg) * npz));
    }
    CK(cudaMalloc(&h->stage, sizeof(double) * (size_t)NX * NY * NZ));
    CK(cudaMalloc(&h->stage2, sizeof(double) * (size_t)NX * NY * NZ));
    CK(cudaStreamCreateWithFlags(&h->cst, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        CK(cudaEventCreateWithFlags(&h->ev_copy[i], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->ev_kern[i], cudaEventDisableTiming));
    }
    CK(cudaMalloc(&h->ctl, sizeof(Control)));
    CK(cudaMalloc(&h->acc, sizeof(Accum)));

    // 1-D arrays: 11 metric/kappa arrays, the two plume factors, 9 fast-mode
    // stencil factors, 4 fast-mode CFL factors
    constexpr int NMET = 26;
    const int lens[NMET] = {NX, NX, NX, NY, NY, NY, NZ, NZ, NZ, NZ, NZ, NX, NY,
                            NX, NX, NX, NY, NY, NY, NZ, NZ, NZ, NX, NY, NZ, NZ};
    size_t tot = 0;
    for (int i = 0; i < NMET; ++i) tot += lens[i];
    double* hm = (double*)std::malloc(sizeof(double) * tot);
    const double* exx = arrs[0];
    const double* wyy = arrs[4];
    const double* src[11] = {arrs[1], arrs[2], arrs[3], arrs[5], arrs[6], arrs[7], arrs[9], arrs[10], arrs[11],
                             arrs[12], arrs[13]};
    size_t off = 0;
    size_t offs[NMET];
    for (int i = 0; i < 11; ++i) {
        offs[i] = off;
        std::memcpy(hm + off, src[i], sizeof(double) * lens[i]);
        off += lens[i];
    }
    // plume factors EXP(CLN*(EXX(I)-XP)**2), EXP(CLN*(WYY(J)-YP)**2) with
    // CLN=-4.0E00*LOG(2.0E00)/HH/HH (3dmhdsub.f:2818, 2803-2804)
    const int plume = (p->tp != 0.0 && (p->itcon == 0 || p->itcon == 1)) ? 1 : 0;
    const double cln = plume ? (double)(-(4.0f * std::log(2.0f))) / p->hh / p->hh : 0.0;
    offs[11] = off;
    for (int i = 0; i < NX; ++i) {
        const double d = exx[i] - p->xp;
        hm[off + i] = plume ? std::exp(cln * (d * d)) : 0.0;
    }
    off += NX;
    offs[12] = off;
    for (int j = 0; j < NY; ++j) {
        const double d = wyy[j] - p->yp;
        hm[off + j] = plume ? std::exp(cln * (d * d)) : 0.0;
    }
    off += NY;
    // fast-mode metric factors (products the reference forms per use)
    {
        const double* d1[3] = {src[0], src[3], src[6]};   // DXXDX, DYYDY, DZZDZ
        const double* d2[3] = {src[1], src[4], src[7]};   // D2XXDX2, D2YYDY2, D2ZZDZ2
        const double hh[3] = {p->hx, p->hy, p->hz}, h2[3] = {p->h2x, p->h2y, p->h2z};
        const int len[3] = {NX, NY, NZ};
        for (int d = 0; d < 3; ++d) {
            offs[13 + 3 * d] = off;
            for (int i = 0; i < len[d]; ++i) hm[off + i] = hh[d] * d1[d][i];
            off += len[d];
            offs[14 + 3 * d] = off;
            for (int i = 0; i < len[d]; ++i) hm[off + i] = hh[d] * d2[d][i];
            off += len[d];
            offs[15 + 3 * d] = off;
            for (int i = 0; i < len[d]; ++i) hm[off + i] = h2[d] * d1[d][i] * d1[d][i];
            off += len[d];
        }
        // CFL: reciprocals of DDX, DDY, DDZ and W2's factor 0.5*REPR*CV/RKAPA(K)
        const double* dd[3] = {src[2], src[5], src[8]};
        for (int d = 0; d < 3; ++d) {
            offs[22 + d] = off;
            for (int i = 0; i < len[d]; ++i) hm[off + i] = 1.0 / dd[d][i];
            off += len[d];
        }
        offs[25] = off;
        for (int k = 0; k < NZ; ++k) hm[off + k] = 0.5 * p->repr * p->cv / src[9][k];
        off += NZ;
    }
    // W4=0.5*DD*DD*RM (3dmhdsub.f:851) depends on the grid alone and is monotone
    // in DD, so its minimum over the cells is that of the smallest or largest
    // DD=MIN(DDX(I),DDY(J),DDZ(K)), I=2..NX-1, J=2..NY-1, K=2..NZ-1
    if (p->lmag) {
        double lo[3], hi[3];
        const double* dd[3] = {src[2], src[5], src[8]};
        const int n[3] = {npx, npy, npz};
        for (int d = 0; d < 3; ++d) {
            lo[d] = hi[d] = dd[d][1];
            for (int i = 2; i <= n[d]; ++i) {
                lo[d] = dd[d][i] < lo[d] ? dd[d][i] : lo[d];
                hi[d] = dd[d][i] > hi[d] ? dd[d][i] : hi[d];
            }
        }
        const double dlo = std::min(std::min(lo[0], lo[1]), lo[2]);
        const double dhi = std::min(std::min(hi[0], hi[1]), hi[2]);
        const double f_lo = 0.5 * dlo * dlo * p->rm, f_hi = 0.5 * dhi * dhi * p->rm;
        h->w4key = std::min(key_of(f_lo), key_of(f_hi));
    }
    h->faz_h.assign(hm + offs[19], hm + offs[19] + NZ);
    h->fbz_h.assign(hm + offs[20], hm + offs[20] + NZ);
    h->fcz_h.assign(hm + offs[21], hm + offs[21] + NZ);
    h->rka_h.assign(src[9], src[9] + NZ);
    h->dka_h.assign(src[10], src[10] + NZ);
    h->ddz_h.assign(src[8], src[8] + NZ);
    if (h->f32) {
        // column constants of the FP32 kernel
        std::vector<ColC> cc((size_t)NX + NY);
        for (int i = 0; i < NX; ++i) {
            ColC& c = cc[i];
            c.a = (float)hm[offs[13] + i];
            c.b = (float)hm[offs[14] + i];
            c.c = (float)hm[offs[15] + i];
            c.rdd = (float)(1.0 / src[2][i]);
            c.dd = (float)src[2][i];
        }
        for (int j = 0; j < NY; ++j) {
            ColC& c = cc[(size_t)NX + j];
            c.a = (float)hm[offs[16] + j];
            c.b = (float)hm[offs[17] + j];
            c.c = (float)hm[offs[18] + j];
            c.rdd = (float)(1.0 / src[5][j]);
            c.dd = (float)src[5][j];
        }
        CK(cudaMalloc(&h->cxy, sizeof(ColC) * cc.size()));
        CK(cudaMemcpy(h->cxy, cc.data(), sizeof(ColC) * cc.size(), cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&h->met, sizeof(double) * tot));
    CK(cudaMemcpy(h->met, hm, sizeof(double) * tot, cudaMemcpyHostToDevice));
    h->m.dxxdx = h->met + offs[0];
    h->m.d2xxdx2 = h->met + offs[1];
    h->m.ddx = h->met + offs[2];
    h->m.dyydy = h->met + offs[3];
    h->m.d2yydy2 = h->met + offs[4];
    h->m.ddy = h->met + offs[5];
    h->m.dzzdz = h->met + offs[6];
    h->m.d2zzdz2 = h->met + offs[7];
    h->m.ddz = h->met + offs[8];
    h->m.rkapa = h->met + offs[9];
    h->m.dkapa = h->met + offs[10];
    h->m.plume_gx = h->met + offs[11];
    h->m.plume_gy = h->met + offs[12];
    h->m.fax = h->met + offs[13];
    h->m.fbx = h->met + offs[14];
    h->m.fcx = h->met + offs[15];
    h->m.fay = h->met + offs[16];
    h->m.fby = h->met + offs[17];
    h->m.fcy = h->met + offs[18];
    h->m.faz = h->met + offs[19];
    h->m.fbz = h->met + offs[20];
    h->m.fcz = h->met + offs[21];
    h->m.rddx = h->met + offs[22];
    h->m.rddy = h->met + offs[23];
    h->m.rddz = h->met + offs[24];
    h->m.fw2z = h->met + offs[25];
    {
        // FP32 screening copies: 1/DD and DD per axis, MIN(0.375*RE, 0.5*REPR*CV/RKAPA(K))
        const size_t nf = 2 * ((size_t)NX + NY + NZ) + NZ;
        std::vector<float> fm(nf);
        size_t o = 0;
        const double* dd[3] = {src[2], src[5], src[8]};
        const int len[3] = {NX, NY, NZ};
        size_t fo[7];
        for (int d = 0; d < 3; ++d) {
            fo[d] = o;
            for (int i = 0; i < len[d]; ++i) fm[o + i] = (float)(1.0 / dd[d][i]);
            o += len[d];
        }
        for (int d = 0; d < 3; ++d) {
            fo[3 + d] = o;
            for (int i = 0; i < len[d]; ++i) fm[o + i] = (float)dd[d][i];
            o += len[d];
        }
        fo[6] = o;
        for (int k = 0; k < NZ; ++k) fm[o + k] = (float)std::min(0.375 * p->re, hm[offs[25] + k]);
        CK(cudaMalloc(&h->metf, sizeof(float) * nf));
        CK(cudaMemcpy(h->metf, fm.data(), sizeof(float) * nf, cudaMemcpyHostToDevice));
        h->m.rddx_f = h->metf + fo[0];
        h->m.rddy_f = h->metf + fo[1];
        h->m.rddz_f = h->metf + fo[2];
        h->m.ddx_f = h->metf + fo[3];
        h->m.ddy_f = h->metf + fo[4];
        h->m.ddz_f = h->metf + fo[5];
        h->m.wfz_f = h->metf + fo[6];
    }

    // scalars (3dmhd.f:105-240 values; FLUXES/BCON per-call products)
    Scalars& s = h->s;
    s.c13 = p->c13; s.c23 = p->c23; s.c43 = p->c43;
    s.hx = p->hx; s.h2x = p->h2x; s.hy = p->hy; s.h2y = p->h2y; s.hz = p->hz; s.h2z = p->h2z;
    s.gam1 = p->gam1; s.gam2 = p->gam2; s.gam3 = p->gam3; s.zeta1 = p->zeta1; s.zeta2 = p->zeta2;
    s.cv = p->cv; s.ocv = p->ocv; s.ore = p->ore; s.re = p->re; s.repr = p->repr;
    s.theta = p->theta; s.grav = p->grav; s.gamma = p->gamma; s.ogamma = 1.0 / p->gamma; s.sf = p->sf;
    s.rm = p->rm; s.omx = p->omx; s.omz = p->omz; s.orm = p->orm; s.obeta = p->obeta;
    s.tmp_cond = p->ocv / p->repr;
    s.tmp_a = p->ocv * p->ore;
    s.tmp_b = p->c43 * p->ocv * p->ore;
    s.tmp_13 = p->c13 * p->ore;
    s.tmp_m = p->obeta * p->orm * p->ocv;
    s.cw3 = 0.375 * p->re;
    s.ogamma_f = (float)(1.0 / p->gamma);
    s.gamma_f = (float)p->gamma;
    s.obeta_f = (float)p->obeta;
    {
        Scalars32& f = h->s32;
        f.grav = (float)p->grav; f.ore = (float)p->ore; f.c13 = (float)p->c13; f.c43 = (float)p->c43;
        f.tmp13 = (float)s.tmp_13; f.tmpa = (float)s.tmp_a; f.tmpb = (float)s.tmp_b; f.tmpc = (float)s.tmp_cond;
        f.ocv = (float)p->ocv; f.omx = (float)p->omx; f.omz = (float)p->omz; f.orm = (float)p->orm;
        f.obeta = (float)p->obeta; f.tmpm = (float)s.tmp_m; f.ogamma = (float)(1.0 / p->gamma);
        f.gamma = (float)p->gamma; f.cw3 = (float)s.cw3;
    }
    s.tb = p->tb; s.tp = p->tp; s.tc = p->tc; s.hh = p->hh;
    const double dzs = (double)(1.0f / (float)(npz - 1));
    s.top_dz = dzs / src[6][1];                         // DZ=1.0E00/FLOAT(NPZ-1)/DZZDZ(2)
    s.top_flux = p->c23 * s.top_dz * p->theta;
    const double bot_dz = dzs / src[6][NZ - 2];         // DZZDZ(NZ-1)
    s.bot_flux = p->c23 * bot_dz * p->theta / src[9][NZ - 2];
    s.dtmin = p->dtmin;
    s.timi = p->timi;
    s.npx = npx; s.npy = npy; s.npz = npz; s.pitch = h->upitch;
    s.lmag = p->lmag; s.lrot = p->lrot; s.izcon = p->izcon; s.itcon = p->itcon; s.ibcon = p->ibcon;
    s.plume = plume;
    std::free(hm);

    // work decomposition: TX x TY tiles, z chunks of <= MHD3D_ZCHUNK planes;
    // small grids take shorter chunks (>= 4 planes) so that the launch still
    // fills about two waves of the SMs
    h->ntx = (npx + TX - 1) / TX;
    const int tyw = h->f32 ? TY32 : TY;
    const long ntiles = (long)h->ntx * ((npy + tyw - 1) / tyw);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->dev);
    const long want = 2L * sms * (h->f32 ? MHD3D_MINB32 : MHD3D_MINB);   // CTAs resident per SM
    int nch = (npz + MHD3D_ZCHUNK - 1) / MHD3D_ZCHUNK;
    const int fill = (int)std::min<long>((want + ntiles - 1) / ntiles, npz / 4);
    if (fill > nch) nch = fill;
    while (nch > 1 && npz / nch < 3) --nch;
    h->nchunks = nch;
    h->zlen = npz / nch;

    Control c0{};
    c0.timc = p->timc;
    c0.timi = p->timi;
    c0.timt = 0.0;
    CK(cudaMemcpy(h->ctl, &c0, sizeof(Control), cudaMemcpyHostToDevice));
    k_reset<<<1, 1, 0, h->st>>>(h->ctl, h->acc, 1, h->w4key);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
    *out = h;
    return MHD3D_OK;
}

// background index of a field in the FP32 form (-1: stored whole)
int bg_index(int fi)
{
    switch (fi) {
        case F_RO: return 0;
        case F_TT: return 1;
        case F_BX: return 2;
        case F_BY: return 3;
        case F_BZ: return 4;
        default: return -1;
    }
}

// FP32 form: per-plane background terms from the FP64 horizontal means
int set_background(Handle* h)
{
    const int npz = h->p.npz, NZ = npz + 2;
    std::vector<double> b(5 * (size_t)NZ);
    CK(cudaMemcpyAsync(b.data(), h->bgd, sizeof(double) * b.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    const double* R = b.data();
    const double* T = R + NZ;
    const double* B[3] = {R + 2 * NZ, R + 3 * NZ, R + 4 * NZ};
    std::vector<float> b32(2 * (size_t)NZ);
    for (int u = 0; u < NZ; ++u) {
        b32[u] = (float)R[u];
        b32[NZ + u] = (float)T[u];
    }
    const double grav = h->p.grav;
    std::vector<PlaneBg> pb(npz);
    for (int k = 0; k < npz; ++k) {
        const int u = k + 1;   // U plane of interior plane k (Fortran K = k+2)
        const double az = h->faz_h[u], bzq = h->fbz_h[u], czq = h->fcz_h[u];
        PlaneBg& q = pb[k];
        q.az = (float)az;
        q.bzq = (float)bzq;
        q.czq = (float)czq;
        q.rka = (float)h->rka_h[u];
        q.dka = (float)h->dka_h[u];
        q.rddz = (float)(1.0 / h->ddz_h[u]);
        q.ddz = (float)h->ddz_h[u];
        q.fw2z = (float)(0.5 * h->p.repr * h->p.cv / h->rka_h[u]);
        q.robm = (float)R[u - 1];
        q.robc = (float)R[u];
        q.robp = (float)R[u + 1];
        q.ttbm = (float)T[u - 1];
        q.ttbc = (float)T[u];
        q.ttbp = (float)T[u + 1];
        const double tz = T[u + 1] - T[u - 1];
        q.tz = (float)tz;
        q.tlz = (float)(tz * bzq + (T[u + 1] + T[u - 1] - 2.0 * T[u]) * czq);
        q.fw = (float)(grav * R[u] - (R[u + 1] * T[u + 1] - R[u - 1] * T[u - 1]) * az);
        float* bc[3] = {&q.bx, &q.by, &q.bz};
        float* bd[3] = {&q.bxz, &q.byz, &q.bzz};
        float* bl[3] = {&q.bxlz, &q.bylz, &q.bzlz};
        for (int c = 0; c < 3; ++c) {
            const double* Bc = B[c];
            *bc[c] = (float)Bc[u];
            *bd[c] = (float)(Bc[u + 1] - Bc[u - 1]);
            double lz;
            // BX and BY take the one-sided second difference on the walls (as in the kernel)
            if (c < 2 && k == 0)
                lz = (-3.0 * Bc[u] + 4.0 * Bc[u + 1] - Bc[u + 2]) * bzq
                   + (2.0 * Bc[u] - 5.0 * Bc[u + 1] + 4.0 * Bc[u + 2] - Bc[u + 3]) * czq;
            else if (c < 2 && k == npz - 1)
                lz = (3.0 * Bc[u] - 4.0 * Bc[u - 1] + Bc[u - 2]) * bzq
                   + (2.0 * Bc[u] - 5.0 * Bc[u - 1] + 4.0 * Bc[u - 2] - Bc[u - 3]) * czq;
            else
                lz = (Bc[u + 1] - Bc[u - 1]) * bzq + (Bc[u + 1] + Bc[u - 1] - 2.0 * Bc[u]) * czq;
            *bl[c] = (float)lz;
        }
    }
    // wall temperatures in perturbation form (BCON 3dmhdsub.f:2833-2868, 2917-2941)
    const double C13 = h->p.c13, C43 = h->p.c43;
    h->top_tb = T[1];
    h->top_lin = C43 * T[2] - C13 * T[3] - T[1];
    h->t_top_fix = (float)(1.0 - T[1]);
    h->t_top_fix4 = (float)((1.0 - h->p.tp) - T[1]);
    h->t_top_flux = (float)(h->top_lin - h->s.top_flux);
    h->t_bot = h->p.izcon == 0 ? (float)(h->p.tb - T[npz])
                               : (float)(C43 * T[npz - 1] - C13 * T[npz - 2] + h->s.bot_flux - T[npz]);
    CK(cudaMemcpyAsync(h->bg32, b32.data(), sizeof(float) * b32.size(), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->pb, pb.data(), sizeof(PlaneBg) * pb.size(), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return MHD3D_OK;
}

// Upload and download move one field at a time through two staging fields:
// the copy of field i (on the copy stream) overlaps the unpack or pack of
// field i-1 (on the handle's stream); events order each staging field's
// copy, kernel and reuse two fields later.
int upload(Handle* h, const double* const f[8])
{
    CK(cudaSetDevice(h->dev));
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const size_t nfort = (size_t)(npx + 2) * (npy + 2) * (npz + 2);
    for (int i = 0; i < h->nf; ++i)
        if (!f[i]) return MHD3D_ERR_ARG;
    // the staging fields are free once the handle's stream has drained
    CK(cudaEventRecord(h->ev_kern[1], h->st));
    CK(cudaStreamWaitEvent(h->cst, h->ev_kern[1], 0));
    for (int fi = 0; fi < h->nf; ++fi) {
        const int b = fi & 1;
        double* const stg = b ? h->stage2 : h->stage;
        if (fi >= 2) CK(cudaStreamWaitEvent(h->cst, h->ev_kern[b], 0));   // field fi-2 unpacked
        CK(cudaMemcpyAsync(stg, f[fi], sizeof(double) * nfort, cudaMemcpyDefault, h->cst));
        CK(cudaEventRecord(h->ev_copy[b], h->cst));
        CK(cudaStreamWaitEvent(h->st, h->ev_copy[b], 0));
        if (h->f32) {
            const int bi = bg_index(fi);
            double* bg = bi >= 0 ? h->bgd + (size_t)bi * (npz + 2) : nullptr;
            if (bg) k_hmean<<<npz + 2, 256, 0, h->st>>>(stg, bg, npx, npy);
            float* u0 = reinterpret_cast<float*>(h->ubuf[0]) + (size_t)fi * h->uf;
            float* u1 = reinterpret_cast<float*>(h->ubuf[1]) + (size_t)fi * h->uf;
            k_unpack32<<<grid_for(nfort), 256, 0, h->st>>>(stg, bg, u0, u1, npx, npy, npz, h->upitch, h->uz);
        } else {
            k_unpack<<<grid_for(nfort), 256, 0, h->st>>>(stg, h->ubuf[0] + (size_t)fi * h->uf,
                                                         h->ubuf[1] + (size_t)fi * h->uf, npx, npy, npz, h->upitch,
                                                         h->uz);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->ev_kern[b], h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    if (h->f32) {
        int st = set_background(h);
        if (st) return st;
    }
    h->dt_valid = false;
    h->cur_base = h->cur;
    h->pending = 0;
    return MHD3D_OK;
}

int download(Handle* h, double* const f[8])
{
    CK(cudaSetDevice(h->dev));
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const size_t nfort = (size_t)(npx + 2) * (npy + 2) * (npz + 2);
    int n = 0;
    for (int fi = 0; fi < h->nf; ++fi) {
        if (!f[fi]) continue;
        const int b = n & 1;
        double* const stg = b ? h->stage2 : h->stage;
        if (n >= 2) CK(cudaStreamWaitEvent(h->st, h->ev_copy[b], 0));   // the copy of two fields ago done
        if (h->f32) {
            const int bi = bg_index(fi);
            k_pack32<<<grid_for(nfort), 256, 0, h->st>>>(
                reinterpret_cast<const float*>(h->ubuf[h->cur]) + (size_t)fi * h->uf,
                bi >= 0 ? h->bgd + (size_t)bi * (npz + 2) : nullptr, stg, npx, npy, npz, h->upitch, h->uz);
        } else {
            k_pack<<<grid_for(nfort), 256, 0, h->st>>>(h->ubuf[h->cur] + (size_t)fi * h->uf, stg, npx, npy,
                                                       npz, h->upitch, h->uz);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->ev_kern[b], h->st));
        CK(cudaStreamWaitEvent(h->cst, h->ev_kern[b], 0));
        CK(cudaMemcpyAsync(f[fi], stg, sizeof(double) * nfort, cudaMemcpyDefault, h->cst));
        CK(cudaEventRecord(h->ev_copy[b], h->cst));
        ++n;
    }
    CK(cudaStreamSynchronize(h->cst));
    CK(cudaStreamSynchronize(h->st));
    return MHD3D_OK;
}

int initial_dt(Handle* h)
{
    StageArgs a = make_args(h);
    k_reset<<<1, 1, 0, h->st>>>(h->ctl, h->acc, 1, h->w4key);
    CK(cudaGetLastError());
    CK(launch_cfl(h, a));
    k_finalize<<<1, 1, 0, h->st>>>(h->ctl, h->acc, h->s.sf, h->s.dtmin, h->p.lmag, 0, h->w4key);
    CK(cudaGetLastError());
    h->dt_valid = true;
    return MHD3D_OK;
}

int record_event(Handle* h, int stage)
{
    if (h->ev_used + 2 > h->ev_pool.size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            h->ev_pool.push_back(e);
        }
    }
    if (stage >= 0) h->ev_stage.push_back(stage);
    CK(cudaEventRecord(h->ev_pool[h->ev_used++], h->st));
    return MHD3D_OK;
}

int closure_eval(Handle* h, int cur);

int step_async(Handle* h, int n)
{
    CK(cudaSetDevice(h->dev));
    if (n < 0) return MHD3D_ERR_ARG;
    // a call that starts from a synced state clears the stop flag; DT of the
    // current state comes from the last stage-3 reduction, or from a fresh
    // CFL pass after the state changed
    if (!h->dt_valid) {
        int st = initial_dt(h);
        if (st) return st;
    } else if (h->pending == 0) {
        k_reset<<<1, 1, 0, h->st>>>(h->ctl, h->acc, 1, h->w4key);
        CK(cudaGetLastError());
    }
    int cur = h->cur_base ^ (h->pending & 1);
    for (int s = 0; s < n; ++s) {
        if (h->clo) {
            int st = closure_eval(h, cur);
            if (st) return st;
        }
        for (int stg = 1; stg <= 3; ++stg) {
            if (h->prof) {
                int st = record_event(h, stg - 1);
                if (st) return st;
            }
            if (h->f32) {
                StageArgs32 a = make_args32(h);
                a.map_u = h->map_u[cur];
                a.u_in = reinterpret_cast<const float*>(h->ubuf[cur]);
                a.u_out = reinterpret_cast<float*>(h->ubuf[cur ^ 1]);
                CK(f32::launch_stage(stg, a, h->st));
            } else {
                StageArgs a = make_args(h);
                a.map_u = h->map_u[cur];
                a.u_in = h->ubuf[cur];
                a.u_out = h->ubuf[cur ^ 1];
                CK(launch_stage(h, stg, a));
            }
            if (h->prof) {
                int st = record_event(h, -1);
                if (st) return st;
            }
            cur ^= 1;
        }
        k_finalize<<<1, 1, 0, h->st>>>(h->ctl, h->acc, h->s.sf, h->s.dtmin, h->p.lmag, 1, h->w4key);
        CK(cudaGetLastError());
        h->pending += 1;
    }
    h->cur = cur;
    return MHD3D_OK;
}

int sync(Handle* h, double* dt, double* timc, double* timt, double* umach, int32_t* nit)
{
    CK(cudaSetDevice(h->dev));
    Control c{};
    CK(cudaMemcpyAsync(&c, h->ctl, sizeof(Control), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    // steps after a stop returned at once: the state is where the last completed step left it
    const int ran = c.nit - h->nit_base;
    h->cur = h->cur_base ^ (ran & 1);
    h->cur_base = h->cur;
    h->nit_base = c.nit;
    h->pending = 0;
    if (dt) *dt = c.last_dt;
    if (timc) *timc = c.timc;
    if (timt) *timt = c.timt;
    if (umach) *umach = c.last_umach;
    if (nit) *nit = c.nit;
    return c.stop ? c.status : MHD3D_OK;
}

// reconcile enqueued steps before an entry point that reads the state
int settle(Handle* h)
{
    if (h->pending == 0) return MHD3D_OK;
    int st = sync(h, nullptr, nullptr, nullptr, nullptr, nullptr);
    return (st == MHD3D_ERR_CUDA) ? st : MHD3D_OK;
}

int fluxes(Handle* h, double* const out[8])
{
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    if (!h->fout) CK(cudaMalloc(&h->fout, (h->f32 ? sizeof(float) : sizeof(double)) * h->nf * h->zf));
    if (h->f32) {
        CK(f32::launch_stage(0, make_args32(h), h->st));
    } else {
        StageArgs a = make_args(h);
        CK(launch_stage(h, 0, a));
    }
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const size_t nfort = (size_t)(npx + 2) * (npy + 2) * (npz + 2);
    for (int fi = 0; fi < h->nf; ++fi) {
        if (!out[fi]) continue;
        if (h->f32)
            k_pack_interior32<<<grid_for(nfort), 256, 0, h->st>>>(
                reinterpret_cast<const float*>(h->fout) + (size_t)fi * h->zf, h->stage, npx, npy, npz, h->zpitch, h->zz);
        else
            k_pack_interior<<<grid_for(nfort), 256, 0, h->st>>>(h->fout + (size_t)fi * h->zf, h->stage, npx, npy,
                                                                npz, h->zpitch, h->zz);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out[fi], h->stage, sizeof(double) * nfort, cudaMemcpyDeviceToHost, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    return MHD3D_OK;
}

int profiles(Handle* h, double* out)
{
    CK(cudaSetDevice(h->dev));
    if (!out) return MHD3D_ERR_ARG;
    if (int st = settle(h)) return st;
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    double* dout = h->stage;   // the staging field holds far more than MHD3D_NPROF x NPZ doubles
    if (h->f32)
        k_profiles<true><<<npz, PROF_THREADS, 0, h->st>>>(h->ubuf[h->cur], h->bgd, dout, npx, npy, npz, h->upitch,
                                                         h->uz, h->uf, h->p.lmag);
    else
        k_profiles<false><<<npz, PROF_THREADS, 0, h->st>>>(h->ubuf[h->cur], h->bgd, dout, npx, npy, npz, h->upitch,
                                                          h->uz, h->uf, h->p.lmag);
    CK(cudaGetLastError());
    k_frad<<<1, 256, 0, h->st>>>(dout, h->m.dzzdz, h->m.rkapa, h->p.hz, h->p.repr, npz);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout, sizeof(double) * MHD3D_NPROF * npz, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return MHD3D_OK;
}

UView uview(const Handle* h, int cur)
{
    UView v;
    v.u = h->ubuf[cur];
    v.bgd = h->f32 ? h->bgd : nullptr;
    v.uf = h->uf;
    v.uz = h->uz;
    v.NZ = (size_t)h->p.npz + 2;
    v.upitch = h->upitch;
    v.f32 = h->f32 ? 1 : 0;
    return v;
}

// one evaluation of the attached closure on buffer cur: features, three
// convolutions, tendencies and the error indicator, all on the handle's stream
int closure_eval(Handle* h, int cur)
{
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const UView v = uview(h, cur);
    CK(cudaMemsetAsync(h->cflag, 0, sizeof(int), h->st));
    CK(launch_features(h, v, h->cin_scale, h->cmeans, h->cfeat, h->st));
    CK(cudaGetLastError());
    int32_t* err = h->cflag + 3;
    if (mhd3d_conv3d(16, 32, h->cfeat, h->cw[0], h->cb[0], nullptr, 1, h->cact1, nullptr, npx, npy, npz, err, h->st) ||
        mhd3d_conv3d(32, 32, h->cact1, h->cw[1], h->cb[1], nullptr, 1, h->cact2, nullptr, npx, npy, npz, err, h->st) ||
        mhd3d_conv3d(32, 16, h->cact2, h->cw[2], h->cb[2], nullptr, 0, nullptr, h->cpred, npx, npy, npz, err, h->st))
        return MHD3D_ERR_CUDA;
    CK(launch_tendency(v, h->cpred, h->cout_scale, h->m, h->cbias, npx, npy, npz, h->ctrip, h->cfcl, h->zf, h->zz,
                       (size_t)h->zpitch, h->cflag, h->st));
    k_trip_count<<<1, 1, 0, h->st>>>(h->cflag);
    CK(cudaGetLastError());
    return MHD3D_OK;
}

int closure_set(Handle* h, const void* const w[3], const float* const b[3], const float* in_scale,
                const float* out_scale, float trip)
{
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    if (!w[0]) {
        h->clo = false;
        return MHD3D_OK;
    }
    if (!h->f32 || !w[1] || !w[2] || !b[0] || !b[1] || !b[2] || !in_scale || !out_scale)
        return MHD3D_ERR_ARG;
    const size_t nv = (size_t)h->p.npx * h->p.npy * h->p.npz;
    const size_t wn[3] = {32 * 27 * 16, 32 * 27 * 32, 16 * 27 * 32}, bn[3] = {32, 32, 16};
    if (!h->cbuf) {
        size_t bytes = 0;
        auto take = [&](size_t b) { const size_t o = bytes; bytes += (b + 255) / 256 * 256; return o; };
        size_t ow[3], ob[3];
        for (int l = 0; l < 3; ++l) ow[l] = take(wn[l] * 2), ob[l] = take(bn[l] * 4);
        const size_t oin = take(8 * 4), oout = take(12 * 4), ofeat = take(nv * 16 * 2), oa1 = take(nv * 32 * 2),
                     oa2 = take(nv * 32 * 2), opred = take(nv * 16 * 4), ofcl = take((size_t)7 * h->zf * 4),
                     omeans = take((size_t)3 * h->p.npz * 8), oflag = take(4 * 4);
        CK(cudaMalloc(&h->cbuf, bytes));
        CK(cudaMemset(h->cbuf, 0, bytes));
        char* base = static_cast<char*>(h->cbuf);
        for (int l = 0; l < 3; ++l) {
            h->cw[l] = reinterpret_cast<__nv_bfloat16*>(base + ow[l]);
            h->cb[l] = reinterpret_cast<float*>(base + ob[l]);
        }
        h->cin_scale = reinterpret_cast<float*>(base + oin);
        h->cout_scale = reinterpret_cast<float*>(base + oout);
        h->cfeat = reinterpret_cast<__nv_bfloat16*>(base + ofeat);
        h->cact1 = reinterpret_cast<__nv_bfloat16*>(base + oa1);
        h->cact2 = reinterpret_cast<__nv_bfloat16*>(base + oa2);
        h->cpred = reinterpret_cast<float*>(base + opred);
        h->cfcl = reinterpret_cast<float*>(base + ofcl);
        h->cmeans = reinterpret_cast<double*>(base + omeans);
        h->cflag = reinterpret_cast<int*>(base + oflag);
    }
    if (!h->hpart) CK(cudaMalloc(&h->hpart, sizeof(double) * 3 * h->p.npz * HM_SPLIT));   // not in the step path
    for (int l = 0; l < 3; ++l) {
        CK(cudaMemcpyAsync(h->cw[l], w[l], wn[l] * 2, cudaMemcpyDefault, h->st));
        CK(cudaMemcpyAsync(h->cb[l], b[l], bn[l] * 4, cudaMemcpyDefault, h->st));
    }
    CK(cudaMemcpyAsync(h->cin_scale, in_scale, 8 * 4, cudaMemcpyDefault, h->st));
    CK(cudaMemcpyAsync(h->cout_scale, out_scale, 12 * 4, cudaMemcpyDefault, h->st));
    CK(cudaMemsetAsync(h->cflag, 0, 4 * sizeof(int), h->st));
    CK(cudaStreamSynchronize(h->st));
    h->ctrip = trip;
    h->clo = true;
    return MHD3D_OK;
}

// ---- batched ensemble of FP32 grids ---------------------------------------
// Members are ordinary FP32 handles on one stream.  Each RK3 stage of every
// member runs in ONE persistent launch (f32::launch_stage_multi) over a work
// table (member, tile, z chunk), largest members first; k_finalize_multi
// ends the step of all members; one step is one CUDA graph (two graphs,
// for the two ping-pong parities of a step).  The member arguments live in
// device tables that each call refreshes, so the graphs never need
// re-capturing while the decomposition is unchanged.
struct Ensemble {
    std::vector<Handle*> mem;
    cudaStream_t st = nullptr;
    int dev = -1, lmag = 0, lrot = 0, sms = 148;
    int ctas_per_sm = 4;                    // persistent CTAs per SM
    int ty = TY32;                          // tile rows (TX x ty columns a tile)
    StageArgs32* dargs[2] = {nullptr, nullptr};
    int* dorder = nullptr;                  // members by decreasing work
    int* dbase = nullptr;                   // first item of each member in that order (+ total)
    unsigned* dcount = nullptr;             // work counters of the three stages
    FinArgs* dfin = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaStream_t own_st = nullptr;          // the ensemble's own stream while a caller's is in use
    std::vector<int> order;
    int nitems = 0;
};

int ens_destroy(Ensemble* e)
{
    if (!e) return MHD3D_OK;
    if (e->dev >= 0) cudaSetDevice(e->dev);
    for (int q = 0; q < 2; ++q) {
        if (e->graph[q]) cudaGraphExecDestroy(e->graph[q]);
        cudaFree(e->dargs[q]);
    }
    cudaFree(e->dorder);
    cudaFree(e->dbase);
    cudaFree(e->dcount);
    cudaFree(e->dfin);
    for (Handle* h : e->mem) destroy(h);
    if (e->own_st) cudaStreamDestroy(e->own_st);
    else if (e->st) cudaStreamDestroy(e->st);
    delete e;
    return MHD3D_OK;
}

// work table: member order (largest first) and item prefix sums
int ens_layout(Ensemble* e)
{
    const int n = (int)e->mem.size();
    std::vector<long> items(n);
    for (int i = 0; i < n; ++i) {
        Handle* h = e->mem[i];
        items[i] = (long)h->ntx * ((h->p.npy + e->ty - 1) / e->ty) * h->nchunks;
    }
    e->order.resize(n);
    for (int i = 0; i < n; ++i) e->order[i] = i;
    std::stable_sort(e->order.begin(), e->order.end(), [&](int a, int b) { return items[a] > items[b]; });
    std::vector<int> base(n + 1, 0);
    for (int i = 0; i < n; ++i) base[i + 1] = base[i] + (int)items[e->order[i]];
    e->nitems = base[n];
    CK(cudaMemcpyAsync(e->dorder, e->order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, e->st));
    CK(cudaMemcpyAsync(e->dbase, base.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    for (int q = 0; q < 2; ++q)
        if (e->graph[q]) {
            cudaGraphExecDestroy(e->graph[q]);
            e->graph[q] = nullptr;
        }
    return MHD3D_OK;
}

int ens_set_tile(Ensemble* e, int ty);

int ens_create(int n, const mhd3d_params* ps, const double* const* grids, Ensemble** out)
{
    if (n < 1 || !ps || !grids) return MHD3D_ERR_ARG;
    for (int i = 0; i < n; ++i)
        if (ps[i].mode != MHD3D_MODE_FP32 || ps[i].lmag != ps[0].lmag || ps[i].lrot != ps[0].lrot)
            return MHD3D_ERR_ARG;
    Ensemble* e = new (std::nothrow) Ensemble();
    if (!e) return MHD3D_ERR_NOMEM;
    *out = e;
    CK(cudaGetDevice(&e->dev));
    CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
    cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->dev);
    e->lmag = ps[0].lmag;
    e->lrot = ps[0].lrot;
    e->mem.assign(n, nullptr);
    for (int i = 0; i < n; ++i) {
        void* hv = nullptr;
        int st = create(&ps[i], grids + 14 * (size_t)i, &hv);
        e->mem[i] = static_cast<Handle*>(hv);
        if (st) return st;
        e->mem[i]->st = e->st;   // every member works on the ensemble's stream
    }
    for (int q = 0; q < 2; ++q) CK(cudaMalloc(&e->dargs[q], sizeof(StageArgs32) * n));
    CK(cudaMalloc(&e->dorder, sizeof(int) * n));
    CK(cudaMalloc(&e->dbase, sizeof(int) * (n + 1)));
    CK(cudaMalloc(&e->dcount, sizeof(unsigned) * 4));
    CK(cudaMalloc(&e->dfin, sizeof(FinArgs) * n));
    std::vector<FinArgs> fin(n);
    for (int i = 0; i < n; ++i) {
        Handle* h = e->mem[i];
        fin[i] = FinArgs{h->ctl, h->acc, h->s.sf, h->s.dtmin, h->w4key, h->p.lmag, 0};
    }
    CK(cudaMemcpy(e->dfin, fin.data(), sizeof(FinArgs) * n, cudaMemcpyHostToDevice));
    for (int ty : {2, 4, 8})   // kernel attributes are set outside any graph capture
        for (int stg = 1; stg <= 3; ++stg)
            CK(f32::launch_stage_multi(stg, e->lmag, e->lrot, ty, nullptr, nullptr, nullptr, 0, nullptr, 0, e->st));
    if (int st = ens_set_tile(e, TY32)) return st;
    return ens_layout(e);
}

// tile rows every member can take: boxes of ty+2 U rows and ty Z rows must
// fit the padded arrays
bool ens_tile_fits(const Ensemble* e, int ty)
{
    if (!f32::multi_tile_rows_ok(ty)) return false;
    for (const Handle* h : e->mem)
        if (ty + 2 > h->urows || ty > h->zrows) return false;
    return true;
}

// set the ensemble's tile rows: TMA maps of every member for that box height
// (emap_*, used by the ensemble's argument tables only) and the work table
int ens_set_tile(Ensemble* e, int ty)
{
    if (!ens_tile_fits(e, ty)) return MHD3D_ERR_ARG;
    for (Handle* h : e->mem) {
        const int NZ = h->p.npz + 2;
        const cuuint64_t du[4] = {(cuuint64_t)h->upitch, (cuuint64_t)h->urows, (cuuint64_t)NZ, (cuuint64_t)h->nf};
        const cuuint32_t bu[4] = {(cuuint32_t)BW32, (cuuint32_t)(ty + 2), 1, (cuuint32_t)h->nf};
        for (int b = 0; b < 2; ++b)
            if (int st = make_map(&h->emap_u[b], h->ubuf[b], du, bu, true)) return st;
        const cuuint64_t dz[4] = {(cuuint64_t)h->zpitch, (cuuint64_t)h->zrows, (cuuint64_t)h->p.npz,
                                  (cuuint64_t)h->nf};
        const cuuint32_t bz[4] = {TX, (cuuint32_t)ty, 1, (cuuint32_t)h->nf};
        if (int st = make_map(&h->emap_z, h->z, dz, bz, true)) return st;
        h->ety = ty;
    }
    e->ty = ty;
    return ens_layout(e);
}

// set every member's z chunk length (<= 0: the single-grid default) and re-lay the work table
int ens_set_zlen(Ensemble* e, int zlen)
{
    for (Handle* h : e->mem) {
        const int npz = h->p.npz;
        int nch;
        if (zlen > 0) nch = std::max(1, npz / std::max(zlen, 3));
        else nch = std::max(1, (npz + MHD3D_ZCHUNK - 1) / MHD3D_ZCHUNK);
        while (nch > 1 && npz / nch < 3) --nch;
        h->nchunks = nch;
        h->zlen = npz / nch;
    }
    return ens_layout(e);
}

int ens_capture(Ensemble* e, int q)
{
    // a step whose stage 1 reads table q: stages use tables q, q^1, q
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    const int nb = std::max(1, std::min(e->nitems, e->sms * e->ctas_per_sm));
    const int n = (int)e->mem.size();
    cudaError_t err = cudaMemsetAsync(e->dcount, 0, sizeof(unsigned) * 4, e->st);
    for (int stg = 1; stg <= 3 && err == cudaSuccess; ++stg)
        err = f32::launch_stage_multi(stg, e->lmag, e->lrot, e->ty, e->dargs[(stg == 2) ? (q ^ 1) : q], e->dorder,
                                      e->dbase, n, e->dcount + (stg - 1), nb, e->st);
    if (err == cudaSuccess) {
        k_finalize_multi<<<(n + 127) / 128, 128, 0, e->st>>>(e->dfin, n);
        err = cudaGetLastError();
    }
    cudaError_t e2 = cudaStreamEndCapture(e->st, &g);
    if (err != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        CK(err != cudaSuccess ? err : e2);
    }
    err = cudaGraphInstantiate(&e->graph[q], g, 0);
    cudaGraphDestroy(g);
    CK(err);
    return MHD3D_OK;
}

int ens_step(Ensemble* e, int nsteps)
{
    CK(cudaSetDevice(e->dev));
    if (nsteps < 0) return MHD3D_ERR_ARG;
    const int n = (int)e->mem.size();
    std::vector<StageArgs32> tab[2];
    tab[0].resize(n);
    tab[1].resize(n);
    std::vector<int> cur0(n);
    for (int i = 0; i < n; ++i) {
        Handle* h = e->mem[i];
        if (!h->dt_valid) {
            int st = initial_dt(h);
            if (st) return st;
        } else if (h->pending == 0) {
            k_reset<<<1, 1, 0, h->st>>>(h->ctl, h->acc, 1, h->w4key);
            CK(cudaGetLastError());
        }
        const int cur = h->cur_base ^ (h->pending & 1);
        cur0[i] = cur;
        for (int p = 0; p < 2; ++p) {
            StageArgs32 a = make_args32(h);
            const int in = cur ^ p;
            a.map_u = h->emap_u[in];   // the ensemble's tile rows
            a.map_z = h->emap_z;
            a.u_in = reinterpret_cast<const float*>(h->ubuf[in]);
            a.u_out = reinterpret_cast<float*>(h->ubuf[in ^ 1]);
            tab[p][i] = a;
        }
    }
    for (int p = 0; p < 2; ++p)
        CK(cudaMemcpyAsync(e->dargs[p], tab[p].data(), sizeof(StageArgs32) * n, cudaMemcpyHostToDevice, e->st));
    for (int q = 0; q < 2; ++q)
        if (!e->graph[q]) {
            int st = ens_capture(e, q);
            if (st) return st;
        }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(e->graph[s & 1], e->st));
    for (int i = 0; i < n; ++i) {
        Handle* h = e->mem[i];
        h->pending += nsteps;
        h->cur = cur0[i] ^ (nsteps & 1);
    }
    return MHD3D_OK;
}

int ens_sync(Ensemble* e, double* dt, double* timt, int32_t* nit, int32_t* status)
{
    CK(cudaSetDevice(e->dev));
    int worst = MHD3D_OK;
    for (size_t i = 0; i < e->mem.size(); ++i) {
        double d = 0, tc = 0, tt = 0, um = 0;
        int32_t ni = 0;
        const int st = sync(e->mem[i], &d, &tc, &tt, &um, &ni);
        if (dt) dt[i] = d;
        if (timt) timt[i] = tt;
        if (nit) nit[i] = ni;
        if (status) status[i] = st;
        if (st == MHD3D_ERR_CUDA) return st;
        if (st && !worst) worst = st;
    }
    return worst;
}

// Autotuner: time a few steps for each (z chunk length, persistent CTAs per
// SM) pair on the live state, keep the fastest, and put the state back.
int ens_tune(Ensemble* e, int steps, int32_t* zlen_out, int32_t* ctas_out, double* ms_out)
{
    CK(cudaSetDevice(e->dev));
    if (int st = ens_sync(e, nullptr, nullptr, nullptr, nullptr)) {
        if (st == MHD3D_ERR_CUDA) return st;
    }
    const int n = (int)e->mem.size();
    int maxnpz = 0;
    for (Handle* h : e->mem) maxnpz = std::max(maxnpz, h->p.npz);
    // snapshot: both U buffers, Control, Accum of every member
    std::vector<void*> snap(n, nullptr);
    std::vector<size_t> ubytes(n);
    for (int i = 0; i < n; ++i) {
        Handle* h = e->mem[i];
        ubytes[i] = (h->f32 ? sizeof(float) : sizeof(double)) * h->nf * h->uf;
        CK(cudaMalloc(&snap[i], 2 * ubytes[i] + sizeof(Control) + sizeof(Accum)));
        char* b = static_cast<char*>(snap[i]);
        CK(cudaMemcpyAsync(b, h->ubuf[0], ubytes[i], cudaMemcpyDeviceToDevice, e->st));
        CK(cudaMemcpyAsync(b + ubytes[i], h->ubuf[1], ubytes[i], cudaMemcpyDeviceToDevice, e->st));
        CK(cudaMemcpyAsync(b + 2 * ubytes[i], h->ctl, sizeof(Control), cudaMemcpyDeviceToDevice, e->st));
        CK(cudaMemcpyAsync(b + 2 * ubytes[i] + sizeof(Control), h->acc, sizeof(Accum), cudaMemcpyDeviceToDevice,
                           e->st));
    }
    std::vector<int> saved_cur(n), saved_base(n), saved_nit(n), saved_valid(n);
    for (int i = 0; i < n; ++i) {
        saved_cur[i] = e->mem[i]->cur;
        saved_base[i] = e->mem[i]->cur_base;
        saved_nit[i] = e->mem[i]->nit_base;
        saved_valid[i] = e->mem[i]->dt_valid;
    }
    auto restore = [&]() -> int {
        for (int i = 0; i < n; ++i) {
            Handle* h = e->mem[i];
            char* b = static_cast<char*>(snap[i]);
            CK(cudaMemcpyAsync(h->ubuf[0], b, ubytes[i], cudaMemcpyDeviceToDevice, e->st));
            CK(cudaMemcpyAsync(h->ubuf[1], b + ubytes[i], ubytes[i], cudaMemcpyDeviceToDevice, e->st));
            CK(cudaMemcpyAsync(h->ctl, b + 2 * ubytes[i], sizeof(Control), cudaMemcpyDeviceToDevice, e->st));
            CK(cudaMemcpyAsync(h->acc, b + 2 * ubytes[i] + sizeof(Control), sizeof(Accum), cudaMemcpyDeviceToDevice,
                               e->st));
            h->cur = saved_cur[i];
            h->cur_base = saved_base[i];
            h->nit_base = saved_nit[i];
            h->pending = 0;
            h->dt_valid = saved_valid[i];
        }
        CK(cudaStreamSynchronize(e->st));
        return MHD3D_OK;
    };
    // search: tile rows (32 x 2, 32 x 4, 32 x 8 columns a tile, separate
    // kernel instances) x z chunk length x persistent CTAs per SM (8, 12 or 16
    // warps an SM where the tile allows)
    const int zc[] = {4, 6, 8, 12, 16, 24, 32, 48, 64};
    struct TileChoice {
        int ty, nc, cc[3];
    };
    const TileChoice tcs[] = {{2, 3, {4, 6, 8}}, {4, 3, {2, 3, 4}}, {8, 2, {1, 2, 0}}};
    int best_z = 0, best_c = e->ctas_per_sm, best_t = e->ty;
    double best = 1e300;
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    int st = MHD3D_OK;
    for (const TileChoice& tc : tcs) {
        if (st || !ens_tile_fits(e, tc.ty)) continue;
        if ((st = ens_set_tile(e, tc.ty))) break;
        for (int zi = 0; zi < (int)(sizeof(zc) / sizeof(zc[0])) && !st; ++zi) {
            if (zc[zi] > maxnpz) break;
            for (int ci = 0; ci < tc.nc && !st; ++ci) {
                e->ctas_per_sm = tc.cc[ci];
                if ((st = ens_set_zlen(e, zc[zi]))) break;
                if ((st = ens_step(e, 1))) break;   // warm-up, builds the graphs
                cudaEventRecord(t0, e->st);
                if ((st = ens_step(e, steps))) break;
                cudaEventRecord(t1, e->st);
                if (cudaEventSynchronize(t1) != cudaSuccess) { st = MHD3D_ERR_CUDA; break; }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, t0, t1);
                if ((st = restore())) break;
                const double per = ms / std::max(steps, 1);
                if (per < best) {
                    best = per;
                    best_z = zc[zi];
                    best_c = tc.cc[ci];
                    best_t = tc.ty;
                }
            }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    int st2 = restore();
    for (void* p : snap) cudaFree(p);
    if (st) return st;
    if (st2) return st2;
    e->ctas_per_sm = best_c;
    if (int s3 = ens_set_tile(e, best_t)) return s3;
    if (int s3 = ens_set_zlen(e, best_z)) return s3;
    if (zlen_out) *zlen_out = best_z;
    if (ctas_out) *ctas_out = best_c;
    if (ms_out) *ms_out = best;
    return MHD3D_OK;
}

}  // namespace
}  // namespace mhd3d

using namespace mhd3d;

extern "C" {

int mhd3d_create(const mhd3d_params* p,
                 const double* exx, const double* dxxdx, const double* d2xxdx2, const double* ddx,
                 const double* wyy, const double* dyydy, const double* d2yydy2, const double* ddy,
                 const double* zee, const double* dzzdz, const double* d2zzdz2, const double* ddz,
                 const double* rkapa, const double* dkapa, void** handle)
{
    if (!handle) return MHD3D_ERR_ARG;
    *handle = nullptr;
    const double* arrs[14] = {exx, dxxdx, d2xxdx2, ddx, wyy, dyydy, d2yydy2, ddy, zee, dzzdz, d2zzdz2, ddz, rkapa, dkapa};
    void* h = nullptr;
    int st = create(p, arrs, &h);
    if (st) {
        destroy(static_cast<Handle*>(h));
        return st;
    }
    *handle = h;
    return MHD3D_OK;
}

int mhd3d_destroy(void* handle) { return destroy(static_cast<Handle*>(handle)); }

int mhd3d_upload(void* handle, const double* ru, const double* rv, const double* rw, const double* tt,
                 const double* ro, const double* bx, const double* by, const double* bz)
{
    if (!handle) return MHD3D_ERR_ARG;
    const double* f[8] = {ru, rv, rw, tt, ro, bx, by, bz};
    if (int st = settle(static_cast<Handle*>(handle))) return st;
    return upload(static_cast<Handle*>(handle), f);
}

int mhd3d_download(void* handle, double* ru, double* rv, double* rw, double* tt, double* ro, double* bx,
                   double* by, double* bz)
{
    if (!handle) return MHD3D_ERR_ARG;
    double* f[8] = {ru, rv, rw, tt, ro, bx, by, bz};
    if (int st = settle(static_cast<Handle*>(handle))) return st;
    return download(static_cast<Handle*>(handle), f);
}

int mhd3d_step(void* handle, int32_t nsteps, double* dt, double* timc, double* timt, double* umach, int32_t* nit)
{
    if (!handle) return MHD3D_ERR_ARG;
    Handle* h = static_cast<Handle*>(handle);
    int st = step_async(h, nsteps);
    if (st) return st;
    return sync(h, dt, timc, timt, umach, nit);
}

int mhd3d_step_async(void* handle, int32_t nsteps)
{
    if (!handle) return MHD3D_ERR_ARG;
    return step_async(static_cast<Handle*>(handle), nsteps);
}

int mhd3d_sync(void* handle, double* dt, double* timc, double* timt, double* umach, int32_t* nit)
{
    if (!handle) return MHD3D_ERR_ARG;
    return sync(static_cast<Handle*>(handle), dt, timc, timt, umach, nit);
}

int mhd3d_set_stream(void* handle, void* stream)
{
    if (!handle) return MHD3D_ERR_ARG;
    Handle* h = static_cast<Handle*>(handle);
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->st));
    h->st = stream ? static_cast<cudaStream_t>(stream) : h->own;
    return MHD3D_OK;
}

int mhd3d_set_wait_limit(void* handle, int64_t polls)
{
    if (!handle || polls < 0) return MHD3D_ERR_ARG;
    Handle* h = static_cast<Handle*>(handle);
    if (h->f32) return MHD3D_ERR_ARG;   // the FP64 stage kernels only
    h->wait_first = polls ? (long long)std::min<int64_t>(polls, WAIT_LIMIT) : 0;
    return MHD3D_OK;
}

int mhd3d_profile(void* handle, int32_t enable)
{
    if (!handle) return MHD3D_ERR_ARG;
    static_cast<Handle*>(handle)->prof = enable != 0;
    return MHD3D_OK;
}

int mhd3d_profile_read(void* handle, double stage_ms[3], int32_t launches[3])
{
    if (!handle || !stage_ms || !launches) return MHD3D_ERR_ARG;
    Handle* h = static_cast<Handle*>(handle);
    CK(cudaSetDevice(h->dev));
    CK(cudaStreamSynchronize(h->st));
    for (int i = 0; i < 3; ++i) {
        stage_ms[i] = 0.0;
        launches[i] = 0;
    }
    for (size_t q = 0; q < h->ev_stage.size(); ++q) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, h->ev_pool[2 * q], h->ev_pool[2 * q + 1]));
        stage_ms[h->ev_stage[q]] += ms;
        launches[h->ev_stage[q]] += 1;
    }
    h->ev_stage.clear();
    h->ev_used = 0;
    return MHD3D_OK;
}

int mhd3d_fluxes(void* handle, double* fu, double* fv, double* fw, double* fr, double* ft, double* ww1,
                 double* ww2, double* ww3)
{
    if (!handle) return MHD3D_ERR_ARG;
    double* o[8] = {fu, fv, fw, fr, ft, ww1, ww2, ww3};
    return fluxes(static_cast<Handle*>(handle), o);
}

int mhd3d_profiles(void* handle, double* out)
{
    if (!handle) return MHD3D_ERR_ARG;
    return profiles(static_cast<Handle*>(handle), out);
}

int mhd3d_cfl(void* handle, double* dt, double* umach)
{
    if (!handle) return MHD3D_ERR_ARG;
    Handle* h = static_cast<Handle*>(handle);
    CK(cudaSetDevice(h->dev));
    if (int st0 = settle(h)) return st0;
    int st = initial_dt(h);
    if (st) return st;
    Control c{};
    CK(cudaMemcpyAsync(&c, h->ctl, sizeof(Control), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (dt) *dt = c.dt;
    if (umach) *umach = c.umach;
    return c.stop ? c.status : MHD3D_OK;
}

int mhd3d_bcon(void* handle)
{
    if (!handle) return MHD3D_ERR_ARG;
    Handle* h = static_cast<Handle*>(handle);
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    if (h->f32) return MHD3D_ERR_ARG;
    StageArgs a = make_args(h);
    CK(h->p.mode == MHD3D_MODE_FAST ? fast::launch_bcon(a, h->st) : exact::launch_bcon(a, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->dt_valid = false;
    return MHD3D_OK;
}

int mhd3d_closure_set(void* handle, const void* w1, const float* b1, const void* w2, const float* b2, const void* w3,
                      const float* b3, const float* in_scale, const float* out_scale, float trip)
{
    if (!handle) return MHD3D_ERR_ARG;
    const void* w[3] = {w1, w2, w3};
    const float* b[3] = {b1, b2, b3};
    return closure_set(static_cast<Handle*>(handle), w, b, in_scale, out_scale, trip);
}

int mhd3d_closure_set_bias(void* handle, const float* bias)
{
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !h->f32) return MHD3D_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    if (!bias) {
        cudaFree(h->cbias);
        cudaFree(h->cbtend);
        h->cbias = h->cbtend = nullptr;
        return MHD3D_OK;
    }
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const size_t n = (size_t)7 * npz;
    // the bias and, for steps without a network, its tendencies and a zero
    // trip flag: both buffers or neither
    if (!h->cbias || !h->cbtend) {
        cudaFree(h->cbias);
        cudaFree(h->cbtend);
        h->cbias = h->cbtend = nullptr;
        float *pb = nullptr, *pt = nullptr;
        if (cudaMalloc(&pb, n * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&pt, 7 * h->zf * sizeof(float) + 4 * sizeof(int)) != cudaSuccess) {
            (void)cudaGetLastError();
            cudaFree(pb);
            return MHD3D_ERR_NOMEM;
        }
        h->cbias = pb;
        h->cbtend = pt;
    }
    cudaError_t e = cudaMemcpyAsync(h->cbias, bias, n * sizeof(float), cudaMemcpyDefault, h->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->cbtend + 7 * h->zf, 0, 4 * sizeof(int), h->st);
    if (e == cudaSuccess) {
        k_bias_tendency<<<grid_for((size_t)npx * npy * npz), 256, 0, h->st>>>(h->cbias, npx, npy, npz, h->cbtend,
                                                                              h->zf, h->zz, (size_t)h->zpitch);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) {
        // no half-set bias: the handle is left without one
        std::fprintf(stderr, "mhd3d: mhd3d_closure_set_bias failed: %s\n", cudaGetErrorString(e));
        cudaFree(h->cbias);
        cudaFree(h->cbtend);
        h->cbias = h->cbtend = nullptr;
        return MHD3D_ERR_CUDA;
    }
    return MHD3D_OK;
}

int mhd3d_closure_status(void* handle, int32_t* trips, int32_t* evals, int32_t* err)
{
    Handle* h = static_cast<Handle*>(handle);
    if (!h) return MHD3D_ERR_ARG;
    int f[4] = {0, 0, 0, 0};
    CK(cudaSetDevice(h->dev));
    if (h->cflag) {
        CK(cudaMemcpyAsync(f, h->cflag, sizeof f, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    }
    if (trips) *trips = f[1];
    if (evals) *evals = f[2];
    if (err) *err = f[3];
    return MHD3D_OK;
}

int mhd3d_coarsen(void* fine, int32_t fac, double* cstate, float* targets, void* stream)
{
    Handle* h = static_cast<Handle*>(fine);
    if (!h || fac < 1 || !cstate || !targets || h->p.npx % fac || h->p.npy % fac || h->p.npz % fac) return MHD3D_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    CK(cudaStreamSynchronize(h->st));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int npxc = h->p.npx / fac, npyc = h->p.npy / fac, npzc = h->p.npz / fac;
    const size_t nc = (size_t)npxc * npyc * npzc;
    k_coarsen<<<grid_for(nc), 128, 0, s>>>(uview(h, h->cur), fac, npxc, npyc, npzc, h->p.lmag, cstate, targets);
    const size_t nfull = (size_t)(h->p.lmag ? 8 : 5) * (npxc + 2) * (npyc + 2) * (npzc + 2);
    k_fort_wrap<<<grid_for(nfull), 256, 0, s>>>(cstate, h->p.lmag ? 8 : 5, npxc, npyc, npzc);
    CK(cudaGetLastError());
    return MHD3D_OK;
}

int mhd3d_closure_features(void* handle, const float* in_scale, void* feat, double* means, void* stream)
{
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !in_scale || !feat || !means) return MHD3D_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    CK(cudaStreamSynchronize(h->st));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const UView v = uview(h, h->cur);
    CK(launch_features(h, v, in_scale, means, static_cast<__nv_bfloat16*>(feat), s));
    return MHD3D_OK;
}

int mhd3d_closure_loss(const float* pred, const float* target, int64_t nvox, void* dy, double* loss, void* stream)
{
    if (!pred || !target || nvox <= 0 || !loss) return MHD3D_ERR_ARG;
    k_closure_loss<<<grid_for((size_t)nvox), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        pred, target, (size_t)nvox, static_cast<__nv_bfloat16*>(dy), loss);
    CK(cudaGetLastError());
    return MHD3D_OK;
}

int mhd3d_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
               int32_t t, void* p_bf16, void* stream)
{
    if (!p || !g || !m || !v || n <= 0 || t < 1) return MHD3D_ERR_ARG;
    const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
    k_adam<<<grid_for((size_t)n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, g, m, v, (size_t)n, lr, b1, b2, eps, bc1, bc2, static_cast<__nv_bfloat16*>(p_bf16));
    CK(cudaGetLastError());
    return MHD3D_OK;
}

int mhd3d_closure_tendency(void* handle, const float* pred, const float* out_scale, float* out, int32_t* flag,
                           float trip, void* stream)
{
    Handle* h = static_cast<Handle*>(handle);
    // pred rows are read as 16-byte vectors
    if (!h || !pred || (reinterpret_cast<uintptr_t>(pred) & 15u) || !out_scale || !out || !flag) return MHD3D_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    CK(cudaStreamSynchronize(h->st));
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const size_t nv = (size_t)npx * npy * npz;
    CK(launch_tendency(uview(h, h->cur), pred, out_scale, h->m, nullptr, npx, npy, npz, trip, out, nv, (size_t)npx * npy,
                       (size_t)npx, flag, static_cast<cudaStream_t>(stream)));
    return MHD3D_OK;
}

int mhd3d_closure_tendency_adjoint(void* handle, const float* g, const float* out_scale, void* dpred, void* stream)
{
    Handle* h = static_cast<Handle*>(handle);
    if (!h || !g || !out_scale || !dpred) return MHD3D_ERR_ARG;
    CK(cudaSetDevice(h->dev));
    if (int st = settle(h)) return st;
    CK(cudaStreamSynchronize(h->st));
    const int npx = h->p.npx, npy = h->p.npy, npz = h->p.npz;
    const size_t nv = (size_t)npx * npy * npz;
    k_tendency_adj<<<grid_for(nv), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        uview(h, h->cur), g, out_scale, h->m.fax, h->m.fay, h->m.faz, npx, npy, npz, nv,
        static_cast<__nv_bfloat16*>(dpred));
    CK(cudaGetLastError());
    return MHD3D_OK;
}

int mhd3d_closure_tendency_loss(const float* tend, const float* target, const float* weight, int64_t nvox, float* g,
                                double* loss, void* stream)
{
    if (!tend || !target || !weight || nvox <= 0 || !g || !loss) return MHD3D_ERR_ARG;
    k_tendency_loss<<<grid_for((size_t)nvox * 7), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        tend, target, weight, (size_t)nvox, g, loss);
    CK(cudaGetLastError());
    return MHD3D_OK;
}

int mhd3d_ensemble_create(int32_t nmembers, const mhd3d_params* params, const double* const* grids, void** ens)
{
    if (!ens) return MHD3D_ERR_ARG;
    *ens = nullptr;
    Ensemble* e = nullptr;
    int st = ens_create(nmembers, params, grids, &e);
    if (st) {
        ens_destroy(e);
        return st;
    }
    *ens = e;
    return MHD3D_OK;
}

int mhd3d_ensemble_destroy(void* ens) { return ens_destroy(static_cast<Ensemble*>(ens)); }

int mhd3d_ensemble_member(void* ens, int32_t i, void** handle)
{
    Ensemble* e = static_cast<Ensemble*>(ens);
    if (!e || !handle || i < 0 || i >= (int)e->mem.size()) return MHD3D_ERR_ARG;
    *handle = e->mem[i];
    return MHD3D_OK;
}

int mhd3d_ensemble_step(void* ens, int32_t nsteps)
{
    if (!ens) return MHD3D_ERR_ARG;
    return ens_step(static_cast<Ensemble*>(ens), nsteps);
}

int mhd3d_ensemble_sync(void* ens, double* dt, double* timt, int32_t* nit, int32_t* status)
{
    if (!ens) return MHD3D_ERR_ARG;
    return ens_sync(static_cast<Ensemble*>(ens), dt, timt, nit, status);
}

int mhd3d_ensemble_set_stream(void* ens, void* stream)
{
    Ensemble* e = static_cast<Ensemble*>(ens);
    if (!e) return MHD3D_ERR_ARG;
    CK(cudaSetDevice(e->dev));
    CK(cudaStreamSynchronize(e->st));
    if (!e->own_st) e->own_st = e->st;
    e->st = stream ? static_cast<cudaStream_t>(stream) : e->own_st;
    for (Handle* h : e->mem) h->st = e->st;
    return MHD3D_OK;
}

int mhd3d_ensemble_set_tile(void* ens, int32_t tile_y)
{
    if (!ens) return MHD3D_ERR_ARG;
    Ensemble* e = static_cast<Ensemble*>(ens);
    CK(cudaSetDevice(e->dev));
    if (int st = ens_sync(e, nullptr, nullptr, nullptr, nullptr))
        if (st == MHD3D_ERR_CUDA) return st;
    return ens_set_tile(e, tile_y);
}

int mhd3d_ensemble_tile(void* ens, int32_t* tile_x, int32_t* tile_y)
{
    if (!ens) return MHD3D_ERR_ARG;
    const Ensemble* e = static_cast<const Ensemble*>(ens);
    if (tile_x) *tile_x = TX;
    if (tile_y) *tile_y = e->ty;
    return MHD3D_OK;
}

int mhd3d_ensemble_tune(void* ens, int32_t steps, int32_t* zlen, int32_t* ctas_per_sm, double* ms_per_step)
{
    if (!ens || steps < 1) return MHD3D_ERR_ARG;
    return ens_tune(static_cast<Ensemble*>(ens), steps, zlen, ctas_per_sm, ms_per_step);
}

const char* mhd3d_version(void) { return "mhd3d-b200 0.2 (sm_100a, FP64 exact/FMA, FP32 perturbation form)"; }

}  // extern "C"
