// cfl_noalloc.cu -- the CFL/Mach reduction of STEP for callers that cannot
// allocate device memory.
//
// Some hosts cannot call cudaMalloc: a Fortran or C code whose device arrays
// are all declared statically, a framework whose caching allocator owns the
// whole device heap, or a job slot with a hard device-memory cap.  They hold
// the prognostic fields in device memory already and only need DT and the
// Mach number of that state.  This entry point uses no handle and allocates
// nothing: its only scratch, one row of partial results per z plane, is a
// file-scope __device__ array that every GPU loading the library holds until
// the process exits.
//
// Built without FMA contraction, so the result equals the handle-based
// reduction of the reference-rounding mode (mhd3d_cfl) bit for bit.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/mhd3d.h"
#define MHD3D_NS noalloc
#include "cfl_cell.cuh"

namespace mhd3d {
namespace noalloc {

constexpr int NTHR = 256;
constexpr int NKEY = 6;   // w1..w4 minima, Mach^2 maximum, non-finite flag

// Per-plane partial results; sized for MHD3D_NOALLOC_MAX_PLANES planes.
static __device__ __align__(256) unsigned long long g_cfl_partials[MHD3D_NOALLOC_MAX_PLANES * NKEY];

// Device address of g_cfl_partials in the current device's context.  The
// symbol's host-side name is not a device address, so it is looked up with
// the device current.  The lookup runs again on every call made outside a
// stream capture: after cudaDeviceReset (or any teardown of the primary
// context) the module is loaded again, possibly at another address, and a
// remembered address would be stale.  A call whose stream is being captured
// reuses the address the last uncaptured call on this device found, so the
// first call on a device has to come before any capture.
constexpr int MAX_DEVICES = 64;
static void* g_partials_addr[MAX_DEVICES];
static std::mutex g_mutex;

static int partials_address(int dev, cudaStream_t st, void** out)
{
    if (dev < 0 || dev >= MAX_DEVICES) return MHD3D_ERR_ARG;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    bool capturing = false;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        (void)cudaGetLastError();   // the query's own error is not the caller's
        capturing = true;
    } else {
        capturing = cap != cudaStreamCaptureStatusNone;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!capturing) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_cfl_partials) != cudaSuccess || !p) return MHD3D_ERR_CUDA;
        g_partials_addr[dev] = p;
    }
    if (!g_partials_addr[dev]) return MHD3D_ERR_CUDA;
    *out = g_partials_addr[dev];
    return MHD3D_OK;
}

// One block per z plane: reduce the plane's CFL terms into its row of partials.
template <bool MAG>
__global__ void __launch_bounds__(NTHR) k_cfl_planes(Scalars s, const double* __restrict__ ru,
                                                       const double* __restrict__ rv, const double* __restrict__ rw,
                                                       const double* __restrict__ tt, const double* __restrict__ ro,
                                                       const double* __restrict__ bx, const double* __restrict__ by,
                                                       const double* __restrict__ bz, const double* __restrict__ ddx,
                                                       const double* __restrict__ ddy, const double* __restrict__ ddz,
                                                       const double* __restrict__ rkapa, unsigned long long* partials)
{
    const int k = blockIdx.x;
    const int npx = s.npx, npy = s.npy;
    const size_t NX = (size_t)npx + 2, NY = (size_t)npy + 2;
    unsigned long long kw1 = ~0ull, kw2 = ~0ull, kw3 = ~0ull, kw4 = ~0ull, kmu = 0ull;
    unsigned int bad = 0;
    const double ddk = ddz[k + 1], rka = rkapa[k + 1];
    for (int q = threadIdx.x; q < npx * npy; q += NTHR) {
        const int i = q % npx, j = q / npx;
        const size_t c = (size_t)(i + 1) + NX * ((size_t)(j + 1) + NY * (size_t)(k + 1));
        const double dd = dmin(dmin(ddx[i + 1], ddy[j + 1]), ddk);
        CflPart cp;
        cfl_cell<MAG>(s, ru[c], rv[c], rw[c], ro[c], tt[c], MAG ? bx[c] : 0.0, MAG ? by[c] : 0.0,
                      MAG ? bz[c] : 0.0, dd, rka, cp);
        kw1 = min(kw1, key_of(cp.w1));
        kw2 = min(kw2, key_of(cp.w2));
        kw3 = min(kw3, key_of(cp.w3));
        kw4 = min(kw4, key_of(cp.w4));
        kmu = max(kmu, key_of(cp.mach2));
        bad |= cp.bad;
    }
    __shared__ unsigned long long red[NTHR / 32][NKEY];
    for (int o = 16; o > 0; o >>= 1) {
        kw1 = min(kw1, __shfl_xor_sync(0xffffffffu, kw1, o));
        kw2 = min(kw2, __shfl_xor_sync(0xffffffffu, kw2, o));
        kw3 = min(kw3, __shfl_xor_sync(0xffffffffu, kw3, o));
        kw4 = min(kw4, __shfl_xor_sync(0xffffffffu, kw4, o));
        kmu = max(kmu, __shfl_xor_sync(0xffffffffu, kmu, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w][0] = kw1; red[w][1] = kw2; red[w][2] = kw3; red[w][3] = kw4; red[w][4] = kmu; red[w][5] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int v = 1; v < NTHR / 32; ++v) {
            kw1 = min(kw1, red[v][0]); kw2 = min(kw2, red[v][1]); kw3 = min(kw3, red[v][2]);
            kw4 = min(kw4, red[v][3]); kmu = max(kmu, red[v][4]); bad |= (unsigned int)red[v][5];
        }
        unsigned long long* row = partials + (size_t)k * NKEY;
        row[0] = kw1; row[1] = kw2; row[2] = kw3; row[3] = kw4; row[4] = kmu; row[5] = bad;
    }
}

// One block: combine the npz rows written by this call (every row is
// rewritten before it is read, so nothing carries over between calls) into
// DT=SF*MIN(...) and UMACH=SQRT(MAX(...)) (3dmhdsub.f:761, 866-873).
__global__ void __launch_bounds__(NTHR) k_cfl_combine(const unsigned long long* partials, int npz, int lmag,
                                                        double sf, double* out)
{
    unsigned long long kw[4] = {~0ull, ~0ull, ~0ull, ~0ull}, kmu = 0ull, bad = 0ull;
    for (int k = threadIdx.x; k < npz; k += NTHR) {
        const unsigned long long* row = partials + (size_t)k * NKEY;
        for (int v = 0; v < 4; ++v) kw[v] = min(kw[v], row[v]);
        kmu = max(kmu, row[4]);
        bad |= row[5];
    }
    __shared__ unsigned long long red[NTHR][NKEY];
    for (int v = 0; v < 4; ++v) red[threadIdx.x][v] = kw[v];
    red[threadIdx.x][4] = kmu;
    red[threadIdx.x][5] = bad;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int t = 1; t < NTHR; ++t) {
            for (int v = 0; v < 4; ++v) kw[v] = min(kw[v], red[t][v]);
            kmu = max(kmu, red[t][4]);
            bad |= red[t][5];
        }
        double w = of_key(kw[0]);
        const double w2 = of_key(kw[1]), w3 = of_key(kw[2]), w4 = of_key(kw[3]);
        w = w2 < w ? w2 : w;
        w = w3 < w ? w3 : w;
        if (lmag) w = w4 < w ? w4 : w;
        out[0] = sf * w;
        out[1] = sqrt(of_key(kmu));
        out[2] = bad ? 1.0 : 0.0;
    }
}

}  // namespace noalloc
}  // namespace mhd3d

using namespace mhd3d;

extern "C" int mhd3d_cfl_noalloc(const mhd3d_params* p,
                                 const double* ru, const double* rv, const double* rw, const double* tt,
                                 const double* ro, const double* bx, const double* by, const double* bz,
                                 const double* ddx, const double* ddy, const double* ddz, const double* rkapa,
                                 double* out, void* stream)
{
    if (!p || !ru || !rv || !rw || !tt || !ro || !ddx || !ddy || !ddz || !rkapa || !out) return MHD3D_ERR_ARG;
    if (p->lmag && (!bx || !by || !bz)) return MHD3D_ERR_ARG;
    if (p->npx < 2 || p->npy < 2 || p->npz < 1) return MHD3D_ERR_ARG;
    if (p->npz > MHD3D_NOALLOC_MAX_PLANES) return MHD3D_ERR_ARG;   // the scratch holds one row per plane
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MHD3D_ERR_NO_DEVICE;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    void* partials = nullptr;
    int st = noalloc::partials_address(dev, cs, &partials);
    if (st) return st;
    Scalars s{};
    s.gamma = p->gamma;
    s.ogamma = 1.0 / p->gamma;
    s.obeta = p->obeta;
    s.repr = p->repr;
    s.cv = p->cv;
    s.re = p->re;
    s.rm = p->rm;
    s.npx = p->npx;
    s.npy = p->npy;
    s.npz = p->npz;
    auto* part = static_cast<unsigned long long*>(partials);
    if (p->lmag)
        noalloc::k_cfl_planes<true><<<p->npz, noalloc::NTHR, 0, cs>>>(s, ru, rv, rw, tt, ro, bx, by, bz, ddx, ddy, ddz,
                                                                       rkapa, part);
    else
        noalloc::k_cfl_planes<false><<<p->npz, noalloc::NTHR, 0, cs>>>(s, ru, rv, rw, tt, ro, bx, by, bz, ddx, ddy,
                                                                        ddz, rkapa, part);
    if (cudaGetLastError() != cudaSuccess) return MHD3D_ERR_CUDA;
    noalloc::k_cfl_combine<<<1, noalloc::NTHR, 0, cs>>>(part, p->npz, p->lmag, p->sf, out);
    if (cudaGetLastError() != cudaSuccess) return MHD3D_ERR_CUDA;
    return MHD3D_OK;
}
