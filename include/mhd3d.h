/*
 * mhd3d.h -- C-ABI of the B200 time-step library for 3dmhd.
 *
 * This library replaces the reference's per-step call sequence
 *
 *     CALL STEP            (3dmhd.f:912 -> 3dmhdsub.f:687-1176)
 *       = CFL/Mach reduction (3dmhdsub.f:741-873)
 *       + 3 x { FLUXES (1178-2637); RK3 axpy; BCON (2639-2958);
 *               COMMUNICATE/COMM_MPI (2980-3141) }
 *
 * with one handle that keeps the prognostic state resident in GPU memory.
 * The reference has no plugin API: STEP takes no arguments and exchanges
 * everything through COMMON blocks (3dmhd.f:51-75).  The entry points below
 * take those COMMON values explicitly, as plain pointers and sizes, so that
 * a Fortran host can bind them with ISO_C_BINDING (see
 * rast-3dmhd_b200/fortran/mhd3d_gpu.f90) and a C, C++ or Python host can
 * bind them directly.
 *
 * Array conventions (all arrays are host memory, Fortran column-major):
 *   - a 3-D field is REAL*8 (NX,NY,NZ) with NX=NPX+2, NY=NPY+2, NZ=NPZ+2,
 *     i.e. the single-domain form of the reference's local arrays
 *     (3dmhdparam.f:15-19 with NPEY=NPEZ=1, IX=IY=ILAP=2): one periodic
 *     halo cell on each side in x and y, and one z ghost plane above the top
 *     wall (K=1) and below the bottom wall (K=NZ).  The walls are the planes
 *     K=2 and K=NZ-1.
 *   - 1-D metric arrays have the lengths of COMMON/AJACOBI (3dmhd.f:36-38):
 *     NX for x, NY for y, NZ for z and for RKAPA/DKAPA.
 *
 * Semantics follow the reference run with NPEZ>=2 (one-sided wall
 * stencils at both walls: 3dmhdsub.f:1120-1126, 1391-1392, 1511-1513).
 *
 * Status codes: every entry point returns 0 on success, else one of the
 * MHD3D_ERR_* codes.  Nothing crosses the ABI as an exception and nothing
 * calls exit().  A handle is not thread-safe: one host thread per handle.
 * Calls are synchronous at the ABI edge unless stated otherwise.
 */
#ifndef MHD3D_H
#define MHD3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MHD3D_OK               0
#define MHD3D_ERR_ARG          1  /* bad argument or configuration the path does not support */
#define MHD3D_ERR_CUDA         2  /* a CUDA runtime call failed */
#define MHD3D_ERR_NONFINITE    3  /* NaN or Inf met by the CFL reduction */
#define MHD3D_ERR_DT_SMALL     4  /* DT < 1e-8: the reference driver's emergency stop (3dmhd.f:924) */
#define MHD3D_ERR_NO_DEVICE    5  /* no usable CUDA device */
#define MHD3D_ERR_TIMEOUT      6  /* a bounded device-side wait gave up */
#define MHD3D_ERR_NOMEM        7  /* device allocation failed */

/* Arithmetic modes. */
#define MHD3D_MODE_EXACT 0   /* FP64, reference operation order, no FMA
                                contraction: bit-equal to the CPU restatement
                                (+0 == -0) */
#define MHD3D_MODE_FAST  1   /* FP64, FMA contraction and pre-multiplied metric
                                products; within 1e-11 of EXACT after 10 steps */
#define MHD3D_MODE_FP32  2   /* FP32 state held as perturbations from FP64
                                background profiles (the horizontal means of
                                TT, RO, BX, BY, BZ at upload), FP32 arithmetic,
                                FP64 metrics and CFL reduction.  No counterpart
                                in the reference; its per-field error against
                                the FP64 path is measured by the tests.
                                mhd3d_bcon is not available in this mode. */

/*
 * Scalars of the COMMON blocks the step reads.  The host fills them exactly
 * as the reference main program does (3dmhd.f:105-240), i.e. holding the
 * float-rounded values of the REAL(4) literals (C13=1.0E00/3.0E00 etc.).
 * They are never re-derived inside the library.
 */
typedef struct mhd3d_params {
    int32_t npx, npy, npz;      /* NPX,NPY,NPZ (3dmhdparam.f:13)                 */
    int32_t lmag, lrot;         /* LMAG, LROT (3dmhdparam.f:8)                    */
    int32_t izcon, itcon, ibcon;/* IZC, ITC, IBC (COMMON/BCT, 3dmhdparam.f:27)   */
    int32_t mode;               /* MHD3D_MODE_EXACT, _FAST or _FP32               */
    int32_t reserved0;
    /* COMMON/GRID (DD is a STEP-local scratch there and is not passed) */
    double c13, c23, c43;
    double hx, h2x, hy, h2y, hz, h2z;
    /* COMMON/RUNGKU */
    double gam1, gam2, gam3, zeta1, zeta2;
    /* COMMON/CPAR */
    double cv, ocv, ore, re, repr, theta, grav, gamma, sf;
    /* COMMON/CROT */
    double omx, omz;
    /* COMMON/CMAG */
    double orm, rm, obeta;
    /* COMMON/CPEN, COMMON/CPER: bottom temperature and the upper-boundary
       plume (used only when TP != 0 and ITC is 0 or 1, 3dmhdsub.f:2790-2826) */
    double tb, tp, tc, xp, yp, hh;
    /* COMMON/CTIM at the start of the run: TIMI (restart time), TIMC */
    double timi, timc;
    /* DT threshold of the driver's emergency stop, REAL(4) 1.0E-08 */
    double dtmin;
} mhd3d_params;

/*
 * Create a handle: validates the configuration, allocates the device state
 * (U, Z and stage buffers, 1-D metrics) on the current CUDA device and
 * copies the metric arrays.  Replaces the COMMON set-up the reference does
 * before its main loop (3dmhd.f:105-279).
 *
 * Unsupported configurations return MHD3D_ERR_ARG: IXCON/IYCON != 0
 * (FLUXES stops on those, 3dmhdsub.f:1262-1265), LREM, ID != 0, RLAX > 0,
 * ITCON = 2 (embedded heat loss), IZCON not in {0,1}.
 */
int mhd3d_create(const mhd3d_params* p,
                 const double* exx, const double* dxxdx, const double* d2xxdx2, const double* ddx,
                 const double* wyy, const double* dyydy, const double* d2yydy2, const double* ddy,
                 const double* zee, const double* dzzdz, const double* d2zzdz2, const double* ddz,
                 const double* rkapa, const double* dkapa,
                 void** handle);

/* Release every device resource of the handle. */
int mhd3d_destroy(void* handle);

/*
 * Upload the prognostic state from Fortran (NX,NY,NZ) arrays, in the order
 * of the reference's dump records RU,RV,RW,TT,RO[,BX,BY,BZ]
 * (3dmhd.f:941-962).  bx/by/bz may be NULL when lmag == 0.  The x/y halos
 * of the uploaded arrays are ignored (the library wraps periodically); the
 * z ghost planes K=1 and K=NZ are kept, as the reference keeps them.  The
 * arrays may be host or device memory (mhd3d_download likewise).
 */
int mhd3d_upload(void* handle,
                 const double* ru, const double* rv, const double* rw,
                 const double* tt, const double* ro,
                 const double* bx, const double* by, const double* bz);

/*
 * Download the state into Fortran (NX,NY,NZ) arrays, halos filled as
 * COMMUNICATE leaves them (periodic copies, 3dmhdsub.f:3128-3138) and the
 * z ghost planes as the reference leaves them.  Call before every dump.
 */
int mhd3d_download(void* handle,
                   double* ru, double* rv, double* rw,
                   double* tt, double* ro,
                   double* bx, double* by, double* bz);

/*
 * Advance nsteps full RK3 steps: each is one CALL STEP (3dmhdsub.f:687).
 * On return: dt = DT of the last step, timc/timt = COMMON/CTIM after it,
 * umach = max Mach number (COMMON/TRACE), nit = COMMON/ITER NIT.
 * Any output pointer may be NULL.  Steps stop early, with the step that
 * produced it completed, when DT < dtmin (MHD3D_ERR_DT_SMALL, the
 * reference's GOTO 5010 at 3dmhd.f:924) or when the CFL reduction meets
 * a non-finite value (MHD3D_ERR_NONFINITE).
 */
int mhd3d_step(void* handle, int32_t nsteps,
               double* dt, double* timc, double* timt, double* umach, int32_t* nit);

/*
 * Test-only entry points with the semantics of the Fortran routines.
 *
 * mhd3d_fluxes: evaluate FLUXES on the current state without changing it
 * and copy the right-hand sides to Fortran (NX,NY,NZ) arrays: FU,FV,FW,FR,FT
 * and, with LMAG, the induction terms WW1..WW3 (3dmhdsub.f:2129-2634).
 * Only interior cells (I=2..NX-1, J=2..NY-1, K=2..NZ-1) are written.
 * Values on the wall planes that BCON overwrites (FU,FV,FW,FT and WW3 at
 * K=2 and K=NZ-1) are written as 0; the reference computes them from the
 * ghost planes and then discards them.
 */
int mhd3d_fluxes(void* handle,
                 double* fu, double* fv, double* fw, double* fr, double* ft,
                 double* ww1, double* ww2, double* ww3);

/* CFL/Mach reduction of STEP (3dmhdsub.f:741-873) on the current state. */
int mhd3d_cfl(void* handle, double* dt, double* umach);

/* BCON (3dmhdsub.f:2639-2958) applied to the current state in place. */
int mhd3d_bcon(void* handle);

/*
 * Horizontally averaged profiles of the current state: the averages the
 * reference forms with HORIZONTAL_MEAN (3dmhdsub.f:3143-3223: the sum over
 * the interior I=2..NX-1, J=2..NY-1 divided by FLOAT(NPX*NPY)) for its flux
 * diagnostics (3dmhdsub.f:1519-1528, 1651-1676), computed on the device in
 * FP64.  out holds MHD3D_NPROF rows of NPZ values, row r at
 * out[r*NPZ + (K-2)] for the interior planes K=2..NZ-1.  With u=RU/RO etc.:
 */
#define MHD3D_NPROF        7
#define MHD3D_PROF_RHO     0  /* <RO>                                                  */
#define MHD3D_PROF_T       1  /* <TT>, TTM (1523)                                      */
#define MHD3D_PROF_KE      2  /* <0.5*RO*|u|**2>                                       */
#define MHD3D_PROF_ENTH    3  /* <2.5*RO*TT>, c_p=2.5 as the reference takes it (1654) */
#define MHD3D_PROF_FCONV   4  /* <-RW*(2.5*(TT-TTM)+0.5*|u|**2)>, FCONM (1653-1661)    */
#define MHD3D_PROF_FRAD    5  /* (TTM(K+1)-TTM(K-1))*HZ*DZZDZ*RKAPA/REPR, one-sided at
                                 K=2 and K=NZ-1, FRADM (1663-1676)                    */
#define MHD3D_PROF_ME      6  /* <0.5*|B|**2> (0 without LMAG; no counterpart in the
                                 reference)                                           */
int mhd3d_profiles(void* handle, double* out);

/*
 * Stream control and asynchronous stepping (no counterpart in the
 * reference; they let a host overlap its own work with the step, capture
 * steps in a CUDA graph and time them on its own stream).
 *
 * mhd3d_set_stream: run all later work of the handle on stream (a
 *   cudaStream_t passed as void*); NULL returns to the handle's own stream.
 * mhd3d_step_async: enqueue nsteps steps and return without waiting.
 * mhd3d_sync: wait for enqueued steps and report as mhd3d_step does.
 */
int mhd3d_set_stream(void* handle, void* stream);
int mhd3d_step_async(void* handle, int32_t nsteps);
int mhd3d_sync(void* handle, double* dt, double* timc, double* timt, double* umach, int32_t* nit);

/*
 * Kernel timing for diagnostics: with enable != 0 every RK3 stage kernel
 * is bracketed by CUDA events on the stream it runs on.  mhd3d_profile_read
 * (after mhd3d_sync) returns the summed milliseconds and launch counts of
 * stages 1, 2, 3 since the last read, then clears them.
 */
/*
 * Test entry point (no counterpart in the reference, whose only run-time
 * check is DT<1e-8, 3dmhd.f:924): the poll limit of the first wait of every
 * CTA of the FP64 stage kernels on its shared-memory ring (default and
 * maximum 2^22 polls).  With 0 that wait gives up at once; the CTA then
 * waits, at the normal limit, for every copy it has in flight, records
 * MHD3D_ERR_TIMEOUT and returns, so the next mhd3d_step reports the
 * timeout the way a real expiry would.  Returns MHD3D_ERR_ARG for an FP32
 * handle or a negative limit.
 */
int mhd3d_set_wait_limit(void* handle, int64_t polls);
int mhd3d_profile(void* handle, int32_t enable);
int mhd3d_profile_read(void* handle, double stage_ms[3], int32_t launches[3]);

/*
 * CFL/Mach reduction that allocates nothing.  It has no counterpart in the
 * reference: it serves hosts that cannot call cudaMalloc (device arrays
 * declared statically by a Fortran or C code, a framework allocator that
 * owns the device heap, a hard device-memory cap) and already hold the
 * state in device memory.
 *
 * Inputs are device pointers: the fields as Fortran (NX,NY,NZ) arrays
 * (bx/by/bz only with lmag; NULL otherwise), and DDX(NX), DDY(NY), DDZ(NZ),
 * RKAPA(NZ).  out is a device pointer to 3 doubles: DT = SF*MIN(limits),
 * UMACH, and 1.0 if any limit was not finite (else 0.0), equal bit for bit
 * to what mhd3d_cfl returns in the reference-rounding mode.  The work is
 * enqueued on stream (a cudaStream_t, NULL for the default stream) and the
 * call returns without waiting.
 *
 * Scratch: one file-scope __device__ array of MHD3D_NOALLOC_MAX_PLANES x 6
 * 64-bit words (192 KiB), held by every GPU that loads the library until
 * the process exits; npz above MHD3D_NOALLOC_MAX_PLANES returns
 * MHD3D_ERR_ARG.  Each call made outside a stream capture looks the array's
 * device address up on the current device (so a cudaDeviceReset between
 * calls is harmless); a call made while its stream is being captured reuses
 * the address found by the last such call on that device, so make the first
 * call on a device before any stream capture.  All calls share the array
 * and keep the last call's contents: calls that can overlap on the GPU
 * (different streams, or devices sharing a context) race and must be
 * ordered by the caller.
 */
#define MHD3D_NOALLOC_MAX_PLANES 4096
int mhd3d_cfl_noalloc(const mhd3d_params* p,
                      const double* ru, const double* rv, const double* rw, const double* tt,
                      const double* ro, const double* bx, const double* by, const double* bz,
                      const double* ddx, const double* ddy, const double* ddz, const double* rkapa,
                      double* out, void* stream);

/* Version string of the library. */
/*
 * Batched ensemble (no counterpart in the reference): nmembers independent
 * FP32 grids of any sizes (params[i].mode must be MHD3D_MODE_FP32; LMAG and
 * LROT equal across members), stepped together.  Each RK3 stage of all
 * members is one persistent launch over a work table (member, tile, z
 * chunk), largest members first; a step is one CUDA graph.  grids holds
 * 14*nmembers pointers, the mhd3d_create metric arrays of each member in
 * turn.  Members keep their own DT, TIMT, NIT and stop status.
 *
 * mhd3d_ensemble_member returns member i's handle for mhd3d_upload,
 * mhd3d_download, mhd3d_profiles and mhd3d_cfl; it stays owned by the
 * ensemble (never pass it to mhd3d_destroy).  mhd3d_ensemble_step enqueues
 * nsteps steps of every member without waiting; mhd3d_ensemble_sync waits
 * and returns per-member DT, TIMT, NIT and status (arrays of nmembers; any
 * may be NULL) and the first non-zero status.  mhd3d_ensemble_tune times
 * `steps` steps for each tile shape (32x2, 32x4, 32x8 columns; separate
 * kernel instances, each member's TMA boxes re-made for it), z-chunk length
 * in {4,6,8,12,16,24,32,48,64} and number of persistent CTAs per SM (8, 12
 * or 16 warps an SM where the tile allows) on the current state, restores
 * the state, and keeps the fastest; mhd3d_ensemble_tile reports the tile
 * shape in use (32x4 until a tune), mhd3d_ensemble_set_tile sets its rows
 * (2, 4 or 8; MHD3D_ERR_ARG for others or rows a member's arrays cannot
 * hold).  Every tile shape gives the same bits.
 */
int mhd3d_ensemble_create(int32_t nmembers, const mhd3d_params* params, const double* const* grids, void** ens);
int mhd3d_ensemble_destroy(void* ens);
int mhd3d_ensemble_member(void* ens, int32_t i, void** handle);
int mhd3d_ensemble_step(void* ens, int32_t nsteps);
int mhd3d_ensemble_sync(void* ens, double* dt, double* timt, int32_t* nit, int32_t* status);
int mhd3d_ensemble_tune(void* ens, int32_t steps, int32_t* zlen, int32_t* ctas_per_sm, double* ms_per_step);
int mhd3d_ensemble_tile(void* ens, int32_t* tile_x, int32_t* tile_y);
int mhd3d_ensemble_set_tile(void* ens, int32_t tile_y);
/* enqueue the ensemble's work on a caller's cudaStream_t (NULL: its own) */
int mhd3d_ensemble_set_stream(void* ens, void* stream);

/*
 * Learned-closure building blocks (no counterpart in the reference).  All
 * arrays are device pointers; activations are channels-last BF16
 * [nz][ny][nx][C] (periodic in x and y, zero outside in z), weights BF16
 * [cout][27*cin] with k = tap*cin + ci, tap = (dx+1) + 3*(dy+1) + 9*(dz+1).
 * Any nx >= 1 (x segments of 128 voxels; a segment that runs past the row's
 * end, or a row shorter than 128, wraps periodically and stores only its own
 * voxels; nx a multiple of 128 takes the TMA loader); every array is 16-byte
 * aligned.
 * Supported (cin, cout): (16,32), (32,32),
 * (32,16).  Work is enqueued on stream; err (device int) is set non-zero if
 * a bounded wait of the tensor-core pipeline gave up.
 *
 * mhd3d_conv3d: y = act(conv(x, w) + bias), act = ReLU if relu; with mask
 * (channels-last, cout channels) the output is zeroed where mask <= 0 (the
 * ReLU derivative in the input-gradient pass).  y (BF16) and/or yf (FP32).
 * mhd3d_conv3d_wtranspose: w -> wt, the weights of the input-gradient
 * convolution (cin and cout swapped, taps mirrored).
 * mhd3d_conv3d_wgrad: dw[cout][27*cin] += sum over voxels of dy (x) x
 * shifted, db[cout] += sum of dy (FP32, accumulating), on the tensor cores
 * with FP32 accumulation; per-CTA partial sums go to a workspace taken from
 * the stream-ordered allocator (cudaMallocAsync on stream, freed after use)
 * and are added in a fixed order, so repeated calls give the same bits.  If
 * a bounded device-side wait gives up, dw and db receive NaN.
 */
int mhd3d_conv3d(int32_t cin, int32_t cout, const void* x, const void* w, const float* bias, const void* mask,
                 int32_t relu, void* y, float* yf, int32_t nx, int32_t ny, int32_t nz, int32_t* err, void* stream);
int mhd3d_conv3d_wtranspose(int32_t cin, int32_t cout, const void* w, void* wt, void* stream);
int mhd3d_conv3d_wgrad(int32_t cin, int32_t cout, const void* x, const void* dy, float* dw, float* db, int32_t nx,
                       int32_t ny, int32_t nz, void* stream);

/*
 * Learned closure on an FP32 handle (any NPX).
 * mhd3d_closure_set attaches a trained network (weights BF16 [cout][27*cin]:
 * w1 32x432, w2 32x864, w3 16x864; biases FP32 32, 32, 16; in_scale[8] the
 * feature scales; out_scale[12] the target scales; host or device pointers,
 * copied): every step then evaluates it once before stage 1 and adds its
 * tendencies (RU_i -= d_j tau_ij, TT -= (1/RO) d_j q_j, B += curl eps) to the
 * three stages.  When an output is not finite, or the stress trace exceeds
 * trip x RO*TT, that step runs without it (the plain coarse method).  A
 * NULL w1 detaches.  mhd3d_closure_status: steps that fell back, evaluations,
 * and the tensor-core pipeline's error flag.
 *
 * Training support (device pointers, enqueued on stream):
 * mhd3d_coarsen: box filter of a handle's state by fac: coarse state in
 * Fortran (NX,NY,NZ) arrays (8 or 5 fields, halos periodic, ghost planes =
 * walls) and the subgrid targets [k][j][i][12] (tau_xx,yy,zz,xy,xz,yz, q_x,y,z,
 * eps_x,y,z).  mhd3d_closure_features: network input [k][j][i][16] BF16 of a
 * handle's state (u, v, w, TT-<TT>, RO-<RO>, BX, BY-<BY>, BZ times in_scale;
 * means: 3*NPZ doubles of scratch).  mhd3d_closure_loss: adds the mean-square
 * error of pred [v][16] against target [v][12] to *loss and writes its
 * gradient dy [v][16] BF16.  mhd3d_adam: one Adam step on FP32 parameters
 * (step number t), optional BF16 copy.  mhd3d_closure_tendency: the
 * tendencies of pred (16-byte aligned) for a handle's state, out[f][k][j][i]
 * (f = RU, RV, RW, TT, BX, BY, BZ); *flag set when the indicator trips.
 */
int mhd3d_closure_set(void* handle, const void* w1, const float* b1, const void* w2, const float* b2, const void* w3,
                      const float* b3, const float* in_scale, const float* out_scale, float trip);
int mhd3d_closure_status(void* handle, int32_t* trips, int32_t* evals, int32_t* err);
/*
 * A per-plane bias tendency of the closure (no counterpart in the
 * reference): bias[f*NPZ + k] for the fields RU, RV, RW, TT, BX, BY, BZ
 * (f = 0..6) and the interior planes k = 0..NPZ-1 (zero on the walls, which
 * take no tendency), a host or device array of 7*NPZ floats, copied.  With a
 * network attached it is added to the network's tendencies on every step
 * that does not fall back to the plain coarse method (a step that falls back
 * takes neither).  Without one, every step adds the bias alone: it is
 * broadcast once into a tendency array of 7 floats per cell that the stage
 * kernel reads, with no per-step evaluation.  Meant for the horizontally
 * uniform part of the coarse scheme's residual: the mismatch between a
 * box-filtered state and the coarse grid's own discrete balance.  NULL
 * removes it; a call that fails leaves the handle without a bias.  FP32
 * handles only.
 */
int mhd3d_closure_set_bias(void* handle, const float* bias);
int mhd3d_coarsen(void* fine, int32_t fac, double* cstate, float* targets, void* stream);
int mhd3d_closure_features(void* handle, const float* in_scale, void* feat, double* means, void* stream);
int mhd3d_closure_loss(const float* pred, const float* target, int64_t nvox, void* dy, double* loss, void* stream);
int mhd3d_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
               int32_t t, void* p_bf16, void* stream);
int mhd3d_closure_tendency(void* handle, const float* pred, const float* out_scale, float* out, int32_t* flag,
                           float trip, void* stream);

/*
 * Training the closure on tendencies (no counterpart in the reference): a
 * target given as the 7 tendencies a coarse run misses (for instance the
 * filtered fine run's rate of change minus the coarse scheme's right-hand
 * sides) is fitted through the same stress, heat-flux and EMF outputs.
 * mhd3d_closure_tendency_loss: loss += sum_f weight[f] * sum (tend -
 * target)^2 / (7 nvox) over arrays [7][nvox] (device), and g = d loss /
 * d tend.  mhd3d_closure_tendency_adjoint: the transpose of
 * mhd3d_closure_tendency's map for the handle's state, g [7][nvox] ->
 * dpred [nvox][16] BF16 (channels 12..15 zero), the gradient to feed the
 * network's last layer.
 */
int mhd3d_closure_tendency_loss(const float* tend, const float* target, const float* weight, int64_t nvox, float* g,
                                double* loss, void* stream);
int mhd3d_closure_tendency_adjoint(void* handle, const float* g, const float* out_scale, void* dpred, void* stream);

const char* mhd3d_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MHD3D_H */
