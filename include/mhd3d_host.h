/*
 * mhd3d_host.h -- host-side mirror of the reference driver's initialisation
 * (3dmhd.f:105-496, 3dmhdset.f, 3dmhdsub.f:17-657 and 3982-4413), for hosts
 * that are not the Fortran program: C, C++ and the Python test/bench code.
 *
 * The Fortran driver keeps doing this itself and only calls mhd3d.h.  This
 * library produces exactly what the driver holds before its first CALL STEP:
 * the COMMON scalars (mhd3d_params), the COMMON/AJACOBI metric arrays and
 * the prognostic fields in Fortran (NX,NY,NZ) layout after COMMUNICATE.
 */
#ifndef MHD3D_HOST_H
#define MHD3D_HOST_H

#include <stdint.h>
#include "mhd3d.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Grid maps of MKGRID (3dmhdsub.f:17-175) plus one project map. */
#define MHD3D_GRID_UNIFORM   0   /* NGRID=0 */
#define MHD3D_GRID_ARCTAN    1   /* NGRID=1 (XX1..ZZ2) */
#define MHD3D_GRID_DIP       2   /* NGRID=2 (XA..ZD) */
#define MHD3D_GRID_TANH_Z    3   /* uniform x,y; z = ZMAX*(1 - tanh(S(1-s))/tanh(S)), points clustered at the top */

/*
 * Run configuration: the values the reference takes from 3dmhdparam.f
 * PARAMETERs and from SETUP (3dmhdset.f:36-146).  Values the reference
 * writes as REAL(4) literals (GAMMA=5.00E00/3.00E00, SFF=0.4E00, ...) must
 * be given float-rounded; mhd3d_host_default_config does that.
 */
typedef struct mhd3d_run_config {
    int32_t npx, npy, npz;
    int32_t lmag, lrot;
    int32_t izcon, itcon, ibcon;
    int32_t ngrid;
    int32_t ntube;          /* IPAR(16): TUBE model, 0 (no field) or 4 (uniform BY layer) */
    int32_t seed;           /* IDUM = -seed for RAN2 (3dmhdsub.f:599) */
    int32_t mode;           /* MHD3D_MODE_* copied into mhd3d_params */
    double xmax, ymax, zmax;
    double zstretch;        /* S of MHD3D_GRID_TANH_Z */
    double xx1, xx2, yy1, yy2, zz1, zz2;          /* NGRID=1 */
    double xa, xb, xc, xd, ya, yb, yc, yd, za, zb, zc, zd; /* NGRID=2 */
    double re, pr, theta, grav, ry, ang, rm, beta;
    double pzp, sigma, polys;
    double tp, tc, xp, yp, hh;
    double ampt, ampb, bfh, bzp;
    double zcent, rmax, cmt, atube;  /* PAR(35..38) for TUBE model 4 */
    double gamma, sff;
    double timi;
} mhd3d_run_config;

/* Fill a configuration with the values of 3dmhdset.f:36-146 and
 * 3dmhdparam.f (float-rounded where the reference uses REAL(4) literals),
 * resized to npx x npy x npz with one z ghost plane on each side. */
void mhd3d_host_default_config(mhd3d_run_config* c, int32_t npx, int32_t npy, int32_t npz);

/*
 * Rotating MHD polytrope set up from dimensionless numbers (the mapping is
 * the project convention: every number evaluated at mid-depth).
 *   contrast = rho_bottom/rho_top, m = polytropic index -> THETA, GRAV
 *   Ra, Pr (physical Prandtl = c_p*PR), Ta = (OMZ*RE*rho_mid)^2, Pm = RM/(RE*rho_mid),
 *   beta = plasma beta at the top (BETA).
 * Box 4:4:1, x,y periodic, tanh z stretch S, stress-free walls, fixed
 * flux bottom (IZCON=1), fixed T top (ITCON=0), uniform BY (TUBE model 4),
 * TP=0, SFF=0.4, perturbation amplitude ampt.
 */
void mhd3d_host_convection_config(mhd3d_run_config* c, int32_t npx, int32_t npy, int32_t npz,
                                  double ra, double ta, double pr_phys, double pm, double contrast,
                                  double m, double beta, double stretch, double ampt, int32_t seed);

/* COMMON scalars as 3dmhd.f:105-240 derives them; TB from STATIC. */
int mhd3d_host_params(const mhd3d_run_config* c, mhd3d_params* p);

/* XJACOBI/YJACOBI/ZJACOBI (3dmhdsub.f:177-353) for a single domain with
 * the NPEZ>=2 ghost conventions, and RKAPA/DKAPA (3dmhd.f:266-279).
 * Lengths: x arrays NPX+2, y arrays NPY+2, z arrays NPZ+2. */
int mhd3d_host_grid(const mhd3d_run_config* c,
                    double* exx, double* dxxdx, double* d2xxdx2, double* ddx,
                    double* wyy, double* dyydy, double* d2yydy2, double* ddy,
                    double* zee, double* dzzdz, double* d2zzdz2, double* ddz,
                    double* rkapa, double* dkapa);

/* STATIC (3dmhdsub.f:355-657) with TUBE (3982-4413, models 0 and 4) and
 * the RAN2 temperature perturbation, then COMMUNICATE: the state at
 * 3dmhd.f:365.  Fields are Fortran (NPX+2,NPY+2,NPZ+2); bx/by/bz may be
 * NULL when lmag == 0.  zee must come from mhd3d_host_grid. */
int mhd3d_host_static(const mhd3d_run_config* c, const double* zee,
                      double* ru, double* rv, double* rw, double* tt, double* ro,
                      double* bx, double* by, double* bz);

/* RAN2 (3dmhdsub.f:3377-3410): one deviate; state is idum, iy, ir[97]. */
double mhd3d_host_ran2(int32_t* idum, int32_t* iy, int32_t* ir);

#ifdef __cplusplus
}
#endif

#endif
