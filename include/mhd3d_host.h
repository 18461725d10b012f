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

/*
 * The reference driver's dump and restart files (3dmhd.f:284-363 restart,
 * 505-524 and 912-1009 dumps), for hosts that are not the Fortran program.
 *
 * mhd3d_host_par1: the 96-value PAR1 record: IPAR(1:32) as reals (ipar15 =
 * NCASE, NCASEP, NTOTAL, NSTEP0, NSTART; the rest from the config, NPE,
 * NPEY and NIT) and PAR(1:64) from the config, with PAR1(63)=DT and
 * PAR1(64), PAR1(65) as the driver sets them (TIMT, 0 at the last step,
 * else TIMI, TIMC).
 *
 * mhd3d_host_write_dump: dump number ndump (0-based, the driver's NDUMP0)
 * of a single-domain run: FOUT.dat0.0000 records nf*ndump+1.. (interior of
 * each field, REAL*8, direct access without record markers), FOUT.par
 * record ndump+1 (PAR1), and the dump's seven 80-character records of
 * FOUT.lis.  Fields are Fortran (NPX+2, NPY+2, NPZ+2) arrays.
 *
 * mhd3d_host_read_dump: restart from dump nstart (the driver's NSTART,
 * 1-based) written by a run with npey x npez ranks (FINP.dat0.NNNN per
 * rank): checks the sizes against FINP.par as the driver does, returns the
 * PAR1 record (TIMI = PAR1(64)+PAR1(65)) and the global fields with the
 * periodic halos filled; z ghost planes take the wall planes' values.
 */
void mhd3d_host_par1(const mhd3d_run_config* c, const int32_t ipar15[5], int32_t npe, int32_t npey, int32_t nit,
                     double dt, double par64, double par65, double par1[96]);
int mhd3d_host_write_dump(const char* fout, int32_t ndump, const double par1[96], int32_t npx, int32_t npy,
                          int32_t npz, int32_t lmag, const double* ru, const double* rv, const double* rw,
                          const double* tt, const double* ro, const double* bx, const double* by, const double* bz,
                          double timt, double timc, double umach, double dt);
int mhd3d_host_read_dump(const char* finp, int32_t nstart, int32_t npey, int32_t npez, int32_t lmag, int32_t npx,
                         int32_t npy, int32_t npz, double par1[96], double* ru, double* rv, double* rw, double* tt,
                         double* ro, double* bx, double* by, double* bz);

#ifdef __cplusplus
}
#endif

#endif
