/*
 * oracle3dmhd.c -- CPU restatement of the 3dmhd time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU path, loaded by the
 * tests, the smoke check and the CPU-baseline leg of the benchmark.
 *
 * What it restates (file:line of the reference, dsmithlasp/Rast-3dmhd):
 *   STEP        3dmhdsub.f:687-1176   CFL/Mach, 3 low-storage RK3 stages
 *   FLUXES      3dmhdsub.f:1249-1295, 1376-1506, 1583-1611, 1818-2634
 *               (continuity, pressure, advection, conduction, viscosity,
 *                heating, Coriolis, induction/Lorentz/Ohmic heating)
 *   BCON        3dmhdsub.f:2751-2955  stress-free impenetrable walls
 *   COMM_MPI    3dmhdsub.f:3031-3141  as a single-domain periodic wrap
 *
 * Every sweep keeps the reference's loop ranges, the order of its
 * floating-point operations and its intermediate roundings, so that the
 * result is the one gfortran -O2 produces (IEEE double, no FMA
 * contraction: build with -ffp-contract=off).  Scalars hold the
 * float-rounded values of the REAL(4) literals, as the host passes them.
 *
 * The domain is one block with the reference's NPEZ>=2 semantics: both
 * walls take their one-sided stencils (the NPEZ=1 build skips the bottom
 * ones through ELSE IF at 3dmhdsub.f:1120-1126, 1391-1392, 1511-1513).
 * The z ghost planes are kept and treated as the reference treats them:
 * never refreshed, and RO there is inverted by every FLUXES call
 * (3dmhdsub.f:1386-1391).
 *
 * Parity unpinned by the reference's own tests (it has none); pinned by
 * the translated reference build (oracle/make_ref.py) and the golden
 * fixtures it produced under tests/golden/.
 */
#include "oracle3dmhd.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct oracle3dmhd {
    mhd3d_params p;
    int nx, ny, nz;
    size_t n;
    /* COMMON/AJACOBI and CPEN 1-D arrays, 1-based (element 0 unused) */
    double *exx, *dxxdx, *d2xxdx2, *ddx;
    double *wyy, *dyydy, *d2yydy2, *ddy;
    double *zee, *dzzdz, *d2zzdz2, *ddz;
    double *rkapa, *dkapa;
    /* COMMON/BIG (3dmhd.f:51-56) */
    double *ru, *rv, *rw, *ro, *tt, *uu, *vv, *ww;
    double *fu, *fv, *fw, *fr, *ft;
    double *zru, *zrv, *zrw, *zro, *ztt;
    double *w1, *w2, *w3;
    double *bx, *by, *bz, *zbx, *zby, *zbz;
    /* COMMON/CTIM, ITER, TRACE */
    double dt, timt, timc, timi, umach;
    int nit;
};

#define NX (o->nx)
#define NY (o->ny)
#define NZ (o->nz)
/* Fortran A(I,J,K), 1-based, column-major */
#define IDX(i, j, k) ((size_t)((i) - 1) + (size_t)NX * ((size_t)((j) - 1) + (size_t)NY * (size_t)((k) - 1)))
#define A(a, i, j, k) (o->a[IDX(i, j, k)])

#ifdef _OPENMP
#define PAR_K _Pragma("omp parallel for schedule(static)")
#else
#define PAR_K
#endif

static double* vec1(const double* src, int n)
{
    double* v = (double*)calloc((size_t)n + 1, sizeof(double));
    if (src) memcpy(v + 1, src, (size_t)n * sizeof(double));
    return v;
}

oracle3dmhd* oracle_create(const mhd3d_params* p,
                           const double* exx, const double* dxxdx, const double* d2xxdx2, const double* ddx,
                           const double* wyy, const double* dyydy, const double* d2yydy2, const double* ddy,
                           const double* zee, const double* dzzdz, const double* d2zzdz2, const double* ddz,
                           const double* rkapa, const double* dkapa)
{
    oracle3dmhd* o = (oracle3dmhd*)calloc(1, sizeof(*o));
    o->p = *p;
    o->nx = p->npx + 2;
    o->ny = p->npy + 2;
    o->nz = p->npz + 2;
    o->n = (size_t)o->nx * o->ny * o->nz;
    o->exx = vec1(exx, o->nx);   o->dxxdx = vec1(dxxdx, o->nx);
    o->d2xxdx2 = vec1(d2xxdx2, o->nx); o->ddx = vec1(ddx, o->nx);
    o->wyy = vec1(wyy, o->ny);   o->dyydy = vec1(dyydy, o->ny);
    o->d2yydy2 = vec1(d2yydy2, o->ny); o->ddy = vec1(ddy, o->ny);
    o->zee = vec1(zee, o->nz);   o->dzzdz = vec1(dzzdz, o->nz);
    o->d2zzdz2 = vec1(d2zzdz2, o->nz); o->ddz = vec1(ddz, o->nz);
    o->rkapa = vec1(rkapa, o->nz); o->dkapa = vec1(dkapa, o->nz);
    double** arrs[] = {&o->ru, &o->rv, &o->rw, &o->ro, &o->tt, &o->uu, &o->vv, &o->ww,
                       &o->fu, &o->fv, &o->fw, &o->fr, &o->ft,
                       &o->zru, &o->zrv, &o->zrw, &o->zro, &o->ztt,
                       &o->w1, &o->w2, &o->w3,
                       &o->bx, &o->by, &o->bz, &o->zbx, &o->zby, &o->zbz};
    for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); ++a)
        *arrs[a] = (double*)calloc(o->n, sizeof(double));
    o->timi = p->timi;
    o->timc = p->timc;
    o->timt = 0.0; /* COMMON/CTIM TIMT is first assigned at the end of STEP */
    return o;
}

void oracle_destroy(oracle3dmhd* o)
{
    if (!o) return;
    double* arrs[] = {o->exx, o->dxxdx, o->d2xxdx2, o->ddx, o->wyy, o->dyydy, o->d2yydy2, o->ddy,
                      o->zee, o->dzzdz, o->d2zzdz2, o->ddz, o->rkapa, o->dkapa,
                      o->ru, o->rv, o->rw, o->ro, o->tt, o->uu, o->vv, o->ww,
                      o->fu, o->fv, o->fw, o->fr, o->ft, o->zru, o->zrv, o->zrw, o->zro, o->ztt,
                      o->w1, o->w2, o->w3, o->bx, o->by, o->bz, o->zbx, o->zby, o->zbz};
    for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); ++a) free(arrs[a]);
    free(o);
}

void oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* COMM_MPI (3dmhdsub.f:3031-3141) for NPEY=1: y periodic copy over all  */
/* I and K (3128-3129), then x periodic copy over all J and K (3137-3138).*/
/* Vertical ghost planes are not exchanged at the physical walls.        */
/* ------------------------------------------------------------------ */
static void wrap_field(oracle3dmhd* o, double* v)
{
    PAR_K
    for (int k = 1; k <= NZ; ++k) {
        for (int i = 1; i <= NX; ++i) {
            v[IDX(i, 1, k)] = v[IDX(i, NY - 1, k)];
            v[IDX(i, NY, k)] = v[IDX(i, 2, k)];
        }
        for (int j = 1; j <= NY; ++j) {
            v[IDX(1, j, k)] = v[IDX(NX - 1, j, k)];
            v[IDX(NX, j, k)] = v[IDX(2, j, k)];
        }
    }
}

/* COMMUNICATE (3dmhdsub.f:2980-3029): RU,RV,RW,TT,RO then BX,BY,BZ. */
static void communicate(oracle3dmhd* o)
{
    wrap_field(o, o->ru); wrap_field(o, o->rv); wrap_field(o, o->rw);
    wrap_field(o, o->tt); wrap_field(o, o->ro);
    if (o->p.lmag) { wrap_field(o, o->bx); wrap_field(o, o->by); wrap_field(o, o->bz); }
}

void oracle_set_state(oracle3dmhd* o, const double* ru, const double* rv, const double* rw,
                      const double* tt, const double* ro,
                      const double* bx, const double* by, const double* bz)
{
    size_t nb = o->n * sizeof(double);
    memcpy(o->ru, ru, nb); memcpy(o->rv, rv, nb); memcpy(o->rw, rw, nb);
    memcpy(o->tt, tt, nb); memcpy(o->ro, ro, nb);
    if (o->p.lmag) { memcpy(o->bx, bx, nb); memcpy(o->by, by, nb); memcpy(o->bz, bz, nb); }
    communicate(o);
}

void oracle_get_state(const oracle3dmhd* o, double* ru, double* rv, double* rw,
                      double* tt, double* ro, double* bx, double* by, double* bz)
{
    size_t nb = o->n * sizeof(double);
    if (ru) memcpy(ru, o->ru, nb);
    if (rv) memcpy(rv, o->rv, nb);
    if (rw) memcpy(rw, o->rw, nb);
    if (tt) memcpy(tt, o->tt, nb);
    if (ro) memcpy(ro, o->ro, nb);
    if (o->p.lmag) {
        if (bx) memcpy(bx, o->bx, nb);
        if (by) memcpy(by, o->by, nb);
        if (bz) memcpy(bz, o->bz, nb);
    }
}

/* ------------------------------------------------------------------ */
/* FLUXES                                                              */
/* ------------------------------------------------------------------ */
static void fluxes(oracle3dmhd* o)
{
    const mhd3d_params* P = &o->p;
    const double HX = P->hx, H2X = P->h2x, HY = P->hy, H2Y = P->h2y, HZ = P->hz, H2Z = P->h2z;
    const double C13 = P->c13, C43 = P->c43;
    const double OCV = P->ocv, ORE = P->ore, REPR = P->repr, GRAV = P->grav;
    const double *DXXDX = o->dxxdx, *D2XXDX2 = o->d2xxdx2;
    const double *DYYDY = o->dyydy, *D2YYDY2 = o->d2yydy2;
    const double *DZZDZ = o->dzzdz, *D2ZZDZ2 = o->d2zzdz2;
    const double *RKAPA = o->rkapa, *DKAPA = o->dkapa;

    /* 1249-1270: FR = -(d(RU)/dx + d(RV)/dy), horizontal part (loop 10) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy = HY * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fr, i, j, k) = (A(ru, i - 1, j, k) - A(ru, i + 1, j, k)) * HX * DXXDX[i];
                A(fr, i, j, k) = A(fr, i, j, k) - (A(rv, i, j + 1, k) - A(rv, i, j - 1, k)) * tmpy;
            }
        }
    /* 1272-1289: WW1 = d(RW)/dz, one-sided at both walls (loops 40,50,60) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz = HZ * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(w1, i, j, k) = (A(rw, i, j, k + 1) - A(rw, i, j, k - 1)) * tmpz;
    }
    {
        double tmpz = HZ * DZZDZ[2];
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(w1, i, j, 2) = (4.0 * A(rw, i, j, 3) - A(rw, i, j, 4)) * tmpz;
        tmpz = HZ * DZZDZ[NZ - 1];
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(w1, i, j, NZ - 1) = (A(rw, i, j, NZ - 3) - 4.0 * A(rw, i, j, NZ - 2)) * tmpz;
    }
    /* 1291-1295: FR = FR - WW1 (loop 70); 1376-1380: FW = GRAV*RO (loop 80) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(fr, i, j, k) = A(fr, i, j, k) - A(w1, i, j, k);
                A(fw, i, j, k) = GRAV * A(ro, i, j, k);
            }
    /* 1386-1391: WW1 = RO*TT (pressure) and RO <- 1/RO on the whole array (loop 90) */
    PAR_K
    for (int k = 1; k <= NZ; ++k)
        for (int j = 1; j <= NY; ++j)
            for (int i = 1; i <= NX; ++i) {
                A(w1, i, j, k) = A(ro, i, j, k) * A(tt, i, j, k);
                A(ro, i, j, k) = 1.0 / A(ro, i, j, k);
            }
    /* 1396-1404: pressure gradient (loop 120) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz = HZ * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy = HY * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fw, i, j, k) = A(fw, i, j, k) - (A(w1, i, j, k + 1) - A(w1, i, j, k - 1)) * tmpz;
                A(fv, i, j, k) = (A(w1, i, j - 1, k) - A(w1, i, j + 1, k)) * tmpy;
                A(fu, i, j, k) = (A(w1, i - 1, j, k) - A(w1, i + 1, j, k)) * HX * DXXDX[i];
            }
        }
    }
    /* 1411-1425: velocities on the whole array (loops 160,170,180) */
    PAR_K
    for (int k = 1; k <= NZ; ++k)
        for (int j = 1; j <= NY; ++j)
            for (int i = 1; i <= NX; ++i) {
                A(uu, i, j, k) = A(ru, i, j, k) * A(ro, i, j, k);
                A(vv, i, j, k) = A(rv, i, j, k) * A(ro, i, j, k);
                A(ww, i, j, k) = A(rw, i, j, k) * A(ro, i, j, k);
            }
    /* 1435-1482: momentum advection (loops 210, 280, 330) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz = HZ * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy = HY * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fu, i, j, k) = A(fu, i, j, k) - (A(ru, i + 1, j, k) * A(uu, i + 1, j, k)
                                                 - A(ru, i - 1, j, k) * A(uu, i - 1, j, k)) * HX * DXXDX[i];
                A(fu, i, j, k) = A(fu, i, j, k) - (A(ru, i, j + 1, k) * A(vv, i, j + 1, k)
                                                 - A(ru, i, j - 1, k) * A(vv, i, j - 1, k)) * tmpy;
                A(fu, i, j, k) = A(fu, i, j, k) - (A(ru, i, j, k + 1) * A(ww, i, j, k + 1)
                                                 - A(ru, i, j, k - 1) * A(ww, i, j, k - 1)) * tmpz;
            }
        }
    }
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz = HZ * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy = HY * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fv, i, j, k) = A(fv, i, j, k) - (A(rv, i + 1, j, k) * A(uu, i + 1, j, k)
                                                 - A(rv, i - 1, j, k) * A(uu, i - 1, j, k)) * HX * DXXDX[i];
                A(fv, i, j, k) = A(fv, i, j, k) - (A(rv, i, j + 1, k) * A(vv, i, j + 1, k)
                                                 - A(rv, i, j - 1, k) * A(vv, i, j - 1, k)) * tmpy;
                A(fv, i, j, k) = A(fv, i, j, k) - (A(rv, i, j, k + 1) * A(ww, i, j, k + 1)
                                                 - A(rv, i, j, k - 1) * A(ww, i, j, k - 1)) * tmpz;
            }
        }
    }
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz = HZ * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy = HY * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fw, i, j, k) = A(fw, i, j, k) - (A(rw, i + 1, j, k) * A(uu, i + 1, j, k)
                                                 - A(rw, i - 1, j, k) * A(uu, i - 1, j, k)) * HX * DXXDX[i];
                A(fw, i, j, k) = A(fw, i, j, k) - (A(rw, i, j + 1, k) * A(vv, i, j + 1, k)
                                                 - A(rw, i, j - 1, k) * A(vv, i, j - 1, k)) * tmpy;
                A(fw, i, j, k) = A(fw, i, j, k) - (A(rw, i, j, k + 1) * A(ww, i, j, k + 1)
                                                 - A(rw, i, j, k - 1) * A(ww, i, j, k - 1)) * tmpz;
            }
        }
    }
    /* 1495-1506: temperature advection (loop 450) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz = HZ * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy = HY * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(ft, i, j, k) = -(1.0 * A(uu, i, j, k) * (A(tt, i + 1, j, k) - A(tt, i - 1, j, k)) * HX * DXXDX[i]);
                A(ft, i, j, k) = A(ft, i, j, k) - A(vv, i, j, k) * (A(tt, i, j + 1, k) - A(tt, i, j - 1, k)) * tmpy;
                A(ft, i, j, k) = A(ft, i, j, k) - A(ww, i, j, k) * (A(tt, i, j, k + 1) - A(tt, i, j, k - 1)) * tmpz;
            }
        }
    }
    /* 1583-1611: conduction, non-LREM branch (loop 519); RO holds 1/rho */
    {
        const double TMP = OCV / REPR;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k) {
            double tmpz1 = HZ * D2ZZDZ2[k];
            double tmpz2 = H2Z * DZZDZ[k] * DZZDZ[k];
            for (int j = 2; j <= NY - 1; ++j) {
                double tmpy1 = HY * D2YYDY2[j];
                double tmpy2 = H2Y * DYYDY[j] * DYYDY[j];
                for (int i = 2; i <= NX - 1; ++i) {
                    A(ft, i, j, k) = A(ft, i, j, k)
                        + ((A(tt, i + 1, j, k) - A(tt, i - 1, j, k)) * HX * D2XXDX2[i]
                           + (A(tt, i + 1, j, k) - 2.0 * A(tt, i, j, k) + A(tt, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i])
                          * A(ro, i, j, k) * TMP * RKAPA[k];
                    A(ft, i, j, k) = A(ft, i, j, k)
                        + ((A(tt, i, j + 1, k) - A(tt, i, j - 1, k)) * tmpy1
                           + (A(tt, i, j + 1, k) - 2.0 * A(tt, i, j, k) + A(tt, i, j - 1, k)) * tmpy2)
                          * A(ro, i, j, k) * TMP * RKAPA[k];
                    A(ft, i, j, k) = A(ft, i, j, k)
                        + ((A(tt, i, j, k + 1) - A(tt, i, j, k - 1)) * tmpz1
                           + (A(tt, i, j, k + 1) - 2.0 * A(tt, i, j, k) + A(tt, i, j, k - 1)) * tmpz2)
                          * A(ro, i, j, k) * TMP * RKAPA[k];
                    A(ft, i, j, k) = A(ft, i, j, k) + (A(tt, i, j, k + 1) - A(tt, i, j, k - 1))
                                                      * HZ * DZZDZ[k] * A(ro, i, j, k) * TMP * DKAPA[k];
                }
            }
        }
    }
    /* 1818-1886: viscous momentum terms (loops 530, 540, 550) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz1 = HZ * D2ZZDZ2[k];
        double tmpz2 = H2Z * DZZDZ[k] * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy1 = HY * D2YYDY2[j];
            double tmpy2 = H2Y * DYYDY[j] * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fu, i, j, k) = A(fu, i, j, k) + ORE * (
                    C43 * ((A(uu, i + 1, j, k) - A(uu, i - 1, j, k)) * HX * D2XXDX2[i]
                           + (A(uu, i + 1, j, k) - 2.0 * A(uu, i, j, k) + A(uu, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i])
                    + (A(uu, i, j + 1, k) - A(uu, i, j - 1, k)) * tmpy1
                    + (A(uu, i, j + 1, k) - 2.0 * A(uu, i, j, k) + A(uu, i, j - 1, k)) * tmpy2
                    + (A(uu, i, j, k + 1) - A(uu, i, j, k - 1)) * tmpz1
                    + (A(uu, i, j, k + 1) - 2.0 * A(uu, i, j, k) + A(uu, i, j, k - 1)) * tmpz2);
            }
        }
    }
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz1 = HZ * D2ZZDZ2[k];
        double tmpz2 = H2Z * DZZDZ[k] * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy1 = HY * D2YYDY2[j];
            double tmpy2 = H2Y * DYYDY[j] * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fv, i, j, k) = A(fv, i, j, k) + ORE * (
                    (A(vv, i + 1, j, k) - A(vv, i - 1, j, k)) * HX * D2XXDX2[i]
                    + (A(vv, i + 1, j, k) - 2.0 * A(vv, i, j, k) + A(vv, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i]
                    + C43 * ((A(vv, i, j + 1, k) - A(vv, i, j - 1, k)) * tmpy1
                             + (A(vv, i, j + 1, k) - 2.0 * A(vv, i, j, k) + A(vv, i, j - 1, k)) * tmpy2)
                    + (A(vv, i, j, k + 1) - A(vv, i, j, k - 1)) * tmpz1
                    + (A(vv, i, j, k + 1) - 2.0 * A(vv, i, j, k) + A(vv, i, j, k - 1)) * tmpz2);
            }
        }
    }
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        double tmpz1 = HZ * D2ZZDZ2[k];
        double tmpz2 = H2Z * DZZDZ[k] * DZZDZ[k];
        for (int j = 2; j <= NY - 1; ++j) {
            double tmpy1 = HY * D2YYDY2[j];
            double tmpy2 = H2Y * DYYDY[j] * DYYDY[j];
            for (int i = 2; i <= NX - 1; ++i) {
                A(fw, i, j, k) = A(fw, i, j, k) + ORE * (
                    (A(ww, i + 1, j, k) - A(ww, i - 1, j, k)) * HX * D2XXDX2[i]
                    + (A(ww, i + 1, j, k) - 2.0 * A(ww, i, j, k) + A(ww, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i]
                    + (A(ww, i, j + 1, k) - A(ww, i, j - 1, k)) * tmpy1
                    + (A(ww, i, j + 1, k) - 2.0 * A(ww, i, j, k) + A(ww, i, j - 1, k)) * tmpy2
                    + C43 * ((A(ww, i, j, k + 1) - A(ww, i, j, k - 1)) * tmpz1
                             + (A(ww, i, j, k + 1) - 2.0 * A(ww, i, j, k) + A(ww, i, j, k - 1)) * tmpz2));
            }
        }
    }
    /* 1891-2101: viscous and compressional heating, (1/3) grad(div u) */
    /* loops 650, 670 cover J=1..NY so the y-differences at 720/730 see halo rows */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 1; j <= NY; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(w1, i, j, k) = (A(uu, i + 1, j, k) - A(uu, i - 1, j, k)) * HX * DXXDX[i];
                A(w2, i, j, k) = (A(vv, i + 1, j, k) - A(vv, i - 1, j, k)) * HX * DXXDX[i];
            }
    {
        const double TMPA = OCV * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 690 */
                    A(w3, i, j, k) = (A(ww, i + 1, j, k) - A(ww, i - 1, j, k)) * HX * DXXDX[i];
                    /* 700 */
                    A(ft, i, j, k) = A(ft, i, j, k) + (C43 * A(w1, i, j, k) * A(w1, i, j, k)
                                                     + A(w2, i, j, k) * A(w2, i, j, k)
                                                     + A(w3, i, j, k) * A(w3, i, j, k)) * A(ro, i, j, k) * TMPA;
                    /* 710 */
                    A(ft, i, j, k) = A(ft, i, j, k) - OCV * A(w1, i, j, k) * A(tt, i, j, k);
                }
    }
    {
        const double TMP = C13 * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 720 */
                    A(fu, i, j, k) = A(fu, i, j, k) + TMP * (A(w2, i, j + 1, k) - A(w2, i, j - 1, k)) * HY * DYYDY[j];
                    /* 730 */
                    A(fv, i, j, k) = A(fv, i, j, k) + TMP * (A(w1, i, j + 1, k) - A(w1, i, j - 1, k)) * HY * DYYDY[j];
                }
    }
    /* 740-770 (pointwise; overwrite WW1, WW2 after 720/730 have read them) */
    {
        const double TMPA = OCV * ORE, TMPB = C43 * OCV * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    A(w1, i, j, k) = (A(uu, i, j + 1, k) - A(uu, i, j - 1, k)) * HY * DYYDY[j];
                    A(ft, i, j, k) = A(ft, i, j, k) + (A(w1, i, j, k) * A(w1, i, j, k)
                                                     + 2.0 * A(w1, i, j, k) * A(w2, i, j, k)) * A(ro, i, j, k) * TMPA;
                    A(w2, i, j, k) = (A(vv, i, j + 1, k) - A(vv, i, j - 1, k)) * HY * DYYDY[j];
                    A(ft, i, j, k) = A(ft, i, j, k) + A(w2, i, j, k) * A(w2, i, j, k) * A(ro, i, j, k) * TMPB;
                    A(ft, i, j, k) = A(ft, i, j, k) - OCV * A(w2, i, j, k) * A(tt, i, j, k);
                    /* 780 */
                    A(w1, i, j, k) = (A(uu, i + 1, j, k) - A(uu, i - 1, j, k)) * HX * DXXDX[i];
                }
    }
    /* 790: WW3 = dW/dz over J=1..NY, I=1..NX (central, also at the walls) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 1; j <= NY; ++j)
            for (int i = 1; i <= NX; ++i)
                A(w3, i, j, k) = (A(ww, i, j, k + 1) - A(ww, i, j, k - 1)) * HZ * DZZDZ[k];
    {
        const double TMPB = C43 * OCV * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 820 */
                    A(ft, i, j, k) = A(ft, i, j, k) + (A(w3, i, j, k) * A(w3, i, j, k)
                                                     - A(w1, i, j, k) * A(w3, i, j, k)
                                                     - A(w1, i, j, k) * A(w2, i, j, k)
                                                     - A(w2, i, j, k) * A(w3, i, j, k)) * A(ro, i, j, k) * TMPB;
                    /* 830 */
                    A(ft, i, j, k) = A(ft, i, j, k) - OCV * A(w3, i, j, k) * A(tt, i, j, k);
                }
    }
    {
        const double TMP = C13 * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 840, 850 */
                    A(fu, i, j, k) = A(fu, i, j, k) + TMP * (A(w3, i + 1, j, k) - A(w3, i - 1, j, k)) * HX * DXXDX[i];
                    A(fv, i, j, k) = A(fv, i, j, k) + TMP * (A(w3, i, j + 1, k) - A(w3, i, j - 1, k)) * HY * DYYDY[j];
                }
    }
    /* 860: WW1 = dU/dz for J=2..NY-1, I=1..NX;  880: WW2 = dV/dz for J=1..NY, I=2..NX-1 */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k) {
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 1; i <= NX; ++i)
                A(w1, i, j, k) = (A(uu, i, j, k + 1) - A(uu, i, j, k - 1)) * HZ * DZZDZ[k];
        for (int j = 1; j <= NY; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(w2, i, j, k) = (A(vv, i, j, k + 1) - A(vv, i, j, k - 1)) * HZ * DZZDZ[k];
    }
    {
        const double TMPA = OCV * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 900 */
                    A(w3, i, j, k) = (A(ww, i, j + 1, k) - A(ww, i, j - 1, k)) * HY * DYYDY[j];
                    /* 910 */
                    A(ft, i, j, k) = A(ft, i, j, k) + (A(w1, i, j, k) * A(w1, i, j, k)
                                                     + A(w2, i, j, k) * A(w2, i, j, k)
                                                     + A(w3, i, j, k) * A(w3, i, j, k)
                                                     + 2.0 * A(w2, i, j, k) * A(w3, i, j, k)) * A(ro, i, j, k) * TMPA;
                }
    }
    {
        const double TMP = C13 * ORE, TMPA = OCV * ORE;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 920 */
                    A(fw, i, j, k) = A(fw, i, j, k) + TMP * ((A(w1, i + 1, j, k) - A(w1, i - 1, j, k)) * HX * DXXDX[i]
                                                           + (A(w2, i, j + 1, k) - A(w2, i, j - 1, k)) * HY * DYYDY[j]);
                }
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    /* 930, 940 (after 920 has read the WW1 neighbours) */
                    A(w3, i, j, k) = (A(ww, i + 1, j, k) - A(ww, i - 1, j, k)) * HX * DXXDX[i];
                    A(ft, i, j, k) = A(ft, i, j, k) + 2.0 * A(w1, i, j, k) * A(w3, i, j, k) * A(ro, i, j, k) * TMPA;
                }
    }
    /* 2106-2125: Coriolis (loops 950, 960, 970) */
    if (P->lrot) {
        const double OMX = P->omx, OMZ = P->omz;
        PAR_K
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    A(fu, i, j, k) = A(fu, i, j, k) + OMZ * A(rv, i, j, k);
                    A(fv, i, j, k) = A(fv, i, j, k) - OMZ * A(ru, i, j, k) + OMX * A(rw, i, j, k);
                    A(fw, i, j, k) = A(fw, i, j, k) - OMX * A(rv, i, j, k);
                }
    }
    if (!P->lmag) return;

    /* 2129-2634: induction (WW1..WW3 = dB/dt), Lorentz force, Ohmic heating.
       RU,RV,RW,TT interior cells serve as pointwise scratch from here on. */
    const double OBETA = P->obeta, ORM = P->orm;
    const double TMPM = OBETA * ORM * OCV;
    /* 1000-1040: x-derivatives of velocity; WW2, WW3 start */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(ru, i, j, k) = (A(uu, i + 1, j, k) - A(uu, i - 1, j, k)) * HX * DXXDX[i];
                A(rv, i, j, k) = (A(vv, i + 1, j, k) - A(vv, i - 1, j, k)) * HX * DXXDX[i];
                A(rw, i, j, k) = (A(ww, i + 1, j, k) - A(ww, i - 1, j, k)) * HX * DXXDX[i];
                A(w2, i, j, k) = A(bx, i, j, k) * A(rv, i, j, k) - A(by, i, j, k) * A(ru, i, j, k);
                A(w3, i, j, k) = A(bx, i, j, k) * A(rw, i, j, k) - A(bz, i, j, k) * A(ru, i, j, k);
            }
    /* 1050-1090: y-derivatives of velocity */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(ru, i, j, k) = (A(uu, i, j + 1, k) - A(uu, i, j - 1, k)) * HY * DYYDY[j];
                A(rv, i, j, k) = (A(vv, i, j + 1, k) - A(vv, i, j - 1, k)) * HY * DYYDY[j];
                A(rw, i, j, k) = (A(ww, i, j + 1, k) - A(ww, i, j - 1, k)) * HY * DYYDY[j];
                A(w1, i, j, k) = A(by, i, j, k) * A(ru, i, j, k) - A(bx, i, j, k) * A(rv, i, j, k);
                A(w3, i, j, k) = A(w3, i, j, k) + A(by, i, j, k) * A(rw, i, j, k) - A(bz, i, j, k) * A(rv, i, j, k);
            }
    /* 1100-1126: z-derivatives of velocity; dW/dz one-sided at both walls */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(ru, i, j, k) = (A(uu, i, j, k + 1) - A(uu, i, j, k - 1)) * HZ * DZZDZ[k];
                A(rv, i, j, k) = (A(vv, i, j, k + 1) - A(vv, i, j, k - 1)) * HZ * DZZDZ[k];
                A(rw, i, j, k) = (A(ww, i, j, k + 1) - A(ww, i, j, k - 1)) * HZ * DZZDZ[k];
            }
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i) {
            A(rw, i, j, 2) = (4.0 * A(ww, i, j, 3) - A(ww, i, j, 4)) * HZ * DZZDZ[2];
            A(rw, i, j, NZ - 1) = (A(ww, i, j, NZ - 3) - 4.0 * A(ww, i, j, NZ - 2)) * HZ * DZZDZ[NZ - 1];
        }
    /* 1130-1250 */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                /* 1130, 1140 */
                A(w1, i, j, k) = A(w1, i, j, k) + A(bz, i, j, k) * A(ru, i, j, k) - A(bx, i, j, k) * A(rw, i, j, k);
                A(w2, i, j, k) = A(w2, i, j, k) + A(bz, i, j, k) * A(rv, i, j, k) - A(by, i, j, k) * A(rw, i, j, k);
                /* 1150-1180: dBx/dx, dBy/dx, dBz/dx, dBx/dy */
                A(ru, i, j, k) = (A(bx, i + 1, j, k) - A(bx, i - 1, j, k)) * HX * DXXDX[i];
                A(rv, i, j, k) = (A(by, i + 1, j, k) - A(by, i - 1, j, k)) * HX * DXXDX[i];
                A(rw, i, j, k) = (A(bz, i + 1, j, k) - A(bz, i - 1, j, k)) * HX * DXXDX[i];
                A(tt, i, j, k) = (A(bx, i, j + 1, k) - A(bx, i, j - 1, k)) * HY * DYYDY[j];
                /* 1190-1210: Lorentz force */
                A(fu, i, j, k) = A(fu, i, j, k) + OBETA * A(by, i, j, k) * (A(tt, i, j, k) - A(rv, i, j, k))
                                 - OBETA * A(bz, i, j, k) * A(rw, i, j, k);
                A(fv, i, j, k) = A(fv, i, j, k) + OBETA * A(bx, i, j, k) * (A(rv, i, j, k) - A(tt, i, j, k));
                A(fw, i, j, k) = A(fw, i, j, k) + OBETA * A(bx, i, j, k) * A(rw, i, j, k);
                /* 1220: Ohmic heating */
                A(ft, i, j, k) = A(ft, i, j, k) + (A(tt, i, j, k) * A(tt, i, j, k)
                                                 + A(rv, i, j, k) * A(rv, i, j, k)
                                                 + A(rw, i, j, k) * A(rw, i, j, k)
                                                 - 2.0 * A(rv, i, j, k) * A(tt, i, j, k)) * A(ro, i, j, k) * TMPM;
                /* 1230-1250 */
                A(w1, i, j, k) = A(w1, i, j, k) - A(uu, i, j, k) * A(ru, i, j, k) - A(vv, i, j, k) * A(tt, i, j, k);
                A(w2, i, j, k) = A(w2, i, j, k) - A(uu, i, j, k) * A(rv, i, j, k);
                A(w3, i, j, k) = A(w3, i, j, k) - A(uu, i, j, k) * A(rw, i, j, k);
            }
    /* 1260-1350: horizontal diffusion of B, dBx/dz, dBy/dy */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(ru, i, j, k) = (A(bx, i + 1, j, k) - A(bx, i - 1, j, k)) * HX * D2XXDX2[i]
                               + (A(bx, i + 1, j, k) - 2.0 * A(bx, i, j, k) + A(bx, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i];
                A(rv, i, j, k) = (A(by, i + 1, j, k) - A(by, i - 1, j, k)) * HX * D2XXDX2[i]
                               + (A(by, i + 1, j, k) - 2.0 * A(by, i, j, k) + A(by, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i];
                A(tt, i, j, k) = (A(bx, i, j + 1, k) - A(bx, i, j - 1, k)) * HY * D2YYDY2[j]
                               + (A(bx, i, j + 1, k) - 2.0 * A(bx, i, j, k) + A(bx, i, j - 1, k)) * H2Y * DYYDY[j] * DYYDY[j];
                A(w1, i, j, k) = A(w1, i, j, k) + ORM * (A(ru, i, j, k) + A(tt, i, j, k));
                A(w2, i, j, k) = A(w2, i, j, k) + ORM * A(rv, i, j, k);
                A(tt, i, j, k) = (A(bz, i + 1, j, k) - A(bz, i - 1, j, k)) * HX * D2XXDX2[i]
                               + (A(bz, i + 1, j, k) - 2.0 * A(bz, i, j, k) + A(bz, i - 1, j, k)) * H2X * DXXDX[i] * DXXDX[i];
                A(w3, i, j, k) = A(w3, i, j, k) + ORM * A(tt, i, j, k);
                A(ru, i, j, k) = (A(bx, i, j, k + 1) - A(bx, i, j, k - 1)) * HZ * DZZDZ[k];
                A(rv, i, j, k) = (A(by, i, j + 1, k) - A(by, i, j - 1, k)) * HY * DYYDY[j];
                A(fu, i, j, k) = A(fu, i, j, k) + OBETA * A(bz, i, j, k) * A(ru, i, j, k);
                A(fw, i, j, k) = A(fw, i, j, k) - OBETA * A(bx, i, j, k) * A(ru, i, j, k);
                /* 1360: RW still holds dBz/dx from 1170 */
                A(ft, i, j, k) = A(ft, i, j, k) + (A(ru, i, j, k) * A(ru, i, j, k)
                                                 - 2.0 * A(ru, i, j, k) * A(rw, i, j, k)) * A(ro, i, j, k) * TMPM;
                /* 1370, 1380 */
                A(w1, i, j, k) = A(w1, i, j, k) - A(ww, i, j, k) * A(ru, i, j, k);
                A(w2, i, j, k) = A(w2, i, j, k) - A(vv, i, j, k) * A(rv, i, j, k);
            }
    /* 1390-1392: d2Bx/dz2, one-sided at both walls */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(ru, i, j, k) = (A(bx, i, j, k + 1) - A(bx, i, j, k - 1)) * HZ * D2ZZDZ2[k]
                               + (A(bx, i, j, k + 1) - 2.0 * A(bx, i, j, k) + A(bx, i, j, k - 1)) * H2Z * DZZDZ[k] * DZZDZ[k];
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i) {
            A(ru, i, j, 2) = (-3.0 * A(bx, i, j, 2) + 4.0 * A(bx, i, j, 3) - A(bx, i, j, 4)) * HZ * D2ZZDZ2[2]
                           + (2.0 * A(bx, i, j, 2) - 5.0 * A(bx, i, j, 3) + 4.0 * A(bx, i, j, 4) - A(bx, i, j, 5))
                             * H2Z * DZZDZ[2] * DZZDZ[2];
            A(ru, i, j, NZ - 1) = (3.0 * A(bx, i, j, NZ - 1) - 4.0 * A(bx, i, j, NZ - 2) + A(bx, i, j, NZ - 3)) * HZ * D2ZZDZ2[NZ - 1]
                                + (2.0 * A(bx, i, j, NZ - 1) - 5.0 * A(bx, i, j, NZ - 2) + 4.0 * A(bx, i, j, NZ - 3) - A(bx, i, j, NZ - 4))
                                  * H2Z * DZZDZ[NZ - 1] * DZZDZ[NZ - 1];
        }
    /* 1400-1500 */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(rv, i, j, k) = (A(by, i, j + 1, k) - A(by, i, j - 1, k)) * HY * D2YYDY2[j]
                               + (A(by, i, j + 1, k) - 2.0 * A(by, i, j, k) + A(by, i, j - 1, k)) * H2Y * DYYDY[j] * DYYDY[j];
                A(w1, i, j, k) = A(w1, i, j, k) + ORM * A(ru, i, j, k);
                A(w2, i, j, k) = A(w2, i, j, k) + ORM * A(rv, i, j, k);
                A(rv, i, j, k) = (A(by, i, j, k + 1) - A(by, i, j, k - 1)) * HZ * DZZDZ[k];
                A(rw, i, j, k) = (A(bz, i, j + 1, k) - A(bz, i, j - 1, k)) * HY * DYYDY[j];
                A(ru, i, j, k) = A(rv, i, j, k) - A(rw, i, j, k);
                A(fv, i, j, k) = A(fv, i, j, k) + OBETA * A(bz, i, j, k) * A(ru, i, j, k);
                A(fw, i, j, k) = A(fw, i, j, k) - OBETA * A(by, i, j, k) * A(ru, i, j, k);
                A(ft, i, j, k) = A(ft, i, j, k) + (A(rv, i, j, k) * A(rv, i, j, k)
                                                 + A(rw, i, j, k) * A(rw, i, j, k)
                                                 - 2.0 * A(rv, i, j, k) * A(rw, i, j, k)) * A(ro, i, j, k) * TMPM;
                A(w2, i, j, k) = A(w2, i, j, k) - A(ww, i, j, k) * A(rv, i, j, k);
                A(w3, i, j, k) = A(w3, i, j, k) - A(vv, i, j, k) * A(rw, i, j, k);
            }
    /* 1510-1513: d2By/dz2, one-sided at both walls */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(rv, i, j, k) = (A(by, i, j, k + 1) - A(by, i, j, k - 1)) * HZ * D2ZZDZ2[k]
                               + (A(by, i, j, k + 1) - 2.0 * A(by, i, j, k) + A(by, i, j, k - 1)) * H2Z * DZZDZ[k] * DZZDZ[k];
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i) {
            A(rv, i, j, 2) = (-3.0 * A(by, i, j, 2) + 4.0 * A(by, i, j, 3) - A(by, i, j, 4)) * HZ * D2ZZDZ2[2]
                           + (2.0 * A(by, i, j, 2) - 5.0 * A(by, i, j, 3) + 4.0 * A(by, i, j, 4) - A(by, i, j, 5))
                             * H2Z * DZZDZ[2] * DZZDZ[2];
            A(rv, i, j, NZ - 1) = (3.0 * A(by, i, j, NZ - 1) - 4.0 * A(by, i, j, NZ - 2) + A(by, i, j, NZ - 3)) * HZ * D2ZZDZ2[NZ - 1]
                                + (2.0 * A(by, i, j, NZ - 1) - 5.0 * A(by, i, j, NZ - 2) + 4.0 * A(by, i, j, NZ - 3) - A(by, i, j, NZ - 4))
                                  * H2Z * DZZDZ[NZ - 1] * DZZDZ[NZ - 1];
        }
    /* 1520-1580 */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                A(rw, i, j, k) = (A(bz, i, j + 1, k) - A(bz, i, j - 1, k)) * HY * D2YYDY2[j]
                               + (A(bz, i, j + 1, k) - 2.0 * A(bz, i, j, k) + A(bz, i, j - 1, k)) * H2Y * DYYDY[j] * DYYDY[j];
                A(w2, i, j, k) = A(w2, i, j, k) + ORM * A(rv, i, j, k);
                A(w3, i, j, k) = A(w3, i, j, k) + ORM * A(rw, i, j, k);
                A(rw, i, j, k) = (A(bz, i, j, k + 1) - A(bz, i, j, k - 1)) * HZ * DZZDZ[k];
                A(w3, i, j, k) = A(w3, i, j, k) - A(ww, i, j, k) * A(rw, i, j, k);
                A(rw, i, j, k) = (A(bz, i, j, k + 1) - A(bz, i, j, k - 1)) * HZ * D2ZZDZ2[k]
                               + (A(bz, i, j, k + 1) - 2.0 * A(bz, i, j, k) + A(bz, i, j, k - 1)) * H2Z * DZZDZ[k] * DZZDZ[k];
                A(w3, i, j, k) = A(w3, i, j, k) + ORM * A(rw, i, j, k);
            }
}

/* ------------------------------------------------------------------ */
/* BCON (3dmhdsub.f:2751-2955), non-LSHR, non-LREM                     */
/* ------------------------------------------------------------------ */
static void bcon(oracle3dmhd* o)
{
    const mhd3d_params* P = &o->p;
    const double C13 = P->c13, C23 = P->c23, C43 = P->c43;
    const int ITC = P->itcon, IZC = P->izcon;
    /* Top, K = 2 (2767-2880) */
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i)
            A(ru, i, j, 2) = A(ro, i, j, 2) * (C43 * A(ru, i, j, 3) / A(ro, i, j, 3) - C13 * A(ru, i, j, 4) / A(ro, i, j, 4));
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i)
            A(rv, i, j, 2) = A(ro, i, j, 2) * (C43 * A(rv, i, j, 3) / A(ro, i, j, 3) - C13 * A(rv, i, j, 4) / A(ro, i, j, 4));
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i) A(rw, i, j, 2) = 0.0;
    if (P->tp != 0.0 && (ITC == 0 || ITC == 1)) {
        /* 2790-2826: Gaussian plume on the upper boundary */
        double tpr = (P->tc != 0.0) ? P->tp + (1.0 - P->tp) * exp(-o->timt / P->tc) : P->tp;
        /* CLN=-4.0E00*LOG(2.0E00)/HH/HH: LOG of a REAL(4) literal is REAL(4) */
        double cln = (double)(-(4.0f * logf(2.0f))) / P->hh / P->hh;
        if (ITC == 0) {
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i)
                    A(tt, i, j, 2) = 1.0 - (1.0 - tpr) * exp(cln * ((o->exx[i] - P->xp) * (o->exx[i] - P->xp))) / P->hh
                                                       * exp(cln * ((o->wyy[j] - P->yp) * (o->wyy[j] - P->yp))) / P->hh;
        } else {
            double dz = (double)(1.0f / (float)(P->npz - 1)) / o->dzzdz[2];
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i)
                    A(tt, i, j, 2) = C43 * A(tt, i, j, 3) - C13 * A(tt, i, j, 4)
                                   - C23 * dz * (P->theta - (P->theta - tpr)
                                                 * exp(cln * ((o->exx[i] - P->xp) * (o->exx[i] - P->xp))) / P->hh
                                                 * exp(cln * ((o->wyy[j] - P->yp) * (o->wyy[j] - P->yp))) / P->hh);
        }
    } else {
        if (ITC == 0 || ITC == 2 || ITC == 4) {
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    A(tt, i, j, 2) = 1.0;
                    if (ITC == 4 && i <= NX / 2) A(tt, i, j, 2) = 1.0 - P->tp;
                }
        }
        if (ITC == 1) {
            double dz = (double)(1.0f / (float)(P->npz - 1)) / o->dzzdz[2];
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i)
                    A(tt, i, j, 2) = C43 * A(tt, i, j, 3) - C13 * A(tt, i, j, 4) - C23 * dz * P->theta;
        }
    }
    if (P->lmag && P->ibcon == 0)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) A(bz, i, j, 2) = 0.0;
    /* Bottom, K = NZ-1 (2884-2956) */
    const int KB = NZ - 1;
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i)
            A(ru, i, j, KB) = A(ro, i, j, KB) * (C43 * A(ru, i, j, KB - 1) / A(ro, i, j, KB - 1)
                                               - C13 * A(ru, i, j, KB - 2) / A(ro, i, j, KB - 2));
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i)
            A(rv, i, j, KB) = A(ro, i, j, KB) * (C43 * A(rv, i, j, KB - 1) / A(ro, i, j, KB - 1)
                                               - C13 * A(rv, i, j, KB - 2) / A(ro, i, j, KB - 2));
    for (int j = 2; j <= NY - 1; ++j)
        for (int i = 2; i <= NX - 1; ++i) A(rw, i, j, KB) = 0.0;
    if (IZC == 0) {
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) A(tt, i, j, KB) = P->tb;
    } else {
        double dz = (double)(1.0f / (float)(P->npz - 1)) / o->dzzdz[KB];
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i)
                A(tt, i, j, KB) = C43 * A(tt, i, j, KB - 1) - C13 * A(tt, i, j, KB - 2)
                                + C23 * dz * P->theta / o->rkapa[KB];
    }
    if (P->lmag && P->ibcon == 0)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) A(bz, i, j, KB) = 0.0;
}

void oracle_bcon(oracle3dmhd* o) { bcon(o); }

/* ------------------------------------------------------------------ */
/* STEP: CFL and Mach number (3dmhdsub.f:741-873, ISW=1 branch)        */
/* ------------------------------------------------------------------ */
static void cfl(oracle3dmhd* o, double* dt_out, double* umach_out)
{
    const mhd3d_params* P = &o->p;
    const double GAMMA = P->gamma, OBETA = P->obeta, REPR = P->repr, CV = P->cv, RE = P->re, RM = P->rm;
    const double OGAMMA = 1.0 / GAMMA;
    double umach = 0.0;
    /* loops 10, 20 */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                double r = 1.0 / A(ro, i, j, k);
                A(uu, i, j, k) = (A(ru, i, j, k) * A(ru, i, j, k) + A(rv, i, j, k) * A(rv, i, j, k)
                                  + A(rw, i, j, k) * A(rw, i, j, k)) * (r * r);
            }
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(max : umach)
#endif
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                double v = OGAMMA * A(uu, i, j, k) / A(tt, i, j, k);
                umach = umach > v ? umach : v;
            }
    umach = sqrt(umach);
    /* loops 30 / 40: fast-mode speed squared */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                double u2 = A(uu, i, j, k), t = A(tt, i, j, k);
                if (P->lmag) {
                    double b2 = A(bx, i, j, k) * A(bx, i, j, k) + A(by, i, j, k) * A(by, i, j, k)
                              + A(bz, i, j, k) * A(bz, i, j, k);
                    A(uu, i, j, k) = u2 + GAMMA * t + b2 * OBETA / A(ro, i, j, k)
                                   + 2.0 * sqrt(u2 * (GAMMA * t + b2 * OBETA / A(ro, i, j, k)));
                } else {
                    A(uu, i, j, k) = u2 + GAMMA * t + 2.0 * sqrt(u2 * GAMMA * t);
                }
            }
    /* loop 2 and the MINVALs (835-872) */
    double m1 = HUGE_VAL, m2 = HUGE_VAL, m3 = HUGE_VAL, m4 = HUGE_VAL;
    int bad = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(min : m1, m2, m3, m4) reduction(| : bad)
#endif
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                double dd = o->ddx[i];
                if (o->ddy[j] < dd) dd = o->ddy[j];
                if (o->ddz[k] < dd) dd = o->ddz[k];
                double a = dd / sqrt(A(uu, i, j, k));
                double b = 0.5 * dd * dd * REPR * CV * A(ro, i, j, k) / o->rkapa[k];
                double c = 0.375 * dd * dd * RE * A(ro, i, j, k);
                A(w1, i, j, k) = a; A(w2, i, j, k) = b; A(w3, i, j, k) = c;
                bad |= !(isfinite(a) && isfinite(b) && isfinite(c));
                if (a < m1) m1 = a;
                if (b < m2) m2 = b;
                if (c < m3) m3 = c;
                if (P->lmag) {
                    double d = 0.5 * dd * dd * RM;
                    A(vv, i, j, k) = d;
                    if (d < m4) m4 = d;
                }
            }
    double m = m1;
    if (m2 < m) m = m2;
    if (m3 < m) m = m3;
    if (P->lmag && m4 < m) m = m4;
    *dt_out = bad ? NAN : P->sf * m;
    *umach_out = umach;
}

static int health(oracle3dmhd* o)
{
    if (!isfinite(o->dt) || !isfinite(o->umach)) return MHD3D_ERR_NONFINITE;
    if (o->dt < o->p.dtmin) return MHD3D_ERR_DT_SMALL;
    return MHD3D_OK;
}

int oracle_cfl(oracle3dmhd* o, double* dt, double* umach)
{
    double d, u;
    cfl(o, &d, &u);
    if (dt) *dt = d;
    if (umach) *umach = u;
    if (!isfinite(d) || !isfinite(u)) return MHD3D_ERR_NONFINITE;
    return MHD3D_OK;
}

/* U = Z + COEF*F over the interior (loops 70-140, 270-340, 470-540) */
static void update_u(oracle3dmhd* o, double coef)
{
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                size_t c = IDX(i, j, k);
                o->ru[c] = o->zru[c] + coef * o->fu[c];
                o->rv[c] = o->zrv[c] + coef * o->fv[c];
                o->rw[c] = o->zrw[c] + coef * o->fw[c];
                o->ro[c] = o->zro[c] + coef * o->fr[c];
                o->tt[c] = o->ztt[c] + coef * o->ft[c];
                if (o->p.lmag) {
                    o->bx[c] = o->zbx[c] + coef * o->w1[c];
                    o->by[c] = o->zby[c] + coef * o->w2[c];
                    o->bz[c] = o->zbz[c] + coef * o->w3[c];
                }
            }
}

/* Z = U + COEF*F over the interior (loops 190-260, 390-460) */
static void update_z(oracle3dmhd* o, double coef)
{
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                size_t c = IDX(i, j, k);
                o->zru[c] = o->ru[c] + coef * o->fu[c];
                o->zrv[c] = o->rv[c] + coef * o->fv[c];
                o->zrw[c] = o->rw[c] + coef * o->fw[c];
                o->zro[c] = o->ro[c] + coef * o->fr[c];
                o->ztt[c] = o->tt[c] + coef * o->ft[c];
                if (o->p.lmag) {
                    o->zbx[c] = o->bx[c] + coef * o->w1[c];
                    o->zby[c] = o->by[c] + coef * o->w2[c];
                    o->zbz[c] = o->bz[c] + coef * o->w3[c];
                }
            }
}

/* One STEP (3dmhdsub.f:687-1176). */
static void step_once(oracle3dmhd* o)
{
    const mhd3d_params* P = &o->p;
    cfl(o, &o->dt, &o->umach);
    const double DT = o->dt;
    /* stage 1: Z = U (loops 71-141) */
    PAR_K
    for (int k = 2; k <= NZ - 1; ++k)
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                size_t c = IDX(i, j, k);
                o->zru[c] = o->ru[c]; o->zrv[c] = o->rv[c]; o->zrw[c] = o->rw[c];
                o->zro[c] = o->ro[c]; o->ztt[c] = o->tt[c];
                if (P->lmag) { o->zbx[c] = o->bx[c]; o->zby[c] = o->by[c]; o->zbz[c] = o->bz[c]; }
            }
    fluxes(o);
    update_u(o, P->gam1 * DT);
    bcon(o);
    communicate(o);
    /* stage 2 */
    update_z(o, P->zeta1 * DT);
    fluxes(o);
    update_u(o, P->gam2 * DT);
    bcon(o);
    communicate(o);
    /* stage 3 */
    update_z(o, P->zeta2 * DT);
    fluxes(o);
    update_u(o, P->gam3 * DT);
    bcon(o);
    communicate(o);
    o->nit += 1;
    o->timc = o->timc + DT;
    o->timt = o->timi + o->timc;
}

int oracle_step(oracle3dmhd* o, int nsteps, double* dt, double* timc, double* timt,
                double* umach, int* nit)
{
    int st = MHD3D_OK;
    for (int s = 0; s < nsteps; ++s) {
        step_once(o);
        st = health(o);
        if (st != MHD3D_OK) break;
    }
    if (dt) *dt = o->dt;
    if (timc) *timc = o->timc;
    if (timt) *timt = o->timt;
    if (umach) *umach = o->umach;
    if (nit) *nit = o->nit;
    return st;
}

void oracle_fluxes(oracle3dmhd* o, double* fu, double* fv, double* fw, double* fr, double* ft,
                   double* ww1, double* ww2, double* ww3)
{
    size_t nb = o->n * sizeof(double);
    double* save[8];
    double* cur[8] = {o->ru, o->rv, o->rw, o->ro, o->tt, o->bx, o->by, o->bz};
    for (int a = 0; a < 8; ++a) { save[a] = (double*)malloc(nb); memcpy(save[a], cur[a], nb); }
    memset(o->fu, 0, nb); memset(o->fv, 0, nb); memset(o->fw, 0, nb);
    memset(o->fr, 0, nb); memset(o->ft, 0, nb);
    memset(o->w1, 0, nb); memset(o->w2, 0, nb); memset(o->w3, 0, nb);
    fluxes(o);
    if (fu) memcpy(fu, o->fu, nb);
    if (fv) memcpy(fv, o->fv, nb);
    if (fw) memcpy(fw, o->fw, nb);
    if (fr) memcpy(fr, o->fr, nb);
    if (ft) memcpy(ft, o->ft, nb);
    if (o->p.lmag) {
        if (ww1) memcpy(ww1, o->w1, nb);
        if (ww2) memcpy(ww2, o->w2, nb);
        if (ww3) memcpy(ww3, o->w3, nb);
    }
    for (int a = 0; a < 8; ++a) { memcpy(cur[a], save[a], nb); free(save[a]); }
}

/* HORIZONTAL_MEAN (3dmhdsub.f:3143-3223, NGRID=0 branch): the sum over
 * I=IX/2+1..NX-IX/2, J=IY/2+1..NY-IY/2 of plane K, J outer, divided by
 * FLOAT(NPX*NPY).  The per-cell quantities are those of the flux diagnostics
 * (1651-1661) with u=RU*(1/RO) as FLUXES forms it (1386-1425). */
void oracle_profiles(const oracle3dmhd* o, double* out)
{
    const int npz = o->p.npz;
    const double cnt = (double)(float)(o->p.npx * o->p.npy);
    double* ttm = (double*)malloc(sizeof(double) * (size_t)NZ);
    for (int k = 2; k <= NZ - 1; ++k) {
        double sro = 0.0, stt = 0.0, ske = 0.0, sen = 0.0, sme = 0.0;
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                const size_t c = IDX(i, j, k);
                const double ro = o->ro[c], tt = o->tt[c];
                const double ri = 1.0 / ro;
                const double u = o->ru[c] * ri, v = o->rv[c] * ri, w = o->rw[c] * ri;
                sro = sro + ro;
                stt = stt + tt;
                ske = ske + 0.5 * ro * (u * u + v * v + w * w);
                sen = sen + 2.5 * ro * tt;
                if (o->p.lmag) sme = sme + 0.5 * (o->bx[c] * o->bx[c] + o->by[c] * o->by[c] + o->bz[c] * o->bz[c]);
            }
        const int r = k - 2;
        out[MHD3D_PROF_RHO * npz + r] = sro / cnt;
        out[MHD3D_PROF_T * npz + r] = ttm[k - 1] = stt / cnt;
        out[MHD3D_PROF_KE * npz + r] = ske / cnt;
        out[MHD3D_PROF_ENTH * npz + r] = sen / cnt;
        out[MHD3D_PROF_ME * npz + r] = sme / cnt;
        /* FCONM: WW2=-RW*(2.5*WW1+0.5*(UU*UU+VV*VV+WW*WW)), WW1=TT-TTM (1524-1528, 1653-1656) */
        double sfc = 0.0;
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                const size_t c = IDX(i, j, k);
                const double ri = 1.0 / o->ro[c];
                const double u = o->ru[c] * ri, v = o->rv[c] * ri, w = o->rw[c] * ri;
                sfc = sfc + -o->rw[c] * (2.5 * (o->tt[c] - ttm[k - 1]) + 0.5 * (u * u + v * v + w * w));
            }
        out[MHD3D_PROF_FCONV * npz + r] = sfc / cnt;
    }
    /* FRADM (1663-1676) */
    for (int k = 2; k <= NZ - 1; ++k) {
        double d;
        if (k == 2) d = -3.0 * ttm[1] + 4.0 * ttm[2] - ttm[3];
        else if (k == NZ - 1) d = 3.0 * ttm[NZ - 2] - 4.0 * ttm[NZ - 3] + ttm[NZ - 4];
        else d = ttm[k] - ttm[k - 2];
        out[MHD3D_PROF_FRAD * npz + (k - 2)] = d * o->p.hz * o->dzzdz[k] * o->rkapa[k] / o->p.repr;   /* 1-based */
    }
    free(ttm);
}
