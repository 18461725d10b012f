/*
 * oracle3dmhd.h -- CPU restatement of the 3dmhd time step (test
 * infrastructure only).
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load this library.  It is the checker the GPU path is
 * compared against; nothing in the product links it.
 *
 * Parity pin: the reference has no tests and no golden data.  This
 * restatement is pinned against the reference's own STEP/FLUXES/BCON/
 * COMMUNICATE source, mechanically translated to C and run with the
 * reference's MPI decomposition (oracle/fortran_subset.py,
 * oracle/make_ref.py), and through the golden fixtures that translated
 * reference wrote (tests/golden/).
 *
 * State layout: Fortran column-major REAL*8 (NX,NY,NZ) arrays with
 * NX=NPX+2, NY=NPY+2, NZ=NPZ+2, exactly the reference's local arrays for a
 * single domain; walls at K=2 and K=NZ-1, ghost planes at K=1 and K=NZ.
 */
#ifndef ORACLE3DMHD_H
#define ORACLE3DMHD_H

#include "../include/mhd3d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle3dmhd oracle3dmhd;

/* Metric arrays have the COMMON/AJACOBI lengths NX, NY, NZ (3dmhd.f:36-38). */
oracle3dmhd* oracle_create(const mhd3d_params* p,
                           const double* exx, const double* dxxdx, const double* d2xxdx2, const double* ddx,
                           const double* wyy, const double* dyydy, const double* d2yydy2, const double* ddy,
                           const double* zee, const double* dzzdz, const double* d2zzdz2, const double* ddz,
                           const double* rkapa, const double* dkapa);
void oracle_destroy(oracle3dmhd* o);

/* Copy a state in (then refresh the periodic halos, as the driver's
 * COMMUNICATE after initialisation does, 3dmhd.f:365) / copy it out. */
void oracle_set_state(oracle3dmhd* o, const double* ru, const double* rv, const double* rw,
                      const double* tt, const double* ro,
                      const double* bx, const double* by, const double* bz);
void oracle_get_state(const oracle3dmhd* o, double* ru, double* rv, double* rw,
                      double* tt, double* ro, double* bx, double* by, double* bz);

/* nsteps x STEP (3dmhdsub.f:687-1176).  Returns an MHD3D_* status with the
 * same early-stop rule as mhd3d_step. */
int oracle_step(oracle3dmhd* o, int nsteps, double* dt, double* timc, double* timt,
                double* umach, int* nit);

/* FLUXES (3dmhdsub.f:1178-2637) on a copy of the state; the state is not
 * changed.  Outputs are full (NX,NY,NZ) arrays; ww* may be NULL without LMAG. */
void oracle_fluxes(oracle3dmhd* o, double* fu, double* fv, double* fw, double* fr, double* ft,
                   double* ww1, double* ww2, double* ww3);

/* CFL/Mach part of STEP (3dmhdsub.f:741-873) on the current state. */
int oracle_cfl(oracle3dmhd* o, double* dt, double* umach);

/* BCON (3dmhdsub.f:2639-2958) in place. */
void oracle_bcon(oracle3dmhd* o);

/* Horizontally averaged profiles (HORIZONTAL_MEAN, 3dmhdsub.f:3143-3223) of
 * the current state in the rows of mhd3d_profiles (include/mhd3d.h):
 * out[r*NPZ + (K-2)], K=2..NZ-1.  Sums run in the reference's order (J outer,
 * I inner) and are divided by FLOAT(NPX*NPY). */
void oracle_profiles(const oracle3dmhd* o, double* out);

/* OpenMP threads used by the sweeps (<=0: leave the runtime default). */
void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
