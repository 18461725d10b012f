/*
 * ref_harness.h -- run-time support for the C translation of the
 * reference's time-step routines (test infrastructure).
 *
 * The translation (generated into oracle/_ref/ by oracle/make_ref.py)
 * calls the functions declared here in place of MPI and of STOP.  Ranks
 * are forked processes; point-to-point messages go over socket pairs and
 * collectives over a process-shared barrier, so the reference's own
 * decomposition (NPEY x NPEZ ranks) runs unchanged.
 */
#ifndef REF_HARNESS_H
#define REF_HARNESS_H

#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* names from mpif.h used by the translated routines */
extern int MPI_COMM_WORLD, MPI_STATUS_SIZE, MPI_DOUBLE_PRECISION, MPI_FLOAT, MPI_MIN, MPI_MAX, MPI_SUM;

int ref_param_override(const char* name, void* dst, char type);
void ref_send(void* buf, int count, int type, int dest, int tag);
void ref_recv(void* buf, int count, int type, int src, int tag);
void ref_sendrecv(void* sbuf, int scount, int stype, int dest, int stag,
                  void* rbuf, int rcount, int rtype, int src, int rtag);
void ref_allreduce(void* in, void* out, int count, int type, int op);
void ref_bcast(void* buf, int count, int type, int root);
void ref_stop(const char* unit, int line);
void ref_finalize(void);

/* X**n with an integer exponent, expanded as gcc expands __builtin_powi */
static inline double ipow_d2(double x) { return x * x; }
static inline double ipow_d3(double x) { return x * x * x; }
static inline double ipow_d4(double x) { double t = x * x; return t * t; }
static inline float ipow_f2(float x) { return x * x; }
static inline float ipow_f3(float x) { return x * x * x; }
static inline float ipow_f4(float x) { float t = x * x; return t * t; }
static inline int ipow_i2(int x) { return x * x; }
static inline int ipow_i3(int x) { return x * x * x; }
static inline int ipow_i4(int x) { return x * x * x * x; }
static inline double ipow_dn(double x, int n)
{
    unsigned m = n < 0 ? (unsigned)(-n) : (unsigned)n;
    double r = (m % 2) ? x : 1.0;
    while (m >>= 1) { x = x * x; if (m % 2) r = r * x; }
    return n < 0 ? 1.0 / r : r;
}
static inline float ipow_fn(float x, int n)
{
    unsigned m = n < 0 ? (unsigned)(-n) : (unsigned)n;
    float r = (m % 2) ? x : 1.0f;
    while (m >>= 1) { x = x * x; if (m % 2) r = r * x; }
    return n < 0 ? 1.0f / r : r;
}
static inline int ipow_in(int x, int n)
{
    int r = 1;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

/* MIN/MAX of gfortran for ordered operands */
static inline double fmin_d(double a, double b) { return b < a ? b : a; }
static inline double fmax_d(double a, double b) { return b > a ? b : a; }
static inline float fmin_f(float a, float b) { return b < a ? b : a; }
static inline float fmax_f(float a, float b) { return b > a ? b : a; }
static inline int fmin_i(int a, int b) { return b < a ? b : a; }
static inline int fmax_i(int a, int b) { return b > a ? b : a; }

/* provided by the generated translation */
void ref_params_init(void);
void ref_commons_alloc(void);
size_t ref_common_size(const char* name);
void* ref_common_ptr(const char* name);
void sub_STEP(void);
void sub_FLUXES(void);
void sub_BCON(void);
void sub_COMMUNICATE(void);
void sub_HORIZONTAL_MEAN(double* VARM, double* VAR);

#endif
