/*
 * ref_harness.c -- driver for the translated reference time step
 * (test infrastructure; the CPU "reference" baseline).
 *
 * Usage: ref3dmhd IN OUT
 *
 * IN holds: "R3DI", version, npey, npez, nsteps, mode, [warmup, version>=2], the mhd3d_params
 * struct, the 14 global COMMON/AJACOBI+CPEN arrays and the global fields
 * (Fortran (NPX+2,NPY+2,NPZ+2), as the single-domain driver holds them
 * after COMMUNICATE).  The harness forks NPEY*NPEZ ranks, gives each the
 * slab the reference's decomposition assigns it (3dmhd.f:87-88,
 * 3dmhdparam.f:17-19), sets the COMMON blocks the way the main program does
 * (3dmhd.f:105-240), runs CALL STEP nsteps times (mode 0) or CALL FLUXES
 * once (mode 1), and gathers the result into OUT.  Mode 2 averages the
 * diagnostic quantities of include/mhd3d.h (MHD3D_PROF_*) with the
 * reference's own HORIZONTAL_MEAN (3dmhdsub.f:3143-3223) on every rank and
 * writes the MHD3D_NPROF x NPZ profile rows instead of fields.
 *
 * MPI is emulated: SEND/RECV/SENDRECV over socket pairs between the ranks
 * that talk to each other in COMM_MPI, ALLREDUCE/BCAST through shared
 * memory and a process-shared barrier.  Reductions are MIN/MAX/SUM over
 * ranks in rank order.
 */
#define _GNU_SOURCE
#include "ref_harness.h"
#include "../include/mhd3d.h"

#include <errno.h>
#include <poll.h>
#include <pthread.h>
#include <stdint.h>
#include <sys/mman.h>
#include <sys/socket.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

int MPI_COMM_WORLD = 91, MPI_STATUS_SIZE = 8, MPI_DOUBLE_PRECISION = 1, MPI_FLOAT = 2,
    MPI_MIN = 11, MPI_MAX = 12, MPI_SUM = 13;

/* ---------------------------------------------------------------- */
static int g_rank, g_size, g_npey, g_npez;
static int* g_fd;                 /* g_fd[peer] = socket to peer or -1 */

#define MAXRED 128
typedef struct {
    pthread_barrier_t bar;
    double slot[1];               /* g_size * MAXRED doubles */
} shared_t;
static shared_t* g_sh;

/* overrides of 3dmhdparam.f PARAMETERs */
typedef struct { const char* name; double val; } ovr_t;
static ovr_t g_ovr[64];
static int g_novr;

static void ovr_set(const char* n, double v) { g_ovr[g_novr].name = n; g_ovr[g_novr].val = v; g_novr++; }

int ref_param_override(const char* name, void* dst, char type)
{
    for (int i = 0; i < g_novr; ++i)
        if (!strcmp(g_ovr[i].name, name)) {
            if (type == 'd') *(double*)dst = g_ovr[i].val;
            else *(int*)dst = (int)g_ovr[i].val;
            return 1;
        }
    return 0;
}

static void die(const char* msg)
{
    fprintf(stderr, "ref3dmhd rank %d: %s\n", g_rank, msg);
    _exit(2);
}

void ref_stop(const char* unit, int line)
{
    fprintf(stderr, "ref3dmhd rank %d: STOP in %s at line %d\n", g_rank, unit, line);
    _exit(3);
}

void ref_finalize(void) { /* followed by STOP in the reference */ }

static size_t tsize(int type) { return type == MPI_FLOAT ? 4 : 8; }

static void write_all(int fd, const void* p, size_t n)
{
    const char* c = (const char*)p;
    while (n) {
        ssize_t w = write(fd, c, n);
        if (w < 0) { if (errno == EINTR) continue; die("write"); }
        c += w; n -= (size_t)w;
    }
}

static void read_all(int fd, void* p, size_t n)
{
    char* c = (char*)p;
    while (n) {
        ssize_t r = read(fd, c, n);
        if (r < 0) { if (errno == EINTR) continue; die("read"); }
        if (r == 0) die("peer closed");
        c += r; n -= (size_t)r;
    }
}

static int peer_fd(int peer)
{
    if (peer < 0 || peer >= g_size || g_fd[peer] < 0) die("no channel to peer");
    return g_fd[peer];
}

void ref_send(void* buf, int count, int type, int dest, int tag)
{
    int fd = peer_fd(dest);
    int32_t hdr[2] = {tag, count};
    write_all(fd, hdr, sizeof(hdr));
    write_all(fd, buf, (size_t)count * tsize(type));
}

void ref_recv(void* buf, int count, int type, int src, int tag)
{
    int fd = peer_fd(src);
    int32_t hdr[2];
    read_all(fd, hdr, sizeof(hdr));
    if (hdr[0] != tag || hdr[1] != count) die("message tag/count mismatch");
    read_all(fd, buf, (size_t)count * tsize(type));
}

void ref_sendrecv(void* sbuf, int scount, int stype, int dest, int stag,
                  void* rbuf, int rcount, int rtype, int src, int rtag)
{
    /* progress the send and the receive together so that a chain of ranks
       in SENDRECV cannot block on full socket buffers */
    int sfd = peer_fd(dest), rfd = peer_fd(src);
    int32_t shdr[2] = {stag, scount}, rhdr[2];
    size_t sn = sizeof(shdr) + (size_t)scount * tsize(stype), so = 0;
    size_t rn = sizeof(rhdr) + (size_t)rcount * tsize(rtype), ro = 0;
    char* sb = (char*)malloc(sn);
    char* rb = (char*)malloc(rn);
    memcpy(sb, shdr, sizeof(shdr));
    memcpy(sb + sizeof(shdr), sbuf, sn - sizeof(shdr));
    while (so < sn || ro < rn) {
        struct pollfd pf[2];
        int np = 0, is = -1, ir = -1;
        if (so < sn) { pf[np].fd = sfd; pf[np].events = POLLOUT; is = np++; }
        if (ro < rn) { pf[np].fd = rfd; pf[np].events = POLLIN; ir = np++; }
        if (poll(pf, (nfds_t)np, 600000) <= 0) die("sendrecv poll timeout");
        if (is >= 0 && (pf[is].revents & POLLOUT)) {
            ssize_t w = write(sfd, sb + so, sn - so);
            if (w < 0 && errno != EAGAIN && errno != EINTR) die("sendrecv write");
            if (w > 0) so += (size_t)w;
        }
        if (ir >= 0 && (pf[ir].revents & (POLLIN | POLLHUP))) {
            ssize_t r = read(rfd, rb + ro, rn - ro);
            if (r == 0) die("sendrecv peer closed");
            if (r < 0 && errno != EAGAIN && errno != EINTR) die("sendrecv read");
            if (r > 0) ro += (size_t)r;
        }
    }
    memcpy(rhdr, rb, sizeof(rhdr));
    if (rhdr[0] != rtag || rhdr[1] != rcount) die("sendrecv tag/count mismatch");
    memcpy(rbuf, rb + sizeof(rhdr), rn - sizeof(rhdr));
    free(sb);
    free(rb);
}

static void barrier(void) { pthread_barrier_wait(&g_sh->bar); }

void ref_allreduce(void* in, void* out, int count, int type, int op)
{
    if (type != MPI_DOUBLE_PRECISION || count > MAXRED) die("allreduce type/count");
    double* mine = g_sh->slot + (size_t)g_rank * MAXRED;
    memcpy(mine, in, (size_t)count * sizeof(double));
    barrier();
    double res[MAXRED];
    for (int c = 0; c < count; ++c) {
        double v = g_sh->slot[c];
        for (int r = 1; r < g_size; ++r) {
            double w = g_sh->slot[(size_t)r * MAXRED + c];
            if (op == MPI_MIN) v = w < v ? w : v;
            else if (op == MPI_MAX) v = w > v ? w : v;
            else v = v + w;
        }
        res[c] = v;
    }
    barrier();
    memcpy(out, res, (size_t)count * sizeof(double));
}

void ref_bcast(void* buf, int count, int type, int root)
{
    if (type != MPI_DOUBLE_PRECISION || count > MAXRED) die("bcast type/count");
    if (g_rank == root) memcpy(g_sh->slot, buf, (size_t)count * sizeof(double));
    barrier();
    if (g_rank != root) memcpy(buf, g_sh->slot, (size_t)count * sizeof(double));
    barrier();
}

/* ---------------------------------------------------------------- */
static void* xread(FILE* f, size_t n)
{
    void* p = malloc(n ? n : 1);
    if (n && fread(p, 1, n, f) != n) { fprintf(stderr, "ref3dmhd: short input\n"); exit(2); }
    return p;
}

static double now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void set_d(const char* n, double v)
{
    double* p = (double*)ref_common_ptr(n);
    if (!p) die(n);
    *p = v;
}

static void set_i(const char* n, int v)
{
    int* p = (int*)ref_common_ptr(n);
    if (!p) die(n);
    *p = v;
}

int main(int argc, char** argv)
{
    if (argc != 3) { fprintf(stderr, "usage: ref3dmhd IN OUT\n"); return 2; }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 2; }
    char magic[4];
    int32_t hdr[6] = {0};
    if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "R3DI", 4)) { fprintf(stderr, "bad input\n"); return 2; }
    if (fread(hdr, sizeof(int32_t), 5, f) != 5) return 2;
    if (hdr[0] >= 2 && fread(hdr + 5, sizeof(int32_t), 1, f) != 1) return 2;
    const int npey = hdr[1], npez = hdr[2], nsteps = hdr[3], mode = hdr[4], warmup = hdr[5];
    mhd3d_params P;
    if (fread(&P, sizeof(P), 1, f) != 1) return 2;
    const int NXg = P.npx + 2, NYg = P.npy + 2, NZg = P.npz + 2;
    const size_t ng = (size_t)NXg * NYg * NZg;
    double* met[14];
    const int mlen[14] = {NXg, NXg, NXg, NXg, NYg, NYg, NYg, NYg, NZg, NZg, NZg, NZg, NZg, NZg};
    for (int a = 0; a < 14; ++a) met[a] = (double*)xread(f, (size_t)mlen[a] * sizeof(double));
    const int nfld = P.lmag ? 8 : 5;
    double* fin[8] = {0};
    for (int a = 0; a < nfld; ++a) fin[a] = (double*)xread(f, ng * sizeof(double));
    fclose(f);
    if (npey < 1 || npez < 1 || P.npy % npey || P.npz % npez) { fprintf(stderr, "bad decomposition\n"); return 2; }

    g_npey = npey;
    g_npez = npez;
    g_size = npey * npez;
    const int nry = P.npy / npey, nrz = P.npz / npez;

    /* PARAMETER overrides (3dmhdparam.f): the single-domain run expressed
       as the reference's compile-time configuration */
    ovr_set("LROT", P.lrot); ovr_set("LMAG", P.lmag); ovr_set("LPOT", 0); ovr_set("LREM", 0); ovr_set("LSHR", 0);
    ovr_set("NPEY", npey); ovr_set("NPEZ", npez);
    ovr_set("NPX", P.npx); ovr_set("NPY", P.npy); ovr_set("NPZ", P.npz);
    ovr_set("IXCON", 0); ovr_set("IYCON", 0); ovr_set("IZCON", P.izcon); ovr_set("ITCON", P.itcon);
    ovr_set("IBCON", P.ibcon); ovr_set("SFF", P.sf); ovr_set("ID", 0); ovr_set("DH", 0.0); ovr_set("DV", 0.0);
    ovr_set("IWORD", 8); ovr_set("NGRID", 0);

    /* shared output: gathered global fields (8 + 8 flux arrays) and scalars */
    size_t outn = 16 * ng + 16;
    double* gout = (double*)mmap(NULL, outn * sizeof(double), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    size_t shn = sizeof(shared_t) + (size_t)g_size * MAXRED * sizeof(double);
    g_sh = (shared_t*)mmap(NULL, shn, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (gout == MAP_FAILED || g_sh == MAP_FAILED) { perror("mmap"); return 2; }
    pthread_barrierattr_t ba;
    pthread_barrierattr_init(&ba);
    pthread_barrierattr_setpshared(&ba, PTHREAD_PROCESS_SHARED);
    pthread_barrier_init(&g_sh->bar, &ba, (unsigned)g_size);

    /* channels between the ranks COMM_MPI pairs: z neighbours, y neighbours,
       y periodic ends (3dmhdsub.f:3045-3128) */
    int* chan = (int*)malloc(sizeof(int) * (size_t)g_size * g_size);
    for (int q = 0; q < g_size * g_size; ++q) chan[q] = -1;
    for (int a = 0; a < g_size; ++a)
        for (int b = a + 1; b < g_size; ++b) {
            int ay = a % npey, az = a / npey, by = b % npey, bz = b / npey;
            int need = (ay == by && (bz - az == 1)) || (az == bz && (by - ay == 1 || by - ay == npey - 1));
            if (!need) continue;
            int sv[2];
            if (socketpair(AF_UNIX, SOCK_STREAM, 0, sv)) { perror("socketpair"); return 2; }
            chan[a * g_size + b] = sv[0];
            chan[b * g_size + a] = sv[1];
        }

    for (int r = 0; r < g_size; ++r) {
        pid_t pid = fork();
        if (pid < 0) { perror("fork"); return 2; }
        if (pid > 0) continue;
        /* ---------------- rank r ---------------- */
        g_rank = r;
        g_fd = (int*)malloc(sizeof(int) * (size_t)g_size);
        for (int q = 0; q < g_size; ++q) g_fd[q] = chan[r * g_size + q];
        const int mypey = r % npey, mypez = r / npey;
        ref_params_init();
        ref_commons_alloc();
        const int NX = NXg, NY = nry + 2, NZ = nrz + 2;
        const int joff = mypey * nry, koff = mypez * nrz;
        /* COMMON/COMMUN, BCT, GRID, RUNGKU, CPAR, CROT, CMAG, CPEN, CPER, CTIM, ITER, RELAX */
        set_i("MYPE", r); set_i("MYPEY", mypey); set_i("MYPEZ", mypez); set_i("MPISIZE", MPI_DOUBLE_PRECISION);
        set_i("IXC", 0); set_i("IYC", 0); set_i("IZC", P.izcon); set_i("ITC", P.itcon); set_i("IBC", P.ibcon);
        set_d("HX", P.hx); set_d("H2X", P.h2x); set_d("HY", P.hy); set_d("H2Y", P.h2y);
        set_d("HZ", P.hz); set_d("H2Z", P.h2z); set_d("C13", P.c13); set_d("C23", P.c23); set_d("C43", P.c43);
        set_d("GAM1", P.gam1); set_d("GAM2", P.gam2); set_d("GAM3", P.gam3);
        set_d("ZETA1", P.zeta1); set_d("ZETA2", P.zeta2);
        set_d("CV", P.cv); set_d("OCV", P.ocv); set_d("ORE", P.ore); set_d("RE", P.re); set_d("REPR", P.repr);
        set_d("THETA", P.theta); set_d("GRAV", P.grav); set_d("SF", P.sf); set_d("GAMMA", P.gamma);
        set_d("OMX", P.omx); set_d("OMZ", P.omz);
        set_d("ORM", P.orm); set_d("RM", P.rm); set_d("OBETA", P.obeta);
        set_d("TB", P.tb); set_d("PZP", 0.0);
        set_d("TP", P.tp); set_d("TC", P.tc); set_d("XP", P.xp); set_d("YP", P.yp); set_d("HH", P.hh);
        set_d("TIMI", P.timi); set_d("TIMC", P.timc); set_d("TIMT", 0.0);
        set_i("NIT", 0);
        set_d("RLAX", 0.0);
        /* COMMON/AJACOBI and CPEN arrays: this rank's slices */
        const char* mx[4] = {"EXX", "DXXDX", "D2XXDX2", "DDX"};
        const char* my[4] = {"WYY", "DYYDY", "D2YYDY2", "DDY"};
        const char* mz[6] = {"ZEE", "DZZDZ", "D2ZZDZ2", "DDZ", "RKAPA", "DKAPA"};
        for (int a = 0; a < 4; ++a) {
            double* p = (double*)ref_common_ptr(mx[a]);
            for (int i = 0; i < NX; ++i) p[i] = met[a][i];
            p = (double*)ref_common_ptr(my[a]);
            for (int j = 0; j < NY; ++j) p[j] = met[4 + a][j + joff];
        }
        for (int a = 0; a < 6; ++a) {
            double* p = (double*)ref_common_ptr(mz[a]);
            for (int k = 0; k < NZ; ++k) p[k] = met[8 + a][k + koff];
        }
        /* COMMON/BIG fields */
        const char* fname[8] = {"RU", "RV", "RW", "TT", "RO", "BX", "BY", "BZ"};
        double* loc[8];
        for (int a = 0; a < nfld; ++a) {
            loc[a] = (double*)ref_common_ptr(fname[a]);
            for (int k = 0; k < NZ; ++k)
                for (int j = 0; j < NY; ++j)
                    memcpy(loc[a] + (size_t)NX * (j + (size_t)NY * k),
                           fin[a] + (size_t)NXg * ((j + joff) + (size_t)NYg * (k + koff)), sizeof(double) * NX);
        }
        if (mode == 2) {
            /* per-cell quantities of the flux diagnostics (1651-1661) on the
               local array, averaged by HORIZONTAL_MEAN; WW1=TT-TTM (1524-1528) */
            const size_t nl = (size_t)NX * NY * NZ;
            const double *ru = loc[0], *rv = loc[1], *rw = loc[2], *tt = loc[3], *ro = loc[4];
            double* q = (double*)calloc(nl, sizeof(double));
            double* m = (double*)calloc((size_t)NZ * MHD3D_NPROF, sizeof(double));
            sub_HORIZONTAL_MEAN(m + MHD3D_PROF_RHO * NZ, ro);
            sub_HORIZONTAL_MEAN(m + MHD3D_PROF_T * NZ, tt);
            const double* ttm = m + MHD3D_PROF_T * NZ;
            for (int pass = 0; pass < 4; ++pass) {
                for (int k = 1; k <= NZ; ++k)
                    for (int j = 1; j <= NY; ++j)
                        for (int i = 1; i <= NX; ++i) {
                            const size_t c = (size_t)(i - 1) + (size_t)NX * ((size_t)(j - 1) + (size_t)NY * (k - 1));
                            const double ri = 1.0 / ro[c];
                            const double u = ru[c] * ri, v = rv[c] * ri, w = rw[c] * ri;
                            if (pass == 0) q[c] = 0.5 * ro[c] * (u * u + v * v + w * w);
                            else if (pass == 1) q[c] = 2.5 * ro[c] * tt[c];
                            else if (pass == 2) q[c] = -rw[c] * (2.5 * (tt[c] - ttm[k - 1]) + 0.5 * (u * u + v * v + w * w));
                            else q[c] = P.lmag ? 0.5 * (loc[5][c] * loc[5][c] + loc[6][c] * loc[6][c] + loc[7][c] * loc[7][c]) : 0.0;
                        }
                const int row = pass == 0 ? MHD3D_PROF_KE : pass == 1 ? MHD3D_PROF_ENTH : pass == 2 ? MHD3D_PROF_FCONV : MHD3D_PROF_ME;
                sub_HORIZONTAL_MEAN(m + row * NZ, q);
            }
            if (mypey == 0)
                for (int r2 = 0; r2 < MHD3D_NPROF; ++r2)
                    for (int k = 2; k <= NZ - 1; ++k)
                        gout[(size_t)r2 * P.npz + (size_t)(k - 2 + koff)] = m[(size_t)r2 * NZ + (k - 1)];
            free(q);
            free(m);
            barrier();
            _exit(0);
        }
        if (mode == 0)
            for (int s = 0; s < warmup; ++s) sub_STEP();
        barrier();
        double t0 = now();
        if (mode == 0) {
            for (int s = 0; s < nsteps; ++s) sub_STEP();
        } else {
            sub_FLUXES();
        }
        barrier();
        double t1 = now();
        /* gather: interior J and K rows of every rank, plus the wall ghost planes */
        const char* oname_step[8] = {"RU", "RV", "RW", "TT", "RO", "BX", "BY", "BZ"};
        const char* oname_flux[8] = {"FU", "FV", "FW", "FR", "FT", "WW1", "WW2", "WW3"};
        const char** on = mode == 0 ? oname_step : oname_flux;
        for (int a = 0; a < nfld; ++a) {
            double* src = (double*)ref_common_ptr(on[a]);
            double* dst = gout + (size_t)a * ng;
            int k0 = (mypez == 0) ? 0 : 1, k1 = (mypez == npez - 1) ? NZ - 1 : NZ - 2;
            for (int k = k0; k <= k1; ++k)
                for (int j = 1; j <= NY - 2; ++j)
                    memcpy(dst + (size_t)NXg * ((j + joff) + (size_t)NYg * (k + koff)),
                           src + (size_t)NX * (j + (size_t)NY * k), sizeof(double) * NX);
        }
        if (r == 0) {
            double* sc = gout + 16 * ng;
            sc[0] = *(double*)ref_common_ptr("DT");
            sc[1] = *(double*)ref_common_ptr("TIMC");
            sc[2] = *(double*)ref_common_ptr("TIMT");
            sc[3] = *(double*)ref_common_ptr("UMACH");
            sc[4] = (double)*(int*)ref_common_ptr("NIT");
            sc[5] = t1 - t0;
        }
        _exit(0);
    }
    for (int q = 0; q < g_size * g_size; ++q)
        if (chan[q] >= 0) close(chan[q]);
    int failed = 0;
    for (int r = 0; r < g_size; ++r) {
        int st;
        if (wait(&st) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) failed = 1;
    }
    if (failed) { fprintf(stderr, "ref3dmhd: a rank failed\n"); return 3; }
    if (mode == 2) {
        /* FRADM from the gathered TTM (3dmhdsub.f:1663-1676) */
        const int npz = P.npz;
        const double* ttm = gout + (size_t)MHD3D_PROF_T * npz;
        for (int k = 0; k < npz; ++k) {
            const int K = k + 2;
            double d;
            if (k == 0) d = -3.0 * ttm[0] + 4.0 * ttm[1] - ttm[2];
            else if (k == npz - 1) d = 3.0 * ttm[npz - 1] - 4.0 * ttm[npz - 2] + ttm[npz - 3];
            else d = ttm[k + 1] - ttm[k - 1];
            gout[(size_t)MHD3D_PROF_FRAD * npz + k] = d * P.hz * met[9][K - 1] * met[12][K - 1] / P.repr;
        }
        FILE* o = fopen(argv[2], "wb");
        if (!o) { perror(argv[2]); return 2; }
        fwrite("R3DP", 1, 4, o);
        fwrite(gout, sizeof(double), (size_t)MHD3D_NPROF * npz, o);
        fclose(o);
        return 0;
    }
    /* periodic y halo rows as COMMUNICATE leaves them (x halos came with the rows) */
    for (int a = 0; a < nfld; ++a) {
        double* v = gout + (size_t)a * ng;
        for (int k = 0; k < NZg; ++k) {
            memcpy(v + (size_t)NXg * (0 + (size_t)NYg * k), v + (size_t)NXg * ((NYg - 2) + (size_t)NYg * k), sizeof(double) * NXg);
            memcpy(v + (size_t)NXg * ((NYg - 1) + (size_t)NYg * k), v + (size_t)NXg * (1 + (size_t)NYg * k), sizeof(double) * NXg);
        }
    }
    FILE* o = fopen(argv[2], "wb");
    if (!o) { perror(argv[2]); return 2; }
    int32_t ohdr[2] = {0, (int32_t)gout[16 * ng + 4]};
    fwrite("R3DO", 1, 4, o);
    fwrite(ohdr, sizeof(int32_t), 2, o);
    fwrite(gout + 16 * ng, sizeof(double), 6, o);
    for (int a = 0; a < nfld; ++a) fwrite(gout + (size_t)a * ng, sizeof(double), ng, o);
    fclose(o);
    return 0;
}
