// dumpio.cpp -- the reference driver's dump and restart files, for hosts that
// are not the Fortran program (3dmhd.f:284-363 restart, 505-524 and
// 912-1009 dumps).
//
//   FOUT.dat0.NNNN  one file per rank NNNN (PEEXTN, 3dmhdsub.f:2960-2978),
//                   unformatted direct access, RECL = 8*NPX*(NPY/NPEY)*(NPZ/NPEZ)
//                   bytes; dump d (0-based) holds records nf*d+1 .. nf*d+nf:
//                   RU, RV, RW, TT, RO [, BX, BY, BZ], each the rank's interior
//                   (2:NX-1, 2:NY-1, 2:NZ-1) in Fortran order, REAL*8.
//   FOUT.par        unformatted direct access, RECL = 8*96: record d+1 is PAR1
//                   (IPAR(1:32) as reals, then PAR(1:64)) of dump d.
//   FOUT.lis        formatted direct access, RECL = 80: 80-character records,
//                   text padded with blanks to 79 characters and a newline;
//                   dump records IREC-6..IREC with IREC = 59 + 7*NIT/NSTEP0.
//
// Direct-access records have no markers, so a record is at (r-1)*RECL.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mhd3d_host.h"

namespace {

std::string pe_ext(int rank)
{
    char b[16];
    std::snprintf(b, sizeof b, "%04d", rank);
    return b;
}

bool write_at(const std::string& path, long long offset, const void* data, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "r+b");
    if (!f) f = std::fopen(path.c_str(), "w+b");
    if (!f) return false;
    bool ok = std::fseek(f, 0, SEEK_END) == 0;
    const long long end = ok ? std::ftell(f) : -1;
    if (ok && end < offset) {   // a gap: the unwritten records read as zero bytes
        std::vector<char> z((size_t)(offset - end), 0);
        ok = std::fwrite(z.data(), 1, z.size(), f) == z.size();
    }
    ok = ok && std::fseek(f, (long)offset, SEEK_SET) == 0 && std::fwrite(data, 1, n, f) == n;
    return std::fclose(f) == 0 && ok;
}

bool read_at(const std::string& path, long long offset, void* data, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const bool ok = std::fseek(f, (long)offset, SEEK_SET) == 0 && std::fread(data, 1, n, f) == n;
    std::fclose(f);
    return ok;
}

// Fortran 1PD10.4 (one digit before the point, 4 after, D exponent)
std::string fmt_1pd10_4(double x)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.4E", x);
    std::string s(b);
    const size_t e = s.find('E');
    const int ex = std::atoi(s.c_str() + e + 1);
    std::string mant = s.substr(0, e);
    char t[32];
    if (ex >= -99 && ex <= 99) std::snprintf(t, sizeof t, "D%c%02d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    else std::snprintf(t, sizeof t, "%c%03d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    std::string out = mant + t;
    if (out.size() > 10) return std::string(10, '*');
    return std::string(10 - out.size(), ' ') + out;
}

// one .lis record: STRNG(1:JLEN), BLANKS(1:79-JLEN), CHAR(10)
std::string lis_record(const std::string& text)
{
    std::string r = text.substr(0, 79);
    r.resize(79, ' ');
    r.push_back('\n');
    return r;
}

}  // namespace

extern "C" {

void mhd3d_host_par1(const mhd3d_run_config* c, const int32_t ipar15[5], int32_t npe, int32_t npey, int32_t nit,
                     double dt, double par64, double par65, double par1[96])
{
    for (int i = 0; i < 96; ++i) par1[i] = 0.0;
    double* ip = par1;          // IPAR(1:32) as FLOAT (3dmhd.f:519-521)
    double* pa = par1 + 32;     // PAR(1:64) (3dmhd.f:522-524)
    auto fl = [](int32_t v) { return (double)(float)v; };
    for (int i = 0; i < 5; ++i) ip[i] = fl(ipar15[i]);
    ip[5] = 0.0;                // IXCON: periodic
    ip[6] = 0.0;                // IYCON: periodic
    ip[7] = fl(c->izcon);
    ip[8] = fl(c->itcon);
    ip[9] = fl(c->ibcon);
    ip[10] = fl(c->npx);
    ip[11] = fl(c->npy);
    ip[12] = fl(c->npz);
    ip[13] = fl(npe);
    ip[14] = fl(nit);           // 3dmhd.f:914
    ip[15] = fl(c->ntube);
    ip[16] = fl(c->ngrid);
    ip[17] = 1.0;               // NCOL
    ip[18] = 1.0;               // NROW
    ip[19] = 0.0;               // ID
    ip[20] = fl(npey);
    const double pv[] = {c->re,  c->pr,  c->theta, c->grav, c->ry,   c->ang,  c->rm,   c->beta,
                         c->pzp, c->sigma, c->polys, c->tp, c->tc,   c->xp,   c->yp,   0.0,
                         c->xmax, c->ymax, c->zmax, c->ampt, c->ampb, c->bfh,  c->bzp,  c->xx1,
                         c->xx2, c->yy1, c->yy2,  c->zz1,  c->zz2,  c->sff};
    for (int i = 0; i < (int)(sizeof pv / sizeof pv[0]); ++i) pa[i] = pv[i];
    pa[30] = dt;                // PAR(31): PAR1(63) = DT (3dmhd.f:915)
    pa[33] = 0.0;               // XCENT
    pa[34] = c->zcent;
    pa[35] = c->rmax;
    pa[36] = c->cmt;
    pa[37] = c->atube;
    const double gx[] = {c->xa, c->xb, c->xc, c->xd, c->ya, c->yb, c->yc, c->yd, c->za, c->zb, c->zc, c->zd};
    for (int i = 0; i < 12; ++i) pa[38 + i] = gx[i];
    pa[53] = c->gamma;          // PAR(54)
    pa[54] = c->hh;             // PAR(55)
    par1[63] = par64;           // PAR1(64): TIMT at the last step, else TIMI (3dmhd.f:916-921)
    par1[64] = par65;           // PAR1(65): 0 at the last step, else TIMC
}

int mhd3d_host_write_dump(const char* fout, int32_t ndump, const double par1[96], int32_t npx, int32_t npy,
                          int32_t npz, int32_t lmag, const double* ru, const double* rv, const double* rw,
                          const double* tt, const double* ro, const double* bx, const double* by, const double* bz,
                          double timt, double timc, double umach, double dt)
{
    if (!fout || !par1 || ndump < 0 || npx < 1 || npy < 1 || npz < 1) return MHD3D_ERR_ARG;
    const int nf = lmag ? 8 : 5;
    const double* f[8] = {ru, rv, rw, tt, ro, bx, by, bz};
    for (int i = 0; i < nf; ++i)
        if (!f[i]) return MHD3D_ERR_ARG;
    const std::string base(fout);
    const size_t NX = npx + 2, NY = npy + 2;
    const size_t recl = 8 * (size_t)npx * npy * npz;
    std::vector<double> rec((size_t)npx * npy * npz);
    for (int a = 0; a < nf; ++a) {
        size_t q = 0;
        for (int k = 2; k <= npz + 1; ++k)
            for (int j = 2; j <= npy + 1; ++j)
                for (int i = 2; i <= npx + 1; ++i) rec[q++] = f[a][(i - 1) + NX * ((j - 1) + NY * (k - 1))];
        const long long r = (long long)nf * ndump + a + 1;
        if (!write_at(base + ".dat0." + pe_ext(0), (r - 1) * (long long)recl, rec.data(), recl)) return MHD3D_ERR_ARG;
    }
    if (!write_at(base + ".par", (long long)ndump * 8 * 96, par1, 8 * 96)) return MHD3D_ERR_ARG;
    // the seven log records of a dump (3dmhd.f:958-1001)
    const int nit = (int)std::lround(par1[14]);
    const int nstep0 = std::max(1, (int)std::lround(par1[3]));
    const long long irec = 59 + 7LL * nit / nstep0;
    char b[128];
    std::string lines[7];
    lines[0] = lis_record(std::string(78, ' '));                                 // 4001
    std::snprintf(b, sizeof b, "     Iteration %7d completed", nit);            // 4053
    lines[1] = lis_record(b);
    lines[2] = lis_record("     " + std::string(35, '-'));                       // 4054
    lines[3] = lis_record("     Total simulation time:   " + fmt_1pd10_4(timt));  // 4055
    lines[4] = lis_record("     Present simulation time: " + fmt_1pd10_4(timc));  // 4056
    lines[5] = lis_record("     Maximum Mach number:     " + fmt_1pd10_4(umach)); // 4057
    lines[6] = lis_record("     Present time step:       " + fmt_1pd10_4(dt));   // 4058
    // records before the first dump that the Fortran host would have written read as blank lines
    const std::string lis = base + ".lis";
    {
        FILE* fl = std::fopen(lis.c_str(), "rb");
        long long have = 0;
        if (fl) {
            std::fseek(fl, 0, SEEK_END);
            have = std::ftell(fl) / 80;
            std::fclose(fl);
        }
        const std::string blank = lis_record("");
        for (long long r = have + 1; r < irec - 6; ++r)
            if (!write_at(lis, (r - 1) * 80, blank.data(), 80)) return MHD3D_ERR_ARG;
    }
    for (int i = 0; i < 7; ++i)
        if (!write_at(lis, (irec - 7 + i) * 80, lines[i].data(), 80)) return MHD3D_ERR_ARG;
    return MHD3D_OK;
}

int mhd3d_host_read_dump(const char* finp, int32_t nstart, int32_t npey, int32_t npez, int32_t lmag, int32_t npx,
                         int32_t npy, int32_t npz, double par1[96], double* ru, double* rv, double* rw, double* tt,
                         double* ro, double* bx, double* by, double* bz)
{
    if (!finp || nstart < 1 || npey < 1 || npez < 1 || npy % npey || npz % npez) return MHD3D_ERR_ARG;
    const int nf = lmag ? 8 : 5;
    double* f[8] = {ru, rv, rw, tt, ro, bx, by, bz};
    for (int i = 0; i < nf; ++i)
        if (!f[i]) return MHD3D_ERR_ARG;
    const std::string base(finp);
    double p[96];
    // size check against record 1 (3dmhd.f:300-317)
    if (!read_at(base + ".par", 0, p, sizeof p)) return MHD3D_ERR_ARG;
    const long nx1 = std::lround(p[10]);
    const long ny1 = std::lround(p[11]) / std::lround(p[20]);
    const long nz1 = std::lround(p[12]) / std::lround(p[13] / p[20]);
    const int nyr = npy / npey, nzr = npz / npez;
    if (nx1 != npx || ny1 != nyr || nz1 != nzr || std::lround(p[20]) != npey) return MHD3D_ERR_ARG;
    if (!read_at(base + ".par", (long long)(nstart - 1) * 8 * 96, p, sizeof p)) return MHD3D_ERR_ARG;
    if (par1) std::memcpy(par1, p, sizeof p);
    const size_t NX = npx + 2, NY = npy + 2, NZ = npz + 2;
    const size_t recl = 8 * (size_t)npx * nyr * nzr;
    std::vector<double> rec((size_t)npx * nyr * nzr);
    for (int a = 0; a < nf; ++a) std::memset(f[a], 0, sizeof(double) * NX * NY * NZ);
    for (int r = 0; r < npey * npez; ++r) {
        const int mypey = r % npey, mypez = r / npey;
        const std::string fn = base + ".dat0." + pe_ext(r);
        for (int a = 0; a < nf; ++a) {
            const long long rr = (long long)nf * (nstart - 1) + a + 1;
            if (!read_at(fn, (rr - 1) * (long long)recl, rec.data(), recl)) return MHD3D_ERR_ARG;
            size_t q = 0;
            for (int k = 0; k < nzr; ++k)
                for (int j = 0; j < nyr; ++j)
                    for (int i = 0; i < npx; ++i) {
                        const size_t I = i + 1, J = mypey * nyr + j + 1, K = mypez * nzr + k + 1;
                        f[a][I + NX * (J + NY * K)] = rec[q++];
                    }
        }
    }
    // periodic halos as COMMUNICATE leaves them (3dmhd.f:365); the z ghost
    // planes, which a restart leaves undefined, take the wall planes' values
    for (int a = 0; a < nf; ++a) {
        double* v = f[a];
        for (size_t K = 1; K <= (size_t)npz; ++K) {
            for (size_t J = 1; J <= (size_t)npy; ++J) {
                v[0 + NX * (J + NY * K)] = v[npx + NX * (J + NY * K)];
                v[(NX - 1) + NX * (J + NY * K)] = v[1 + NX * (J + NY * K)];
            }
            std::memcpy(v + NX * (0 + NY * K), v + NX * (npy + NY * K), sizeof(double) * NX);
            std::memcpy(v + NX * ((NY - 1) + NY * K), v + NX * (1 + NY * K), sizeof(double) * NX);
        }
        std::memcpy(v, v + NX * NY, sizeof(double) * NX * NY);
        std::memcpy(v + NX * NY * (NZ - 1), v + NX * NY * (NZ - 2), sizeof(double) * NX * NY);
    }
    return MHD3D_OK;
}

}  // extern "C"
