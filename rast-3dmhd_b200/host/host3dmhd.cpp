// host3dmhd.cpp -- host-side mirror of the reference driver's initialisation.
//
// Everything here runs once, before the first step, exactly where the
// Fortran driver runs it (3dmhd.f:105-496).  Literal semantics follow
// gfortran: an E-exponent literal is REAL(4), so e.g. C13=1.0E00/3.0E00
// is a float division widened to double, FLOAT() is REAL(4), and a
// REAL(4) operand meeting a REAL*8 one is widened first.
#include "../../include/mhd3d_host.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

inline double f2d(float x) { return static_cast<double>(x); }

struct Index3 {
    int nx, ny, nz;
    size_t operator()(int i, int j, int k) const  // Fortran 1-based (I,J,K)
    {
        return static_cast<size_t>(i - 1) + static_cast<size_t>(nx) * (static_cast<size_t>(j - 1) + static_cast<size_t>(ny) * static_cast<size_t>(k - 1));
    }
};

// MKGRID (3dmhdsub.f:17-175) for one coordinate; icoord 1,2,3 = x,y,z.
struct Map {
    double sphys, dssds, d2ssds2;
};

Map mkgrid(const mhd3d_run_config* c, double scode, int icoord)
{
    Map m{};
    double smax = icoord == 1 ? c->xmax : icoord == 2 ? c->ymax : c->zmax;
    int ngrid = c->ngrid;
    if (ngrid == MHD3D_GRID_TANH_Z && icoord != 3) ngrid = MHD3D_GRID_UNIFORM;
    switch (ngrid) {
    case MHD3D_GRID_UNIFORM:  // CASE(0), 3dmhdsub.f:32-48
        m.sphys = scode * smax;
        m.dssds = 1.0 / smax;
        m.d2ssds2 = 0.0;
        break;
    case MHD3D_GRID_ARCTAN: {  // CASE(1), 3dmhdsub.f:67-97
        double s1 = icoord == 1 ? c->xx1 : icoord == 2 ? c->yy1 : c->zz1;
        double s2 = icoord == 1 ? c->xx2 : icoord == 2 ? c->yy2 : c->zz2;
        double a1 = (s2 - s1) / smax;
        double a3 = std::atan(s1);
        double a2 = std::atan(s2) - a3;
        if (scode == 0.0) m.sphys = 0.0;
        else if (scode == 1.0) m.sphys = smax;
        else m.sphys = (std::tan(a2 * scode + a3) - s1) / a1;
        double q = s1 + a1 * m.sphys;
        m.dssds = a1 / a2 / (1.0 + q * q);
        double d = 1.0 + q * q;
        m.d2ssds2 = -(2.0 * (a1 * a1) * q / a2 / (d * d));
        break;
    }
    case MHD3D_GRID_DIP: {  // CASE(2), 3dmhdsub.f:101-161
        const double PI = f2d(2.0f * std::asin(1.0f));
        double A = icoord == 1 ? c->xa : icoord == 2 ? c->ya : c->za;
        double B = icoord == 1 ? c->xb : icoord == 2 ? c->yb : c->zb;
        double C = icoord == 1 ? c->xc : icoord == 2 ? c->yc : c->zc;
        double D = icoord == 1 ? c->xd : icoord == 2 ? c->yd : c->zd;
        if (C <= f2d(1.0e-9f)) {
            m.sphys = scode * smax;
            m.dssds = 1.0 / smax;
            m.d2ssds2 = 0.0;
        } else {
            double sh = (1.0 - D) * PI / (D * std::atan((A - B) * C) + 2.0 * std::atan(B * C) - D * std::atan((A + B) * C));
            double sk = 2.0 * C * PI * smax /
                        (2.0 * C * PI + sh * (2.0 * C * (std::atan((A - B) * C) * (A - B) - std::atan((A + B) * C) * (A + B)
                                                        + std::atan((A - B - 1.0) * C) + std::atan((A + B - 1.0) * C) * (A + B - 1.0)
                                                        + std::atan((1.0 - A + B) * C) * (A - B))
                                              - std::log(1.0 + (A - B) * (A - B) * (C * C)) + std::log(1.0 + (A + B) * (A + B) * (C * C))
                                              - std::log(1.0 + (A + B - 1.0) * (A + B - 1.0) * (C * C))
                                              + std::log(1.0 + (1.0 - A + B) * (1.0 - A + B) * (C * C))));
            m.dssds = 1.0 / (sk * (1.0 + sh / PI * (std::atan(C * (scode - A - B)) + std::atan(C * (A - scode - B)))));
            double dd3 = m.dssds * m.dssds * m.dssds;
            m.d2ssds2 = -dd3 * C * sh * sk / PI *
                        (1.0 / (1.0 + (C * C) * ((A + B - scode) * (A + B - scode))) - 1.0 / (1.0 + (C * C) * ((A - B - scode) * (A - B - scode))));
            m.sphys = sk / (2.0 * C * PI) *
                      (2.0 * C * PI * scode + sh * (2.0 * C * (std::atan((A - B) * C) * (A - B) - std::atan((A + B) * C) * (A + B)
                                                             + std::atan((A - B - scode) * C) * scode + std::atan((A + B - scode) * C) * (A + B - scode)
                                                             + std::atan((scode - A + B) * C) * (A - B))
                                                   - std::log(1.0 + (A - B) * (A - B) * (C * C)) + std::log(1.0 + (A + B) * (A + B) * (C * C))
                                                   - std::log(1.0 + (A + B - scode) * (A + B - scode) * (C * C))
                                                   + std::log(1.0 + (scode - A + B) * (scode - A + B) * (C * C))));
        }
        if (scode == 0.0) m.sphys = 0.0;
        if (scode == 1.0) m.sphys = smax;
        break;
    }
    case MHD3D_GRID_TANH_Z: {  // project map for z: points clustered towards the top (s=0)
        double S = c->zstretch;
        double u = S * (1.0 - scode);
        double th = std::tanh(u), tS = std::tanh(S);
        double sech2 = 1.0 - th * th;
        if (scode == 0.0) m.sphys = 0.0;
        else if (scode == 1.0) m.sphys = smax;
        else m.sphys = smax * (1.0 - th / tS);
        double dzds = smax * S * sech2 / tS;
        double d2zds2 = smax * 2.0 * S * S * sech2 * th / tS;
        m.dssds = 1.0 / dzds;
        m.d2ssds2 = -d2zds2 * m.dssds * m.dssds * m.dssds;
        break;
    }
    default:
        m.sphys = std::nan("");
        m.dssds = std::nan("");
        m.d2ssds2 = std::nan("");
    }
    return m;
}

// Thermal conductivity profile (3dmhd.f:266-279), non-LREM.
void kappa_profile(const mhd3d_run_config* c, double z, double* rk, double* drk)
{
    if (c->pzp == 0.0) {
        *rk = 1.0;
        *drk = 0.0;
        return;
    }
    double rkapst = c->grav == 0.0 ? 1.0 : (c->polys + 1.0) * c->theta / c->grav;
    double x = (z - c->pzp) / c->sigma;
    *rk = 1.0 + (rkapst - 1.0) / 2.0 * (1.0 + std::tanh(x));
    double ch = std::cosh(x);
    *drk = (rkapst - 1.0) / 2.0 / c->sigma / (ch * ch);
}

// Hydrostatic profile T(s), P(s) of STATIC (3dmhdsub.f:470-508):
// dF/ds = THETA/RKAP/DZZDZ, dlnP/ds = GRAV/(1+F)/DZZDZ (DERIVS, 659-685).
void static_profile(const mhd3d_run_config* c, int npz, std::vector<double>& T, std::vector<double>& R)
{
    T.assign(npz + 1, 0.0);
    R.assign(npz + 1, 0.0);
    T[1] = 1.0;
    R[1] = 1.0;
    if (c->pzp == 0.0) {
        // kappa = 1: F = THETA*z and lnP = (GRAV/THETA) ln(1+THETA z) exactly.
        float orz = 1.0f / static_cast<float>(npz - 1);
        for (int k = 2; k <= npz; ++k) {
            double s = (k == npz) ? 1.0 : f2d(static_cast<float>(k - 1)) * f2d(orz);
            double z = mkgrid(c, s, 3).sphys;
            double t = 1.0 + c->theta * z;
            double lnp = c->theta != 0.0 ? c->grav / c->theta * std::log(t) : c->grav * z;
            T[k] = t;
            R[k] = std::exp(lnp) / t;
        }
        return;
    }
    // General kappa(z): classical RK4 in the code coordinate, 256 substeps per interval.
    auto derivs = [&](double s, const double y[2], double dy[2]) {
        Map m = mkgrid(c, s, 3);
        double rk, drk;
        kappa_profile(c, m.sphys, &rk, &drk);
        dy[0] = c->theta / rk / m.dssds;
        dy[1] = c->grav / (1.0 + y[0]) / m.dssds;
    };
    double y[2] = {0.0, 0.0};
    const int sub = 256;
    double ds = 1.0 / (npz - 1) / sub;
    double s = 0.0;
    for (int k = 2; k <= npz; ++k) {
        for (int q = 0; q < sub; ++q) {
            double k1[2], k2[2], k3[2], k4[2], yt[2];
            derivs(s, y, k1);
            for (int v = 0; v < 2; ++v) yt[v] = y[v] + 0.5 * ds * k1[v];
            derivs(s + 0.5 * ds, yt, k2);
            for (int v = 0; v < 2; ++v) yt[v] = y[v] + 0.5 * ds * k2[v];
            derivs(s + 0.5 * ds, yt, k3);
            for (int v = 0; v < 2; ++v) yt[v] = y[v] + ds * k3[v];
            derivs(s + ds, yt, k4);
            for (int v = 0; v < 2; ++v) y[v] += ds / 6.0 * (k1[v] + 2.0 * k2[v] + 2.0 * k3[v] + k4[v]);
            s += ds;
        }
        T[k] = 1.0 + y[0];
        R[k] = std::exp(y[1]) / (1.0 + y[0]);
    }
}

// COMM_MPI periodic copies for one field, NPEY=1 (3dmhdsub.f:3128-3138).
void wrap(double* v, const Index3& I)
{
    for (int k = 1; k <= I.nz; ++k) {
        for (int i = 1; i <= I.nx; ++i) {
            v[I(i, 1, k)] = v[I(i, I.ny - 1, k)];
            v[I(i, I.ny, k)] = v[I(i, 2, k)];
        }
        for (int j = 1; j <= I.ny; ++j) {
            v[I(1, j, k)] = v[I(I.nx - 1, j, k)];
            v[I(I.nx, j, k)] = v[I(2, j, k)];
        }
    }
}

}  // namespace

extern "C" {

double mhd3d_host_ran2(int32_t* idum, int32_t* iy, int32_t* ir)
{
    // RAN2 (3dmhdsub.f:3377-3410); RM is a REAL(4) quotient held in REAL*8.
    const int32_t M = 714025, IA = 1366, IC = 150889;
    const double RM = f2d(1.0f / 714025.0f);
    if (*idum < 0) {
        *idum = (IC - *idum) % M;
        for (int j = 0; j < 97; ++j) {
            *idum = (IA * *idum + IC) % M;
            ir[j] = *idum;
        }
        *idum = (IA * *idum + IC) % M;
        *iy = *idum;
    }
    int j = 1 + (97 * *iy) / M;
    if (j > 97 || j < 1) return std::nan("");
    *iy = ir[j - 1];
    double r = static_cast<double>(*iy) * RM;
    *idum = (IA * *idum + IC) % M;
    ir[j - 1] = *idum;
    return r;
}

void mhd3d_host_default_config(mhd3d_run_config* c, int32_t npx, int32_t npy, int32_t npz)
{
    std::memset(c, 0, sizeof(*c));
    c->npx = npx;
    c->npy = npy;
    c->npz = npz;
    // 3dmhdparam.f:8-34
    c->lmag = 0;
    c->lrot = 0;
    c->izcon = 0;
    c->itcon = 1;
    c->ibcon = 0;
    c->ngrid = MHD3D_GRID_ARCTAN;
    c->xx1 = -7.0; c->xx2 = 7.0;
    c->yy1 = -7.0; c->yy2 = 7.0;
    c->zz1 = -2.0; c->zz2 = 1.0e-2;
    c->xa = f2d(0.5f); c->xb = f2d(0.48f); c->xc = f2d(28.0f); c->xd = f2d(0.025f);
    c->ya = f2d(0.5f); c->yb = f2d(0.48f); c->yc = f2d(28.0f); c->yd = f2d(0.025f);
    c->za = f2d(0.65f); c->zb = f2d(1.0f); c->zc = f2d(5.0f); c->zd = f2d(0.2f);
    c->sff = f2d(0.315f);
    // 3dmhdset.f:36-146
    c->ntube = 0;
    c->re = f2d(2.0f);
    c->pr = f2d(5.0e-2f);
    c->theta = f2d(2.5e-1f);
    c->grav = f2d(6.25e-1f);
    c->tp = f2d(2.0f);
    c->xp = f2d(1.0e1f);
    c->yp = f2d(1.0e1f);
    c->xmax = f2d(2.0e1f);
    c->ymax = f2d(2.0e1f);
    c->zmax = f2d(4.0e1f);
    c->ampt = f2d(5.0e-3f);
    c->gamma = f2d(5.00f / 3.00f);
    c->hh = f2d(1.0f);
    c->seed = 62659;
    c->zstretch = 1.5;
    c->mode = MHD3D_MODE_EXACT;
}

void mhd3d_host_convection_config(mhd3d_run_config* c, int32_t npx, int32_t npy, int32_t npz,
                                  double ra, double ta, double pr_phys, double pm, double contrast,
                                  double m, double beta, double stretch, double ampt, int32_t seed)
{
    mhd3d_host_default_config(c, npx, npy, npz);
    c->lmag = 1;
    c->lrot = 1;
    c->izcon = 1;
    c->itcon = 0;
    c->ibcon = 0;
    c->ngrid = MHD3D_GRID_TANH_Z;
    c->zstretch = stretch;
    c->xmax = 4.0;
    c->ymax = 4.0;
    c->zmax = 1.0;
    c->sff = f2d(0.4f);
    c->gamma = f2d(5.00f / 3.00f);
    const double g = c->gamma;
    const double cp = g / (g - 1.0);
    c->theta = std::pow(contrast, 1.0 / m) - 1.0;
    c->grav = (m + 1.0) * c->theta;
    c->polys = m;
    c->pr = pr_phys / cp;
    const double tmid = 1.0 + c->theta * 0.5 * c->zmax;
    const double rmid = std::pow(tmid, m);
    const double coef = (m + 1.0) * c->theta * c->theta * (m + 1.0 - g * m) / g;  // Ra = coef*RE^2*PR*cp*rho^2/T
    c->re = std::sqrt(ra * tmid / (coef * c->pr * cp * rmid * rmid));
    c->ry = c->re * rmid / std::sqrt(ta);
    c->ang = 0.0;
    c->rm = pm * c->re * rmid;
    c->beta = beta;
    c->pzp = 0.0;
    c->tp = 0.0;
    c->ampt = ampt;
    c->ampb = 0.0;
    c->ntube = 4;
    c->zcent = 0.5;
    c->rmax = 10.0;
    c->atube = 0.01;
    c->seed = seed;
}

int mhd3d_host_params(const mhd3d_run_config* c, mhd3d_params* p)
{
    if (c->npx < 2 || c->npy < 2 || c->npz < 4) return MHD3D_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->npx = c->npx;
    p->npy = c->npy;
    p->npz = c->npz;
    p->lmag = c->lmag;
    p->lrot = c->lrot;
    p->izcon = c->izcon;
    p->itcon = c->itcon;
    p->ibcon = c->ibcon;
    p->mode = c->mode;
    // 3dmhd.f:112-127
    p->c13 = f2d(1.0f / 3.0f);
    p->c23 = 2.0 * p->c13;
    p->c43 = 4.0 * p->c13;
    p->gam1 = f2d(8.0f / 15.0f);
    p->gam2 = f2d(5.0f / 12.0f);
    p->gam3 = f2d(3.0f / 4.0f);
    p->zeta1 = f2d(-17.0f / 60.0f);
    p->zeta2 = f2d(-5.0f / 12.0f);
    p->hx = f2d(0.5f * static_cast<float>(c->npx - 1));
    p->h2x = f2d(static_cast<float>(c->npx - 1) * static_cast<float>(c->npx - 1));
    p->hy = f2d(0.5f * static_cast<float>(c->npy - 1));
    p->h2y = f2d(static_cast<float>(c->npy - 1) * static_cast<float>(c->npy - 1));
    p->hz = f2d(0.5f * static_cast<float>(c->npz - 1));
    p->h2z = f2d(static_cast<float>(c->npz - 1) * static_cast<float>(c->npz - 1));
    // 3dmhd.f:155-240, 382-384
    p->re = c->re;
    p->theta = c->theta;
    p->grav = c->grav;
    p->gamma = c->gamma;
    p->sf = c->sff;
    p->omx = c->lrot ? std::sin(c->ang) / c->ry : 0.0;
    p->omz = c->lrot ? std::cos(c->ang) / c->ry : 0.0;
    p->repr = c->re * c->pr;
    p->ore = 1.0 / c->re;
    if (c->lmag) {
        p->orm = 1.0 / c->rm;
        p->obeta = 2.0 / c->beta;
    }
    p->rm = c->rm;
    p->cv = 1.0 / (c->gamma - 1.0);
    p->ocv = 1.0 / p->cv;
    p->tp = c->tp;
    p->tc = c->tc;
    p->xp = c->xp;
    p->yp = c->yp;
    p->hh = c->hh;
    p->timi = c->timi;
    p->timc = 0.0;
    p->dtmin = f2d(1.0e-8f);
    std::vector<double> T, R;
    static_profile(c, c->npz, T, R);
    p->tb = T[c->npz];
    return MHD3D_OK;
}

int mhd3d_host_grid(const mhd3d_run_config* c,
                    double* exx, double* dxxdx, double* d2xxdx2, double* ddx,
                    double* wyy, double* dyydy, double* d2yydy2, double* ddy,
                    double* zee, double* dzzdz, double* d2zzdz2, double* ddz,
                    double* rkapa, double* dkapa)
{
    const int NX = c->npx + 2, NY = c->npy + 2, NZ = c->npz + 2;
    if (c->npx < 2 || c->npy < 2 || c->npz < 4) return MHD3D_ERR_ARG;
    // XJACOBI (3dmhdsub.f:177-209); ghost entries stay zero as in COMMON.
    for (int i = 0; i < NX; ++i) exx[i] = dxxdx[i] = d2xxdx2[i] = ddx[i] = 0.0;
    {
        const double orx = f2d(1.0f / static_cast<float>(NX - 2 - 1));
        std::vector<double> s(NX + 1, 0.0);
        for (int i = 0; i <= NX - 2 - 1; ++i) s[i + 2] = f2d(static_cast<float>(i)) * orx;
        s[2] = 0.0;
        s[NX - 1] = 1.0;
        for (int i = 2; i <= NX - 1; ++i) {
            Map m = mkgrid(c, s[i], 1);
            exx[i - 1] = m.sphys;
            dxxdx[i - 1] = m.dssds;
            d2xxdx2[i - 1] = m.d2ssds2;
            ddx[i - 1] = orx * (1.0 / m.dssds);
        }
    }
    // YJACOBI (3dmhdsub.f:211-281), single domain: J=1 -> s=0, J=NY -> s=1.
    {
        const int npy = c->npy;
        const double ory = f2d(1.0f / static_cast<float>(npy - 1));
        std::vector<double> yy(npy + 1, 0.0);
        for (int j = 0; j <= npy - 1; ++j) yy[j + 1] = f2d(static_cast<float>(j)) * ory;
        yy[1] = 0.0;
        yy[npy] = 1.0;
        for (int j = 1; j <= NY; ++j) {
            double s = (j == 1) ? 0.0 : (j == NY) ? 1.0 : yy[j - 1];
            Map m = mkgrid(c, s, 2);
            wyy[j - 1] = m.sphys;
            dyydy[j - 1] = m.dssds;
            d2yydy2[j - 1] = m.d2ssds2;
            ddy[j - 1] = ory * (1.0 / m.dssds);
        }
    }
    // ZJACOBI (3dmhdsub.f:283-353) with the first-rank top ghost (s=0) and
    // the last-rank bottom ghost (s=1) conventions.
    {
        const int npz = c->npz;
        const double orz = f2d(1.0f / static_cast<float>(npz - 1));
        std::vector<double> zz(npz + 1, 0.0);
        for (int k = 0; k <= npz - 1; ++k) zz[k + 1] = f2d(static_cast<float>(k)) * orz;
        zz[1] = 0.0;
        zz[npz] = 1.0;
        for (int k = 1; k <= NZ; ++k) {
            double s = (k == 1) ? 0.0 : (k == NZ) ? 1.0 : zz[k - 1];
            Map m = mkgrid(c, s, 3);
            zee[k - 1] = m.sphys;
            dzzdz[k - 1] = m.dssds;
            d2zzdz2[k - 1] = m.d2ssds2;
            ddz[k - 1] = orz * (1.0 / m.dssds);
        }
    }
    for (int k = 0; k < NZ; ++k) kappa_profile(c, zee[k], &rkapa[k], &dkapa[k]);
    return MHD3D_OK;
}

int mhd3d_host_static(const mhd3d_run_config* c, const double* zee,
                      double* ru, double* rv, double* rw, double* tt, double* ro,
                      double* bx, double* by, double* bz)
{
    const int NX = c->npx + 2, NY = c->npy + 2, NZ = c->npz + 2, npz = c->npz;
    const Index3 I{NX, NY, NZ};
    const size_t n = static_cast<size_t>(NX) * NY * NZ;
    if (c->lmag && (!bx || !by || !bz)) return MHD3D_ERR_ARG;
    if (c->lmag && c->ampb == 0.0 && c->ntube != 0 && c->ntube != 4) return MHD3D_ERR_ARG;
    for (size_t q = 0; q < n; ++q) {
        ru[q] = rv[q] = rw[q] = 0.0;
        tt[q] = ro[q] = 0.0;
        if (c->lmag) bx[q] = by[q] = bz[q] = 0.0;
    }
    std::vector<double> T, R;
    static_profile(c, npz, T, R);
    const double TB = T[npz], RB = R[npz];
    // Divide among processors (3dmhdsub.f:525-564) for one block.
    for (int k = 1; k <= NZ; ++k) {
        double t = (k == 1) ? T[1] : (k == NZ) ? TB : T[k - 1];
        double r = (k == 1) ? R[1] : (k == NZ) ? RB : R[k - 1];
        for (int j = 2; j <= NY - 1; ++j)
            for (int i = 2; i <= NX - 1; ++i) {
                tt[I(i, j, k)] = t;
                ro[I(i, j, k)] = r;
            }
    }
    double obeta = c->lmag ? 2.0 / c->beta : 0.0;
    if (c->lmag) {
        if (c->ampb != 0.0) {
            // Horizontal Bx layer (3dmhdsub.f:569-580)
            double cln = f2d(-(4.0f * std::log(2.0f))) / c->bfh / c->bfh;
            for (int k = 2; k <= NZ - 1; ++k) {
                double d = zee[k - 1] - c->bzp;
                double b = c->ampb * std::exp(cln * (d * d));
                for (int j = 1; j <= NY; ++j)
                    for (int i = 1; i <= NX; ++i) bx[I(i, j, k)] = b;
            }
            for (int k = 2; k <= NZ - 1; ++k)
                for (int j = 2; j <= NY - 1; ++j)
                    for (int i = 2; i <= NX - 1; ++i) {
                        size_t q = I(i, j, k);
                        ro[q] = ro[q] - bx[q] * bx[q] / tt[q] * obeta;
                    }
        } else if (c->ntube == 4) {
            // TUBE model 4 (3dmhdsub.f:4272-4302): uniform BY layer, pressure balanced.
            for (int k = 2; k <= NZ - 1; ++k) {
                double znew = zee[k - 1] - c->zcent;
                double rnew = std::sqrt(znew * znew);
                double b = (1.0 - std::tanh((rnew - c->rmax) / c->atube)) / 2.0;
                for (int j = 2; j <= NY - 1; ++j)
                    for (int i = 2; i <= NX - 1; ++i) {
                        size_t q = I(i, j, k);
                        by[q] = b;
                        double pre = ro[q] * tt[q] - b * b * obeta / 2.0;
                        ro[q] = pre / tt[q];
                    }
            }
        }
    }
    // Random temperature perturbation (3dmhdsub.f:594-641), ISW=1.
    if (c->ampt != 0.0) {
        int32_t idum = -c->seed, iy = 0, ir[97];
        for (int k = 2; k <= NZ - 1; ++k)
            for (int j = 2; j <= NY - 1; ++j)
                for (int i = 2; i <= NX - 1; ++i) {
                    double rnd = 1.0 + c->ampt * (mhd3d_host_ran2(&idum, &iy, ir) - 0.5);
                    tt[I(i, j, k)] = tt[I(i, j, k)] * rnd;
                }
    }
    // COMMUNICATE (3dmhd.f:365)
    double* fields[8] = {ru, rv, rw, tt, ro, bx, by, bz};
    for (int f = 0; f < (c->lmag ? 8 : 5); ++f) wrap(fields[f], I);
    return MHD3D_OK;
}

}  // extern "C"
