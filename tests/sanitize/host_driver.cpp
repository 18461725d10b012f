// Host-side code under AddressSanitizer and UndefinedBehaviorSanitizer: the
// set-up library (grid, STATIC/TUBE, RAN2), the dump/restart IO and the CPU
// oracle (built without OpenMP here), driven through the same calls the
// Python binding and the tests make.  Built and run by
// tests/test_host_sanitizers.py; exits non-zero on a mismatch, and the
// sanitizers abort on any invalid access or undefined operation.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mhd3d.h"
#include "mhd3d_host.h"
#include "oracle3dmhd.h"

static int run(int lmag, const char* dir)
{
    mhd3d_run_config c;
    mhd3d_host_convection_config(&c, 24, 16, 12, 1e5, 1e4, 1.0, 4.0, 10.0, 1.0, 1e4, 1.5, 2e-2, 7);
    c.lmag = lmag;
    mhd3d_params p;
    if (mhd3d_host_params(&c, &p)) return 10;
    const int nx = p.npx + 2, ny = p.npy + 2, nz = p.npz + 2;
    const size_t n = (size_t)nx * ny * nz;
    std::vector<double> g[14];
    const int len[14] = {nx, nx, nx, nx, ny, ny, ny, ny, nz, nz, nz, nz, nz, nz};
    for (int i = 0; i < 14; ++i) g[i].assign(len[i], 0.0);
    if (mhd3d_host_grid(&c, g[0].data(), g[1].data(), g[2].data(), g[3].data(), g[4].data(), g[5].data(),
                        g[6].data(), g[7].data(), g[8].data(), g[9].data(), g[10].data(), g[11].data(), g[12].data(),
                        g[13].data()))
        return 11;
    std::vector<double> f[8];
    for (int i = 0; i < 8; ++i) f[i].assign((i < 5 || lmag) ? n : 0, 0.0);
    auto ptr = [&](int i) { return f[i].empty() ? nullptr : f[i].data(); };
    if (mhd3d_host_static(&c, g[8].data(), ptr(0), ptr(1), ptr(2), ptr(3), ptr(4), ptr(5), ptr(6), ptr(7))) return 12;

    oracle_set_threads(1);
    oracle3dmhd* o = oracle_create(&p, g[0].data(), g[1].data(), g[2].data(), g[3].data(), g[4].data(), g[5].data(),
                                   g[6].data(), g[7].data(), g[8].data(), g[9].data(), g[10].data(), g[11].data(),
                                   g[12].data(), g[13].data());
    if (!o) return 13;
    oracle_set_state(o, ptr(0), ptr(1), ptr(2), ptr(3), ptr(4), ptr(5), ptr(6), ptr(7));
    double dt = 0, timc = 0, timt = 0, umach = 0;
    int nit = 0;
    if (oracle_step(o, 3, &dt, &timc, &timt, &umach, &nit) || nit != 3 || !(dt > 0)) return 14;
    std::vector<double> fl[8];
    for (int i = 0; i < 8; ++i) fl[i].assign((i < 5 || lmag) ? n : 0, 0.0);
    auto fp = [&](int i) { return fl[i].empty() ? nullptr : fl[i].data(); };
    oracle_fluxes(o, fp(0), fp(1), fp(2), fp(3), fp(4), fp(5), fp(6), fp(7));
    double dt2 = 0, um2 = 0;
    if (oracle_cfl(o, &dt2, &um2) || !(dt2 > 0)) return 15;
    std::vector<double> prof((size_t)7 * p.npz);
    oracle_profiles(o, prof.data());
    oracle_bcon(o);
    oracle_get_state(o, ptr(0), ptr(1), ptr(2), ptr(3), ptr(4), ptr(5), ptr(6), ptr(7));
    oracle_destroy(o);
    for (int i = 0; i < 8; ++i)
        for (double v : f[i])
            if (!std::isfinite(v)) return 16;

    // a dump written and read back gives the same interior
    const int32_t ipar15[5] = {1, 0, 3, 0, 1};
    double par1[96];
    mhd3d_host_par1(&c, ipar15, 1, 1, nit, dt, timt, timc, par1);
    const std::string fout = std::string(dir) + (lmag ? "/mhd" : "/hydro");
    if (mhd3d_host_write_dump(fout.c_str(), 0, par1, p.npx, p.npy, p.npz, lmag, ptr(0), ptr(1), ptr(2), ptr(3), ptr(4),
                              ptr(5), ptr(6), ptr(7), timt, timc, umach, dt))
        return 17;
    std::vector<double> r[8];
    for (int i = 0; i < 8; ++i) r[i].assign((i < 5 || lmag) ? n : 0, 0.0);
    auto rp = [&](int i) { return r[i].empty() ? nullptr : r[i].data(); };
    double back[96];
    if (mhd3d_host_read_dump(fout.c_str(), 1, 1, 1, lmag, p.npx, p.npy, p.npz, back, rp(0), rp(1), rp(2), rp(3), rp(4),
                             rp(5), rp(6), rp(7)))
        return 18;
    for (int i = 0; i < 8; ++i) {
        if (f[i].empty()) continue;
        for (int k = 1; k < nz - 1; ++k)
            for (int j = 1; j < ny - 1; ++j)
                for (int q = 1; q < nx - 1; ++q) {
                    const size_t at = ((size_t)k * ny + j) * nx + q;
                    if (r[i][at] != f[i][at]) return 19;
                }
    }
    if (std::memcmp(back, par1, sizeof(par1)) != 0) return 20;
    return 0;
}

int main(int argc, char** argv)
{
    const char* dir = argc > 1 ? argv[1] : ".";
    for (int lmag = 0; lmag < 2; ++lmag) {
        const int rc = run(lmag, dir);
        if (rc) {
            std::fprintf(stderr, "host driver failed: lmag=%d code %d\n", lmag, rc);
            return rc;
        }
    }
    std::printf("host driver ok\n");
    return 0;
}
