// Host-side initial conditions written into a reference-layout uin array.
//
// These stand in for the reference's problem plug-ins (src/problem/<name>/condinit.f90),
// which the Fortran driver would keep calling unchanged; the library needs its
// own copies so that tests and the benchmark can build the configured states
// without a Fortran compiler.  Random velocity kicks use a counter-based
// generator (splitmix64 of seed and cell index) instead of the reference's
// wall-clock-seeded random_number (mri/condinit.f90:52-61), so runs are
// reproducible on any number of threads.
#include "dumses_gpu.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Grid {
    int ndim, nx, ny, nz;
    int iu1, iu2, ju1, ju2, ku1, ku2;
    long n0, n1, n2;
    double dx, dy, dz;
    double zoff;  // a z slab's offset dz * nz * zposition (init.f90:491), 0 for one domain
    explicit Grid(const dg_params &p) {
        ndim = p.ndim; nx = p.nx; ny = p.ny; nz = p.nz;
        iu1 = -2; iu2 = nx + 3;
        ju1 = 1; ju2 = 1; ku1 = 1; ku2 = 1;
        if (ndim > 1) { ju1 = -2; ju2 = ny + 3; }
        if (ndim == 3) { ku1 = -2; ku2 = nz + 3; }
        n0 = iu2 - iu1 + 1; n1 = ju2 - ju1 + 1; n2 = ku2 - ku1 + 1;
        dx = (p.xmax - p.xmin) / nx;
        dy = (p.ymax - p.ymin) / ny;
        const int nzslice = p.nzslice > 1 ? p.nzslice : 1;
        dz = (p.zmax - p.zmin) / (nz * nzslice);
        zoff = nzslice > 1 ? dz * nz * p.zposition : 0.0;
    }
    long idx(int i, int j, int k, int v) const {
        return (i - iu1) + n0 * ((j - ju1) + n1 * ((k - ku1) + n2 * (long)(v - 1)));
    }
    // cell centres as init_grid computes them (init.f90:461-501)
    double x(const dg_params &p, int i) const { return p.xmin + dx / 2 + (i - 1) * dx; }
    double y(const dg_params &p, int j) const { return p.ymin + dy / 2 + (j - 1) * dy; }
    double z(const dg_params &p, int k) const {
        return zoff != 0.0 ? p.zmin + zoff + dz / 2 + (k - 1) * dz : p.zmin + dz / 2 + (k - 1) * dz;
    }
};

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// uniform in [0,1) from (seed, stream, counter)
double uniform01(uint64_t seed, uint64_t stream, uint64_t counter) {
    uint64_t h = splitmix64(seed ^ splitmix64(stream * 0x100000001B3ull + counter));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

const double kTwoPi = 4.0 * std::asin(1.0);  // commons.f90:47
const double kPi = 2.0 * std::asin(1.0);

}  // namespace

extern "C" int dg_condinit(const dg_params *p, int ic, double beta, double amp,
                           unsigned long long seed, double *uin) {
    if (!p || !uin) return DG_ERR_ARG;
    Grid g(*p);
    const long total = g.n0 * g.n1 * g.n2 * 11;
    std::memset(uin, 0, sizeof(double) * (size_t)total);
    auto U = [&](int i, int j, int k, int v) -> double & { return uin[g.idx(i, j, k, v)]; };

    if (ic == DG_IC_MRI_TEST || ic == DG_IC_MRI) {
        // mri/condinit.f90:30-105
        if (p->ndim != 3) return DG_ERR_ARG;
        const double d0 = 1.0;
        const double p0 = d0 * p->ciso * p->ciso;
        const double B0 = std::sqrt(2.0 * p0 / beta);
        for (int k = g.ku1; k <= g.ku2; k++)
            for (int j = g.ju1; j <= g.ju2; j++)
                for (int i = g.iu1; i <= g.iu2; i++) {
                    U(i, j, k, 1) = d0;
                    const uint64_t cell = (uint64_t)g.idx(i, j, k, 1);
                    if (ic == DG_IC_MRI_TEST) {
                        // amp = 0 in the regression setup: the kicks are zero
                        U(i, j, k, 2) = 1.e-2 * 1.e-3 * std::cos(kTwoPi * 10.0 * g.z(*p, k)) *
                                        std::cos(kTwoPi * 5.0 * g.x(*p, i));
                        U(i, j, k, 3) = 0.0;
                        U(i, j, k, 4) = 0.0;
                        U(i, j, k, 8) = B0 * std::sin(kTwoPi * g.x(*p, i));
                        U(i, j, k, 11) = B0 * std::sin(kTwoPi * g.x(*p, i));
                    } else {
                        // net vertical field ('fluxZ'), uniform kicks amp*(r-1/2)*sqrt(p0)
                        U(i, j, k, 2) = U(i, j, k, 1) * amp * (uniform01(seed, 1, cell) - 0.5) * std::sqrt(p0);
                        U(i, j, k, 3) = U(i, j, k, 1) * amp * (uniform01(seed, 2, cell) - 0.5) * std::sqrt(p0);
                        U(i, j, k, 4) = U(i, j, k, 1) * amp * (uniform01(seed, 3, cell) - 0.5) * std::sqrt(p0);
                        U(i, j, k, 8) = B0;
                        U(i, j, k, 11) = B0;
                    }
                }
        return DG_OK;
    }

    if (ic == DG_IC_ORSZAG_TANG) {
        // 3D Orszag-Tang-type vortex: rho = 25/(36 pi), P = 5/(12 pi),
        // v = (-sin 2pi y, sin 2pi x, 0.2 sin 2pi z), B = (-sin 2pi y, sin 4pi x, 0)/sqrt(4 pi).
        // Bx depends on y only and By on x only, so face and centre values agree
        // and div B = 0 exactly.
        if (p->ndim != 3) return DG_ERR_ARG;
        const double rho = 25.0 / (36.0 * kPi), pres = 5.0 / (12.0 * kPi);
        const double b0 = 1.0 / std::sqrt(4.0 * kPi);
        for (int k = g.ku1; k <= g.ku2; k++)
            for (int j = g.ju1; j <= g.ju2; j++)
                for (int i = g.iu1; i <= g.iu2; i++) {
                    const double x = g.x(*p, i), y = g.y(*p, j), z = g.z(*p, k);
                    const double vx = -std::sin(kTwoPi * y), vy = std::sin(kTwoPi * x), vz = 0.2 * std::sin(kTwoPi * z);
                    const double bx = -b0 * std::sin(kTwoPi * y), by = b0 * std::sin(2.0 * kTwoPi * x);
                    U(i, j, k, 1) = rho;
                    U(i, j, k, 2) = rho * vx;
                    U(i, j, k, 3) = rho * vy;
                    U(i, j, k, 4) = rho * vz;
                    U(i, j, k, 6) = bx; U(i, j, k, 9) = bx;
                    U(i, j, k, 7) = by; U(i, j, k, 10) = by;
                    U(i, j, k, 5) = pres / (p->gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) +
                                    0.5 * (bx * bx + by * by);
                }
        return DG_OK;
    }

    if (ic == DG_IC_FIELD_LOOP) {
        // 2D field-loop advection in the form of magnetic_loop/condinit.f90:40-104
        // (direction 'x'): A_z = A0 (R - r) inside r < R, face B from its differences.
        if (p->ndim != 2) return DG_ERR_ARG;
        const double A0 = 1.e-3, R = 0.3, rho = 1.0, pres = 1.0, vx = 2.0, vy = 1.0;
        auto Az = [&](int i, int j) {
            const double x = g.x(*p, i), y = g.y(*p, j);
            const double dist = std::sqrt(x * x + y * y);
            return dist <= R ? A0 * (R - dist) : 0.0;
        };
        const int k = 1;
        for (int j = g.ju1; j <= g.ju2; j++)
            for (int i = g.iu1; i <= g.iu2; i++) {
                const double bxl = (Az(i, j + 1) - Az(i, j)) / g.dy;
                const double bxr = (Az(i + 1, j + 1) - Az(i + 1, j)) / g.dy;
                const double byl = -(Az(i + 1, j) - Az(i, j)) / g.dx;
                const double byr = -(Az(i + 1, j + 1) - Az(i, j + 1)) / g.dx;
                U(i, j, k, 1) = rho;
                U(i, j, k, 2) = rho * vx;
                U(i, j, k, 3) = rho * vy;
                U(i, j, k, 4) = 0.0;
                U(i, j, k, 6) = bxl; U(i, j, k, 9) = bxr;
                U(i, j, k, 7) = byl; U(i, j, k, 10) = byr;
                const double bcx = 0.5 * (bxl + bxr), bcy = 0.5 * (byl + byr);
                U(i, j, k, 5) = pres / (p->gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bcx * bcx + bcy * bcy);
            }
        return DG_OK;
    }
    return DG_ERR_ARG;
}
