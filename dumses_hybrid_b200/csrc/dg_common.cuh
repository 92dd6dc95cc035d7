// Shared definitions of the sm_100a MHD step kernels.
//
// Arithmetic rule for the FP64 path: every expression keeps the operation
// order of the reference Fortran (and of the CPU oracle that restates it),
// the translation units are compiled with --fmad=false so no multiply-add is
// contracted, division and sqrt are IEEE round-to-nearest, and Fortran
// MIN/MAX/SIGN map to the ternaries below.  Under those rules the GPU results
// are bit-identical to a gfortran x86-64 build of the reference.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dumses_gpu.h"

namespace dg {

// variable slots of the device state (the reference's uin(:,:,:,1:8))
enum { IR = 0, IU = 1, IV = 2, IW = 3, IP = 4, IA = 5, IB = 6, IC = 7, NVAR = 8 };

constexpr double kSmallr = 1.0e-10;  // commons.f90:48
constexpr double kSmallc = 1.0e-10;  // commons.f90:49

template <typename T> __host__ __device__ __forceinline__ T mn(T a, T b) { return a < b ? a : b; }
template <typename T> __host__ __device__ __forceinline__ T mx(T a, T b) { return a > b ? a : b; }
__device__ __forceinline__ double sgn1(double x) { return copysign(1.0, x); }
__device__ __forceinline__ float sgn1(float x) { return copysignf(1.0f, x); }
__device__ __forceinline__ double fab(double x) { return fabs(x); }
__device__ __forceinline__ float fab(float x) { return fabsf(x); }
__device__ __forceinline__ double sqr(double x) { return sqrt(x); }
__device__ __forceinline__ float sqr(float x) { return sqrtf(x); }

// Unsigned division by a divisor fixed for the context, by a multiply-high and a shift
// (Granlund and Montgomery, "Division by invariant integers using multiplication", PLDI 1994,
// theorem 4.2 with N = 32): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (mulhi(m, n) + n) >> l for every n < 2^31 (the sum then stays below 2^32).  The
// kernels split their linear cell, face and edge indices (all below 2^31, checked when a
// context is made) into (i, j, k) with it instead of 64-bit divisions.
struct FastDiv {
    unsigned d, m;
    int l;
};
inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d;
    f.l = 0;
    while ((1ull << f.l) < d) f.l++;
    f.m = (unsigned)(((1ull << 32) * ((1ull << f.l) - d)) / d + 1);
    return f;
}
__host__ __device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv &f) {
#ifdef __CUDA_ARCH__
    return (__umulhi(f.m, n) + n) >> f.l;
#else
    return (unsigned)((((unsigned long long)f.m * n >> 32) + n) >> f.l);
#endif
}
// a + X (b + Y c) = t  ->  (a, b, c)
__host__ __device__ __forceinline__ void split3(unsigned t, const FastDiv &X, const FastDiv &Y, int &a, int &b, int &c) {
    const unsigned r = fdiv(t, X);
    a = (int)(t - r * X.d);
    const unsigned q = fdiv(r, Y);
    b = (int)(r - q * Y.d);
    c = (int)q;
}

// Geometry of one context, passed to every kernel by value.
struct Geo {
    int ndim, nx, ny, nz;
    int NX, NY, NZ;           // ghosted extents (nx+6, ny+6 or 1, nz+6 or 1)
    int gy, gz;               // ghost layers in y and z (3 or 0)
    long long sy, sz, sv;     // strides of j, k and variable in the state arrays
    // trace-core index space: cells [0, nx+1] x [0, ny+1] x [kc0, kc1]
    int CX, CY, CZ, kc0;
    long long csz;            // cells in the core index space
    // face index space: [1, nx+1] x [1, ny+1] x [1, nz+1] (z extent 1 for ndim = 2)
    int FX, FY, FZ;
    long long fsz;
    // edge electric-field index space of the trace: [0, nx+2] x [0, ny+2] x [ke0, ke1]
    int EX, EY, EZ, ke0;
    long long esz;
    double dx, dy, dz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double gamma, ciso, omega0, courant;
    double nu, eta;           // viscosity and resistivity of dissipation (0 = off)
    int iso, slope_type, iriemann, iriemann2d, fargo, shearing;
    int bc[3];
    int ndim_act;
    // z-slab decomposition: slabs, this slab's position, and the boundary of its lower and
    // upper z sides (bc[2], or kBcHalo where the neighbour's halo fills the ghost planes)
    int nzslice, zposition;
    int bcz_lo, bcz_hi;
    // dividers of the index spaces: face (FX, FY, FZ), core (CX, CY), edge (EX, EY), and the
    // ghosted cells of the primitive variables (nx+5, ny+5)
    FastDiv dFX, dFY, dFZ, dCX, dCY, dEX, dEY, dPX, dPY;
    double smallp;            // pressure floor smallr smallc^2 / gamma of the trace and solvers
    double dvloc;             // 1 / (dx dy dz), as update forms it (scheme.f90:1778-1779)
    double entho;             // 1 / (gamma - 1) of the HLLD solver (solver.f90:646)
    double rdx, rdy, rdz;     // 1 / dx, 1 / dy, 1 / dz
    // 1 where dx (dy, dz) is a power of two: then x / dx and x * (1 / dx) are the same real number
    // correctly rounded, so the FP64 kernels multiply instead of dividing (bit for bit the same)
    int p2x, p2y, p2z;
    __host__ __device__ __forceinline__ double per_dx(double x) const { return p2x ? x * rdx : x / dx; }
    __host__ __device__ __forceinline__ double per_dy(double x) const { return p2y ? x * rdy : x / dy; }
    __host__ __device__ __forceinline__ double per_dz(double x) const { return p2z ? x * rdz : x / dz; }

    __host__ __device__ __forceinline__ long long idx(int i, int j, int k) const {
        return (long long)(i + 2) + sy * (long long)(j + gy - 1) + sz * (long long)(k + gz - 1);
    }
    __host__ __device__ __forceinline__ long long cidx(int i, int j, int k) const {
        return (long long)i + (long long)CX * ((long long)j + (long long)CY * (long long)(k - kc0));
    }
    __host__ __device__ __forceinline__ long long fidx(int i, int j, int k) const {
        return (long long)(i - 1) + (long long)FX * ((long long)(j - 1) + (long long)FY * (long long)(k - 1));
    }
    __host__ __device__ __forceinline__ long long eidx(int i, int j, int k) const {
        return (long long)i + (long long)EX * ((long long)j + (long long)EY * (long long)(k - ke0));
    }
    // cell centre x(i) = xmin + dx/2 + (i-1) dx (init.f90:461-468)
    __host__ __device__ __forceinline__ double xc(int i) const { return xmin + dx / 2 + (i - 1) * dx; }
};

// z side of a slab whose ghost planes are filled from the neighbour slab's halo
constexpr int kBcHalo = 3;

// Scalars that stay on the device across steps (dt, time, CFL reduction).
struct Scalars {
    double dt;
    double time;
    unsigned long long red;   // bits of the running CFL minimum (positive doubles order as integers)
    int err;                  // DG_ERR_* raised by a kernel (0 = none)
    int sh_jp;                // shear offset of the x boundaries: whole cells ...
    double sh_epsi;           // ... and remainder, for the time of the last k_shear_offset launch
};

// number of trace-core fields per cell
constexpr int kCore3 = 47;
constexpr int kCore2 = 30;
// the core is stored in blocks of kCoreLane cells, each block field-major
constexpr int kCoreLane = 32;
__host__ __device__ __forceinline__ long long core_base(long long c, int nf) {
    return (c >> 5) * (long long)(nf * kCoreLane) + (c & (kCoreLane - 1));
}
__host__ __device__ __forceinline__ long long core_elems(long long csz, int nf) {
    return (csz + kCoreLane - 1) / kCoreLane * kCoreLane * nf;
}

// face flux records, face-major: rho, E, rho u, rho v, rho w (scaled by area*dt as
// compflux does), p*_tot, then in 2D the B_z flux and a pad (6 values per face in 3D,
// 8 in 2D, 9 in 1D)
constexpr int kFluxComp = 8;  // the larger record (allocation)
constexpr int kFluxRec3 = 6, kFluxRec2 = 8;
// ndim = 1: rho, E, rho u, rho v, rho w, p*_tot, B_x, B_y, B_z (every field has an x flux)
constexpr int kFluxRec1 = 9;
__host__ __device__ __forceinline__ int flux_rec(int ndim) { return ndim == 3 ? kFluxRec3 : ndim == 2 ? kFluxRec2 : kFluxRec1; }

}  // namespace dg
