// Kernels of the DUMSES Godunov MHD step, written once and instantiated for two
// arithmetics (this header is included by step_fp64.cu and step_fp32.cu):
//
//   FP64 plain path   T = double, state StoreD (8 FP64 planes), --fmad=false:
//                     bit-identical to the reference arithmetic.
//   FP32 mixed path   T = float, state StoreHL (compensated FP32 hi/lo planes),
//                     fast FP32 math; FP64 only where the state is turned into
//                     primitives (pressure recovery from total energy), in the
//                     CFL reduction, FARGO's remap and the history sums.
//
// Pipeline of one step (the call order of src/dumses.f90:82-120):
//   k_prim_dt     compute_dt  (physics.f90:18-132)      primitive(0) into Q + CFL min-reduction
//   k_prim        primitive   (scheme.f90:20-91)        Q on the ghosted grid
//   k_efield      edge E of trace3d/trace2d (scheme.f90:1194-1239, 856-872), once per edge
//   k_trace       slope + trace3d/trace2d (scheme.f90:253-656, 807-1711)
//                 -> per-cell "trace core": predicted cell state, half slopes,
//                    predicted face B and its transverse half slopes; every
//                    face and corner state of the reference is one add (and a
//                    floor) away from these values.
//   k_riemann     riemann_solver + riemann_solver_magnetic + compflux
//                 (solver.f90:65-387, solver_magnetic.f90:55-235, scheme.f90:1716-1760)
//                 one thread per cell: its three left faces and three lower edges.
//   k_update      update + constrained_transport (scheme.f90:1764-1993), with the
//                 shearing-box averaging of the boundary mass flux and emfy
//                 (shearingbox.f90:207-390) applied on the fly.
//   k_fargo_*     fargo_update (fargo.f90:17-288)
//   k_boundary    boundary (boundary.f90:18-92) incl. shearing_boundary (shearingbox.f90:19-203)
#pragma once
#include <utility>
#include <vector>

#include "mhd_kernels.cuh"
#include "solvers.cuh"

#ifndef DG_NS
#error "define DG_NS (f64 or f32) before including step_impl.cuh"
#endif

namespace dg {
namespace DG_NS {
namespace {

constexpr int kThreads = 128;

// Checked build (-DDG_CHECK_BOUNDS, a debug stand-in for a memory sanitizer): every array
// access made through ld(), the record helpers below and the state stores must fall inside
// a device buffer the host registered (debug_register: all buffers of every live context);
// an access outside is counted in g_oob and not made (a load returns 0).
#ifdef DG_CHECK_BOUNDS
constexpr int kMaxBufs = 256;
__device__ const char *g_buf_lo[kMaxBufs];
__device__ const char *g_buf_hi[kMaxBufs];
__device__ int g_nbuf;
__device__ unsigned long long g_oob;
__device__ __forceinline__ bool chk(const void *p, size_t n) {
    const char *c = (const char *)p;
    for (int b = 0; b < g_nbuf; b++)
        if (c >= g_buf_lo[b] && c + n <= g_buf_hi[b]) return true;
    atomicAdd(&g_oob, 1ull);
    return false;
}
#else
__device__ __forceinline__ bool chk(const void *, size_t) { return true; }
#endif

template <typename X> __device__ __forceinline__ X ld(const X *p) { return chk(p, sizeof(X)) ? __ldg(p) : X(0); }

// 8 contiguous values (one face record) with 16-byte vector accesses
__device__ __forceinline__ void load8(const float *p, float v[8]) {
    if (!chk(p, 8 * sizeof(float))) {
        for (int n = 0; n < 8; n++) v[n] = 0.0f;
        return;
    }
    const float4 a = __ldg((const float4 *)p), b = __ldg((const float4 *)p + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void load8(const double *p, double v[8]) {
    if (!chk(p, 8 * sizeof(double))) {
        for (int n = 0; n < 8; n++) v[n] = 0.0;
        return;
    }
#pragma unroll
    for (int n = 0; n < 4; n++) {
        const double2 a = __ldg((const double2 *)p + n);
        v[2 * n] = a.x; v[2 * n + 1] = a.y;
    }
}
__device__ __forceinline__ void store8(float *p, const float v[8]) {
    if (!chk(p, 8 * sizeof(float))) return;
    ((float4 *)p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    ((float4 *)p)[1] = make_float4(v[4], v[5], v[6], v[7]);
}
__device__ __forceinline__ void store8(double *p, const double v[8]) {
    if (!chk(p, 8 * sizeof(double))) return;
#pragma unroll
    for (int n = 0; n < 4; n++) ((double2 *)p)[n] = make_double2(v[2 * n], v[2 * n + 1]);
}
// 6 contiguous values (a 3D face record) with 8-byte (float) / 16-byte (double) vector accesses
__device__ __forceinline__ void load6(const float *p, float v[6]) {
    if (!chk(p, 6 * sizeof(float))) {
        for (int n = 0; n < 6; n++) v[n] = 0.0f;
        return;
    }
#pragma unroll
    for (int n = 0; n < 3; n++) {
        const float2 a = __ldg((const float2 *)p + n);
        v[2 * n] = a.x; v[2 * n + 1] = a.y;
    }
}
__device__ __forceinline__ void load6(const double *p, double v[6]) {
    if (!chk(p, 6 * sizeof(double))) {
        for (int n = 0; n < 6; n++) v[n] = 0.0;
        return;
    }
#pragma unroll
    for (int n = 0; n < 3; n++) {
        const double2 a = __ldg((const double2 *)p + n);
        v[2 * n] = a.x; v[2 * n + 1] = a.y;
    }
}
__device__ __forceinline__ void store6(float *p, const float v[6]) {
    if (!chk(p, 6 * sizeof(float))) return;
#pragma unroll
    for (int n = 0; n < 3; n++) ((float2 *)p)[n] = make_float2(v[2 * n], v[2 * n + 1]);
}
__device__ __forceinline__ void store6(double *p, const double v[6]) {
    if (!chk(p, 6 * sizeof(double))) return;
#pragma unroll
    for (int n = 0; n < 3; n++) ((double2 *)p)[n] = make_double2(v[2 * n], v[2 * n + 1]);
}

inline unsigned nblocks(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// ---------------------------------------------------------------------------
// state storage policies
// ---------------------------------------------------------------------------
// FP64 state: nv planes of doubles, plane v at p + v*sv
struct StoreD {
    using T = double;  // arithmetic of the kernels on this state
    double *p;
    __device__ __forceinline__ double get(const Geo &G, int v, long long c) const {
        return chk(p + G.sv * v + c, 8) ? p[G.sv * v + c] : 0.0;
    }
    __device__ __forceinline__ double getr(const Geo &G, int v, long long c) const { return ld(p + G.sv * v + c); }
    __device__ __forceinline__ void set(const Geo &G, int v, long long c, double x) const {
        if (chk(p + G.sv * v + c, 8)) p[G.sv * v + c] = x;
    }
    // u = u + inc, the reference's in-place update; Val holds a value between a load and
    // a store so that a sequence of increments runs in registers
    using Val = double;
    __device__ __forceinline__ void add(const Geo &G, int v, long long c, double inc) const {
        if (chk(p + G.sv * v + c, 8)) p[G.sv * v + c] = p[G.sv * v + c] + inc;
    }
    __device__ __forceinline__ Val load(const Geo &G, int v, long long c) const { return get(G, v, c); }
    __device__ __forceinline__ static void inc(Val &x, double d) { x = x + d; }
    __device__ __forceinline__ void store(const Geo &G, int v, long long c, Val x) const { set(G, v, c, x); }
    __device__ __forceinline__ const double *faces() const { return p; }
};

// compensated add of an FP32 increment to a normalised (hi, lo) pair: Knuth's
// two-sum of hi and inc, the rounding error folded into lo, then renormalised
__device__ __forceinline__ void add_hl(float &hi, float &lo, float inc) {
    const float s = hi + inc;
    const float bp = s - hi;
    const float e = (hi - (s - bp)) + (inc - bp);
    const float l = lo + e;
    const float h = s + l;
    lo = l - (h - s);
    hi = h;
}

// Compensated FP32 state: value = hi + lo with |lo| <= ulp(hi)/2 (renormalised on
// every write), hi planes at hi + v*sv and lo planes at lo + v*sv.
struct StoreHL {
    using T = float;
    float *hi, *lo;
    __device__ __forceinline__ double get(const Geo &G, int v, long long c) const {
        if (!chk(hi + G.sv * v + c, 4) || !chk(lo + G.sv * v + c, 4)) return 0.0;
        return (double)hi[G.sv * v + c] + (double)lo[G.sv * v + c];
    }
    __device__ __forceinline__ double getr(const Geo &G, int v, long long c) const {
        return (double)ld(hi + G.sv * v + c) + (double)ld(lo + G.sv * v + c);
    }
    __device__ __forceinline__ void set(const Geo &G, int v, long long c, double x) const {
        if (!chk(hi + G.sv * v + c, 4) || !chk(lo + G.sv * v + c, 4)) return;
        const float h = (float)x;
        hi[G.sv * v + c] = h;
        lo[G.sv * v + c] = (float)(x - (double)h);
    }
    __device__ __forceinline__ void add(const Geo &G, int v, long long c, float inc) const {
        if (!chk(hi + G.sv * v + c, 4) || !chk(lo + G.sv * v + c, 4)) return;
        float h = hi[G.sv * v + c], l = lo[G.sv * v + c];
        add_hl(h, l, inc);
        hi[G.sv * v + c] = h;
        lo[G.sv * v + c] = l;
    }
    struct Val {
        float h, l;
    };
    __device__ __forceinline__ Val load(const Geo &G, int v, long long c) const {
        if (!chk(hi + G.sv * v + c, 4) || !chk(lo + G.sv * v + c, 4)) return Val{0.0f, 0.0f};
        return Val{hi[G.sv * v + c], lo[G.sv * v + c]};
    }
    __device__ __forceinline__ static void inc(Val &x, float d) { add_hl(x.h, x.l, d); }
    __device__ __forceinline__ void store(const Geo &G, int v, long long c, Val x) const {
        if (!chk(hi + G.sv * v + c, 4) || !chk(lo + G.sv * v + c, 4)) return;
        hi[G.sv * v + c] = x.h;
        lo[G.sv * v + c] = x.l;
    }
    __device__ __forceinline__ const float *faces() const { return hi; }
};

// ---------------------------------------------------------------------------
// small scalar kernels
// ---------------------------------------------------------------------------
__global__ void k_set_scalars(Scalars *S, double dt, double time, int set_dt, int set_time) {
    if (set_dt) S->dt = dt;
    if (set_time) S->time = time;
}

__global__ void k_advance_time(Scalars *S) { S->time = S->time + S->dt; }

__global__ void k_dt_reset(Geo G, Scalars *S) {
    // dt = courant*dx/smallc before the minimum (physics.f90:40)
    double d0 = G.courant * G.dx / kSmallc;
    S->red = (unsigned long long)__double_as_longlong(d0);
}

__global__ void k_dt_final(Geo G, Scalars *S) {
    double m = __longlong_as_double((long long)S->red);
    double dt = G.courant * m;
    if (!(dt > 0.0) || !isfinite(dt)) S->err = DG_ERR_DT;
    // after a failed CFL pass (a non-finite state, or no valid step) the steps that dg_run has
    // already enqueued behind it run with dt = 0 and change nothing; the host reports the error
    S->dt = S->err ? 0.0 : dt;
}

// primitive variables of one cell in FP64 (scheme.f90:44-86); the right faces are the
// neighbour's left faces (the frozen right z-face when ndim = 2)
template <class Store>
__device__ __forceinline__ void prim_cell(const Geo &G, const Store &U, long long c, double dt, double q[8]) {
    const double one = 1.0, half = 0.5, two = 2.0;
    const double d = U.getr(G, IR, c);
    q[IR] = mx(d, kSmallr);
    q[IU] = U.getr(G, IU, c) / d;
    q[IV] = U.getr(G, IV, c) / d;
    q[IW] = U.getr(G, IW, c) / d;
    q[IA] = half * (U.getr(G, IA, c) + U.getr(G, IA, c + 1));
    // the right faces: the neighbour's left face, or the stored frozen copy (B_y, B_z in 1D,
    // B_z in 2D: the reference never refreshes those)
    if (G.ndim > 1) q[IB] = half * (U.getr(G, IB, c) + U.getr(G, IB, c + G.sy));
    else q[IB] = half * (U.getr(G, IB, c) + U.getr(G, 8, c));
    if (G.ndim == 3) q[IC] = half * (U.getr(G, IC, c) + U.getr(G, IC, c + G.sz));
    else q[IC] = half * (U.getr(G, IC, c) + U.getr(G, G.ndim == 1 ? 9 : 8, c));
    if (G.iso) {
        q[IP] = d * (G.ciso * G.ciso);
    } else {
        const double smallp = G.smallp;
        double eken = half * (q[IU] * q[IU] + q[IV] * q[IV] + q[IW] * q[IW]);
        double emag = half * (q[IA] * q[IA] + q[IB] * q[IB] + q[IC] * q[IC]);
        double eint = (U.getr(G, IP, c) - emag) / d - eken;
        q[IP] = mx((G.gamma - one) * q[IR] * eint, smallp);
    }
    if (G.omega0 > 0.0) {
        double dvx = two * G.omega0 * q[IV];
        double dvy = -(half * G.omega0 * q[IU]);
        q[IU] = q[IU] + dvx * dt * half;
        q[IV] = q[IV] + dvy * dt * half;
    }
}

// comp_speed, physics.f90:148-164
__device__ __forceinline__ double comp_speed(double gamma, double rho, double p, double v, double bn, double bt1,
                                             double bt2) {
    const double half = 0.5;
    double c2 = gamma * p / rho;
    double b2 = bn * bn + bt1 * bt1 + bt2 * bt2;
    double d2 = half * (c2 + b2 / rho);
    double cf = sqrt(d2 + sqrt(d2 * d2 - c2 * bn * bn / rho));
    return cf + fabs(v);
}

// compute_dt (physics.f90:42-121) fused with the primitive variables of the next godunov
// (FP64 path): one pass over the ghosted grid writes Q = primitive(0) (prim_cell with dt = 0,
// no rotation half-kick) and reduces the CFL time step over the active cells; the
// half-kick of primitive(dt) (scheme.f90:78-85) is added once dt is known (k_kick64), to the
// same unkicked values in the same order, so Q ends as primitive(dt) bit for bit
template <class Store>
__global__ void __launch_bounds__(kThreads) k_prim_dt(Geo G, Store U, double *__restrict__ Q, Scalars *S) {
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    const long long n = (long long)ni * nj * nk;
    double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
    int bad = 0;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) {
        int i, j, k;
        split3((unsigned)t, G.dPX, G.dPY, i, j, k);
        i -= 2;
        j = (G.ndim > 1) ? j - 2 : 1;
        k = (G.ndim == 3) ? k - 2 : 1;
        const long long c = G.idx(i, j, k);
        double q[8];
        prim_cell(G, U, c, 0.0, q);
        if (chk(Q + c, 8) && chk(Q + G.sv * 7 + c, 8)) {
#pragma unroll
            for (int v = 0; v < 8; v++) Q[G.sv * v + c] = q[v];
        }
        if (i >= 1 && i <= G.nx && j >= 1 && j <= G.ny && k >= 1 && k <= G.nz) {
            double velx = comp_speed(G.gamma, q[IR], q[IP], q[IU], q[IA], q[IB], q[IC]);
            if (G.nx == 1) velx = 0.0;
            double vely = comp_speed(G.gamma, q[IR], q[IP], q[IV], q[IB], q[IC], q[IA]);
            if ((G.omega0 > 0.0) && !G.fargo) vely = vely + 1.5 * G.omega0 * (G.xmax - G.xmin) * 0.5;
            if (G.ny == 1) vely = 0.0;
            double cdt;
            if (G.ndim == 1) {
                cdt = G.dx / velx;  // physics.f90:101-103
            } else if (G.ndim == 3) {
                double velz = comp_speed(G.gamma, q[IR], q[IP], q[IW], q[IC], q[IA], q[IB]);
                if (G.nz == 1) velz = 0.0;
                cdt = 1.0 / (G.per_dx(velx) + G.per_dy(vely) + G.per_dz(velz));
            } else {
                cdt = 1.0 / (G.per_dx(velx) + G.per_dy(vely));
            }
            if (!(cdt > 0.0)) bad = 1;  // NaN or non-positive
            else best = mn(best, cdt);
        }
    }
    unsigned long long b = (unsigned long long)__double_as_longlong(best);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
        b = ob < b ? ob : b;
    }
    __shared__ unsigned long long sb[kThreads / 32];
    if ((threadIdx.x & 31) == 0) sb[threadIdx.x >> 5] = b;
    if (bad) S->err = DG_ERR_STATE;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long m = sb[0];
        for (int w = 1; w < kThreads / 32; w++) m = sb[w] < m ? sb[w] : m;
        // one block per 128 cells: skip the atomic when the running minimum is already smaller
        if (m < *(volatile unsigned long long *)&S->red) atomicMin(&S->red, m);
    }
}

// ---------------------------------------------------------------------------
// primitive variables on the ghosted grid (cells with a right neighbour)
// ---------------------------------------------------------------------------
template <typename T, class Store>
__global__ void __launch_bounds__(kThreads) k_prim(Geo G, Store U, T *__restrict__ Q, const Scalars *S) {
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    const long long n = (long long)ni * nj * nk;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i, j, k;
    split3((unsigned)t, G.dPX, G.dPY, i, j, k);
    i -= 2;
    j = (G.ndim > 1) ? j - 2 : 1;
    k = (G.ndim == 3) ? k - 2 : 1;
    const long long c = G.idx(i, j, k);
    double q[8];
    prim_cell(G, U, c, S->dt, q);
#pragma unroll
    for (int v = 0; v < 8; v++) Q[G.sv * v + c] = (T)q[v];
}

// the slope limiter of slope() for slope_type 1 and 2 (scheme.f90:450-458)
template <typename T>
__device__ __forceinline__ T limit1(T st, T qm1, T q0, T qp1) {
    const T half = T(0.5);
    T dlft = st * (q0 - qm1);
    T drgt = st * (qp1 - q0);
    T dcen;
    if constexpr (sizeof(T) == 4) dcen = (dlft + drgt) * (half / st);  // FP32: one shared reciprocal
    // FP64: every caller passes st = 1 or 2, whose reciprocal is exact, so the product rounds
    // the same real number as the reference's division by st (no FP64 division)
    else dcen = half * (dlft + drgt) * (st == T(1) ? T(1) : T(0.5));
    T dsgn = sgn1(dcen);
    T slop = mn(fab(dlft), fab(drgt));
    T dlim = slop;
    if ((dlft * drgt) <= T(0)) dlim = T(0);
    return dsgn * mn(dlim, fab(dcen));
}

// ---------------------------------------------------------------------------
// edge electric fields and trace
// ---------------------------------------------------------------------------
template <typename T>
struct QV {
    const T *Q;
    const T *B;  // face-B planes (IA..IC) of the state, left faces
    Geo G;
    __device__ __forceinline__ T q(int v, int i, int j, int k) const { return ld(Q + G.sv * v + G.idx(i, j, k)); }
    __device__ __forceinline__ T bf(int c, int i, int j, int k) const { return ld(B + G.sv * (IA + c) + G.idx(i, j, k)); }
};

// edge electric fields of trace3d (scheme.f90:1194-1239)
template <typename T>
__device__ __forceinline__ T Ex_at(const QV<T> &a, int i, int j, int k) {
    const T forth = T(0.25), half = T(0.5);
    T v = forth * (a.q(IV, i, j - 1, k - 1) + a.q(IV, i, j - 1, k) + a.q(IV, i, j, k - 1) + a.q(IV, i, j, k));
    T w = forth * (a.q(IW, i, j - 1, k - 1) + a.q(IW, i, j - 1, k) + a.q(IW, i, j, k - 1) + a.q(IW, i, j, k));
    T B = half * (a.bf(1, i, j, k - 1) + a.bf(1, i, j, k));
    T C = half * (a.bf(2, i, j - 1, k) + a.bf(2, i, j, k));
    T e = v * C - w * B;
    if ((a.G.omega0 > 0.0) && !a.G.fargo) {
        T shear = (T)(-1.5 * a.G.omega0 * a.G.xc(i));
        e = e + shear * C;
    }
    return e;
}
template <typename T>
__device__ __forceinline__ T Ey_at(const QV<T> &a, int i, int j, int k) {
    const T forth = T(0.25), half = T(0.5);
    T u = forth * (a.q(IU, i - 1, j, k - 1) + a.q(IU, i - 1, j, k) + a.q(IU, i, j, k - 1) + a.q(IU, i, j, k));
    T w = forth * (a.q(IW, i - 1, j, k - 1) + a.q(IW, i - 1, j, k) + a.q(IW, i, j, k - 1) + a.q(IW, i, j, k));
    T A = half * (a.bf(0, i, j, k - 1) + a.bf(0, i, j, k));
    T C = half * (a.bf(2, i - 1, j, k) + a.bf(2, i, j, k));
    return w * A - u * C;
}
template <typename T>
__device__ __forceinline__ T Ez_at(const QV<T> &a, int i, int j, int k) {
    const T forth = T(0.25), half = T(0.5);
    T u = forth * (a.q(IU, i - 1, j - 1, k) + a.q(IU, i - 1, j, k) + a.q(IU, i, j - 1, k) + a.q(IU, i, j, k));
    T v = forth * (a.q(IV, i - 1, j - 1, k) + a.q(IV, i - 1, j, k) + a.q(IV, i, j - 1, k) + a.q(IV, i, j, k));
    T A = half * (a.bf(0, i, j - 1, k) + a.bf(0, i, j, k));
    T B = half * (a.bf(1, i - 1, j, k) + a.bf(1, i, j, k));
    T e = u * B - v * A;
    if ((a.G.omega0 > 0.0) && !a.G.fargo) {
        T shear = (T)(-1.5 * a.G.omega0 * 0.5 * (a.G.xc(i) + a.G.xc(i - 1)));
        e = e - shear * A;
    }
    return e;
}
// trace2d's edge field (scheme.f90:856-872)
template <typename T>
__device__ __forceinline__ T Ez2_at(const QV<T> &a, int i, int j) {
    const int k = 1;
    T u = T(0.25) * (a.q(IU, i - 1, j - 1, k) + a.q(IU, i - 1, j, k) + a.q(IU, i, j - 1, k) + a.q(IU, i, j, k));
    T v = T(0.25) * (a.q(IV, i - 1, j - 1, k) + a.q(IV, i - 1, j, k) + a.q(IV, i, j - 1, k) + a.q(IV, i, j, k));
    T A = T(0.5) * (a.bf(0, i, j - 1, k) + a.bf(0, i, j, k));
    T B = T(0.5) * (a.bf(1, i - 1, j, k) + a.bf(1, i, j, k));
    return u * B - v * A;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_efield3d(Geo G, const T *__restrict__ Q, const T *__restrict__ Bf,
                                                       T *__restrict__ Ex, T *__restrict__ Ey, T *__restrict__ Ez) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.esz) return;
    int i, j, k;
    split3((unsigned)t, G.dEX, G.dEY, i, j, k);
    k += G.ke0;
    const QV<T> a{Q, Bf, G};
    Ex[t] = Ex_at(a, i, j, k);
    Ey[t] = Ey_at(a, i, j, k);
    Ez[t] = Ez_at(a, i, j, k);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_efield2d(Geo G, const T *__restrict__ Q, const T *__restrict__ Bf,
                                                       T *__restrict__ Ez) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.esz) return;
    const int j = (int)fdiv((unsigned)t, G.dEX);
    const int i = (int)((unsigned)t - (unsigned)j * G.dEX.d);
    const QV<T> a{Q, Bf, G};
    Ez[t] = Ez2_at(a, i, j);
}

template <typename T>
__device__ __forceinline__ void cell_slopes2(const QV<T> &a, int v, int i, int j, T d[2]) {
    const int st = a.G.slope_type, k = 1;
    if (st == 0) { d[0] = d[1] = T(0); return; }
    const T c = a.q(v, i, j, k);
    if (st < 3) {
        const T s = (T)st;
        d[0] = limit1(s, a.q(v, i - 1, j, k), c, a.q(v, i + 1, j, k));
        d[1] = limit1(s, a.q(v, i, j - 1, k), c, a.q(v, i, j + 1, k));
        return;
    }
    // scheme.f90:355-391, including its choice of neighbours
    const T half = T(0.5), one = T(1);
    T e[9] = {a.q(v, i - 1, j - 1, k) - c, a.q(v, i - 1, j, k) - c, a.q(v, i, j - 1, k) - c,
              a.q(v, i, j - 1, k) - c,     a.q(v, i, j, k) - c,     a.q(v, i, j + 1, k) - c,
              a.q(v, i + 1, j - 1, k) - c, a.q(v, i + 1, j, k) - c, a.q(v, i + 1, j + 1, k) - c};
    T vmin = e[0], vmax = e[0];
#pragma unroll
    for (int n = 1; n < 9; n++) { vmin = mn(vmin, e[n]); vmax = mx(vmax, e[n]); }
    T dfx = half * (a.q(v, i + 1, j, k) - a.q(v, i - 1, j, k));
    T dfy = half * (a.q(v, i, j + 1, k) - a.q(v, i, j - 1, k));
    T dff = half * (fab(dfx) + fab(dfy));
    T slop = (dff > T(0)) ? mn(one, mn(fab(vmin), fab(vmax)) / dff) : one;
    d[0] = slop * dfx; d[1] = slop * dfy;
}

// transverse slope of a face-B component c (0,1,2) at face (i,j,k) along direction dir
template <typename T>
__device__ __forceinline__ T face_slope(const QV<T> &a, int c, int dir, int i, int j, int k) {
    const int st = a.G.slope_type;
    if (st == 0) return T(0);
    const T s = (T)mn(st, 2);
    int di = dir == 0, dj = dir == 1, dk = dir == 2;
    return limit1(s, a.bf(c, i - di, j - dj, k - dk), a.bf(c, i, j, k), a.bf(c, i + di, j + dj, k + dk));
}

// resident blocks of 128 threads per SM that the trace and Riemann kernels are compiled
// for (register caps 128/80 for the trace, 128/64 for the Riemann kernel, FP64/FP32),
// chosen by timing the variants at 256^3
#ifndef DG_TRACE_MINB64
#define DG_TRACE_MINB64 4
#endif
#ifndef DG_TRACE_MINB32
#define DG_TRACE_MINB32 6
#endif
#ifndef DG_RIEMANN_MINB64
#define DG_RIEMANN_MINB64 4
#endif
#ifndef DG_RIEMANN_MINB32
#define DG_RIEMANN_MINB32 8
#endif
// kPart selects the core fields a launch writes: 0 all 47; 1 the predicted cell state and the
// cell slopes (fields 0-28); 2 the predicted face fields and their transverse slopes (29-46).
// The values a part does not write are not computed (their expressions are dead code), and
// every written value is the same expression of the same inputs in all forms.
#ifndef DG_TRACEC_MINB64
#define DG_TRACEC_MINB64 5
#endif
#ifndef DG_TRACEF_MINB64
#define DG_TRACEF_MINB64 6
#endif
#ifndef DG_TRACEC_MINB32
#define DG_TRACEC_MINB32 6
#endif
#ifndef DG_TRACEF_MINB32
#define DG_TRACEF_MINB32 8
#endif
template <typename T, int kPart>
constexpr int trace_minb() {
    return sizeof(T) == 8 ? (kPart == 0 ? DG_TRACE_MINB64 : kPart == 1 ? DG_TRACEC_MINB64 : DG_TRACEF_MINB64)
                          : (kPart == 0 ? DG_TRACE_MINB32 : kPart == 1 ? DG_TRACEC_MINB32 : DG_TRACEF_MINB32);
}
// The 3D trace of one cell (slope + trace3d, scheme.f90:253-656, 1149-1711) written once over a
// stencil accessor that reads, relative to the cell (i, j, k):
//   a.q(v, di, dj, dk)   primitive variable v of cell (i+di, j+dj, k+dk)
//   a.bf(c, di, dj, dk)  left-face field component c of that cell
//   a.ex(dj, dk), a.ey(di, dk), a.ez(di, dj)   the trace's edge fields at (i, j+dj, k+dk),
//                        (i+di, j, k+dk) and (i+di, j+dj, k)
// k_trace3d reads through global memory, k_trace3d_tile through shared-memory planes; both
// evaluate the same expressions of the same values.
template <typename T>
struct GStencil {
    QV<T> a;
    const T *Ex, *Ey, *Ez;
    int i, j, k;
    __device__ __forceinline__ T q(int v, int di, int dj, int dk) const { return a.q(v, i + di, j + dj, k + dk); }
    __device__ __forceinline__ T bf(int c, int di, int dj, int dk) const { return a.bf(c, i + di, j + dj, k + dk); }
    __device__ __forceinline__ T ex(int dj, int dk) const { return ld(Ex + a.G.eidx(i, j + dj, k + dk)); }
    __device__ __forceinline__ T ey(int di, int dk) const { return ld(Ey + a.G.eidx(i + di, j, k + dk)); }
    __device__ __forceinline__ T ez(int di, int dj) const { return ld(Ez + a.G.eidx(i + di, j + dj, k)); }
};

// limited cell slopes of variable v in the three directions (slope_type st = 1..3)
template <typename T, class Sten>
__device__ __forceinline__ void cell_slopes3s(const Sten &a, int v, int st, T d[3]) {
    if (st == 0) { d[0] = d[1] = d[2] = T(0); return; }
    const T c = a.q(v, 0, 0, 0);
    if (st < 3) {
        const T s = (T)st;
        d[0] = limit1(s, a.q(v, -1, 0, 0), c, a.q(v, 1, 0, 0));
        d[1] = limit1(s, a.q(v, 0, -1, 0), c, a.q(v, 0, 1, 0));
        d[2] = limit1(s, a.q(v, 0, 0, -1), c, a.q(v, 0, 0, 1));
        return;
    }
    // multidimensional limiter, scheme.f90:484-557
    const T half = T(0.5), one = T(1);
    T vmin = T(0), vmax = T(0);
#pragma unroll
    for (int dk = -1; dk <= 1; dk++)
#pragma unroll
        for (int di = -1; di <= 1; di++)
#pragma unroll
            for (int dj = -1; dj <= 1; dj++) {
                T e = a.q(v, di, dj, dk) - c;
                if (dk == -1 && di == -1 && dj == -1) { vmin = e; vmax = e; }
                else { vmin = mn(vmin, e); vmax = mx(vmax, e); }
            }
    T dfx = half * (a.q(v, 1, 0, 0) - a.q(v, -1, 0, 0));
    T dfy = half * (a.q(v, 0, 1, 0) - a.q(v, 0, -1, 0));
    T dfz = half * (a.q(v, 0, 0, 1) - a.q(v, 0, 0, -1));
    T dff = half * (fab(dfx) + fab(dfy) + fab(dfz));
    T slop = (dff > T(0)) ? mn(one, mn(fab(vmin), fab(vmax)) / dff) : one;
    d[0] = slop * dfx; d[1] = slop * dfy; d[2] = slop * dfz;
}

// transverse slope of face-B component c of the face at offset (di, dj, dk) along direction dir
template <typename T, class Sten>
__device__ __forceinline__ T face_slope_s(const Sten &a, int c, int dir, int di, int dj, int dk, int st) {
    if (st == 0) return T(0);
    const T s = (T)mn(st, 2);
    const int ei = dir == 0, ej = dir == 1, ek = dir == 2;
    return limit1(s, a.bf(c, di - ei, dj - ej, dk - ek), a.bf(c, di, dj, dk), a.bf(c, di + ei, dj + ej, dk + ek));
}

// the trace core of cell (i, ., .) from its stencil, stored at o (field f at o[f * kCoreLane]);
// kPart: 0 all 47 fields, 1 the predicted cell state and cell slopes (0-28), 2 the predicted
// face fields and their transverse slopes (29-46)
template <typename T, int kPart, class Sten>
__device__ __forceinline__ void trace3_cell(const Sten &a, const Geo &G, int i, double dtd, T *o) {
    const int st = G.slope_type;
    const T half = T(0.5), gamma = (T)G.gamma;
    const T dtdx = (T)(dtd / G.dx), dtdy = (T)(dtd / G.dy), dtdz = (T)(dtd / G.dz), dx = (T)G.dx;

    const T r = a.q(IR, 0, 0, 0), u = a.q(IU, 0, 0, 0), v = a.q(IV, 0, 0, 0), w = a.q(IW, 0, 0, 0);
    const T p = a.q(IP, 0, 0, 0), A = a.q(IA, 0, 0, 0), B = a.q(IB, 0, 0, 0), C = a.q(IC, 0, 0, 0);
    T d3[3];
    cell_slopes3s<T>(a, IR, st, d3); const T drx = half * d3[0], dry = half * d3[1], drz = half * d3[2];
    cell_slopes3s<T>(a, IU, st, d3); const T dux = half * d3[0], duy = half * d3[1], duz = half * d3[2];
    cell_slopes3s<T>(a, IV, st, d3); const T dvx = half * d3[0], dvy = half * d3[1], dvz = half * d3[2];
    cell_slopes3s<T>(a, IW, st, d3); const T dwx = half * d3[0], dwy = half * d3[1], dwz = half * d3[2];
    cell_slopes3s<T>(a, IP, st, d3); const T dpx = half * d3[0], dpy = half * d3[1], dpz = half * d3[2];
    cell_slopes3s<T>(a, IA, st, d3); const T dAy = half * d3[1], dAz = half * d3[2];
    cell_slopes3s<T>(a, IB, st, d3); const T dBx = half * d3[0], dBz = half * d3[2];
    cell_slopes3s<T>(a, IC, st, d3); const T dCx = half * d3[0], dCy = half * d3[1];

    const T AL = a.bf(0, 0, 0, 0), AR = a.bf(0, 1, 0, 0);
    const T BL = a.bf(1, 0, 0, 0), BR = a.bf(1, 0, 1, 0);
    const T CL = a.bf(2, 0, 0, 0), CR = a.bf(2, 0, 0, 1);
    const T dAx = half * (AR - AL), dBy = half * (BR - BL), dCz = half * (CR - CL);

    const T dALy = half * face_slope_s<T>(a, 0, 1, 0, 0, 0, st), dARy = half * face_slope_s<T>(a, 0, 1, 1, 0, 0, st);
    const T dALz = half * face_slope_s<T>(a, 0, 2, 0, 0, 0, st), dARz = half * face_slope_s<T>(a, 0, 2, 1, 0, 0, st);
    const T dBLx = half * face_slope_s<T>(a, 1, 0, 0, 0, 0, st), dBRx = half * face_slope_s<T>(a, 1, 0, 0, 1, 0, st);
    const T dBLz = half * face_slope_s<T>(a, 1, 2, 0, 0, 0, st), dBRz = half * face_slope_s<T>(a, 1, 2, 0, 1, 0, st);
    const T dCLx = half * face_slope_s<T>(a, 2, 0, 0, 0, 0, st), dCRx = half * face_slope_s<T>(a, 2, 0, 0, 0, 1, st);
    const T dCLy = half * face_slope_s<T>(a, 2, 1, 0, 0, 0, st), dCRy = half * face_slope_s<T>(a, 2, 1, 0, 0, 1, st);

    const T ELL = a.ex(0, 0), ELR = a.ex(0, 1), ERL = a.ex(1, 0), ERR = a.ex(1, 1);
    const T FLL = a.ey(0, 0), FLR = a.ey(0, 1), FRL = a.ey(1, 0), FRR = a.ey(1, 1);
    const T GLL = a.ez(0, 0), GLR = a.ez(0, 1), GRL = a.ez(1, 0), GRR = a.ez(1, 1);

    // source terms, scheme.f90:1351-1389
    T sr0 = (-u * drx - dux * r) * dtdx + (-v * dry - dvy * r) * dtdy + (-w * drz - dwz * r) * dtdz;
    T su0 = (-u * dux - (dpx + B * dBx + C * dCx) / r) * dtdx + (-v * duy + B * dAy / r) * dtdy
          + (-w * duz + C * dAz / r) * dtdz;
    T sv0 = (-u * dvx + A * dBx / r) * dtdx + (-v * dvy - (dpy + A * dAy + C * dCy) / r) * dtdy
          + (-w * dvz + C * dBz / r) * dtdz;
    T sw0 = (-u * dwx + A * dCx / r) * dtdx + (-v * dwy + B * dCy / r) * dtdy
          + (-w * dwz - (dpz + A * dAz + B * dBz) / r) * dtdz;
    T sp0 = (-u * dpx - dux * gamma * p) * dtdx + (-v * dpy - dvy * gamma * p) * dtdy
          + (-w * dpz - dwz * gamma * p) * dtdz;
    T sA0 = (u * dBy + B * duy - v * dAy - A * dvy) * dtdy + (u * dCz + C * duz - w * dAz - A * dwz) * dtdz;
    T sB0 = (v * dAx + A * dvx - u * dBx - B * dux) * dtdx + (v * dCz + C * dvz - w * dBz - B * dwz) * dtdz;
    T sC0 = (w * dAx + A * dwx - u * dCx - C * dux) * dtdx + (w * dBy + B * dwy - v * dCy - C * dvy) * dtdy;
    if ((G.omega0 > 0.0) && !G.fargo) {
        const T Omega0 = (T)G.omega0;
        const T shear = (T)(-1.5 * G.omega0 * G.xc(i));
        sr0 = sr0 - shear * dry * dtdy;
        su0 = su0 - shear * duy * dtdy;
        sv0 = sv0 - shear * dvy * dtdy;
        sw0 = sw0 - shear * dwy * dtdy;
        sp0 = sp0 - shear * dpy * dtdy;
        sA0 = sA0 - shear * dAy * dtdy;
        sB0 = sB0 + (shear * dAx - T(1.5) * Omega0 * A * dx) * dtdx + shear * dBz * dtdz;
        sC0 = sC0 - shear * dCy * dtdy;
    }
    const T sAL0 = +(GLR - GLL) * dtdy * half - (FLR - FLL) * dtdz * half;
    const T sAR0 = +(GRR - GRL) * dtdy * half - (FRR - FRL) * dtdz * half;
    const T sBL0 = -(GRL - GLL) * dtdx * half + (ELR - ELL) * dtdz * half;
    const T sBR0 = -(GRR - GLR) * dtdx * half + (ERR - ERL) * dtdz * half;
    const T sCL0 = +(FRL - FLL) * dtdx * half - (ERL - ELL) * dtdy * half;
    const T sCR0 = +(FRR - FLR) * dtdx * half - (ERR - ELR) * dtdy * half;

    const int cs = kCoreLane;
    if (!chk(o, ((kCore3 - 1) * cs + 1) * sizeof(T))) return;
    if constexpr (kPart != 2) {
        o[0 * cs] = r + sr0; o[1 * cs] = u + su0; o[2 * cs] = v + sv0; o[3 * cs] = w + sw0;
        o[4 * cs] = p + sp0; o[5 * cs] = A + sA0; o[6 * cs] = B + sB0; o[7 * cs] = C + sC0;
        o[8 * cs] = drx; o[9 * cs] = dux; o[10 * cs] = dvx; o[11 * cs] = dwx; o[12 * cs] = dpx; o[13 * cs] = dBx; o[14 * cs] = dCx;
        o[15 * cs] = dry; o[16 * cs] = duy; o[17 * cs] = dvy; o[18 * cs] = dwy; o[19 * cs] = dpy; o[20 * cs] = dAy; o[21 * cs] = dCy;
        o[22 * cs] = drz; o[23 * cs] = duz; o[24 * cs] = dvz; o[25 * cs] = dwz; o[26 * cs] = dpz; o[27 * cs] = dAz; o[28 * cs] = dBz;
    }
    if constexpr (kPart != 1) {
        o[29 * cs] = AL + sAL0; o[30 * cs] = AR + sAR0; o[31 * cs] = BL + sBL0; o[32 * cs] = BR + sBR0;
        o[33 * cs] = CL + sCL0; o[34 * cs] = CR + sCR0;
        o[35 * cs] = dALy; o[36 * cs] = dARy; o[37 * cs] = dALz; o[38 * cs] = dARz;
        o[39 * cs] = dBLx; o[40 * cs] = dBRx; o[41 * cs] = dBLz; o[42 * cs] = dBRz;
        o[43 * cs] = dCLx; o[44 * cs] = dCRx; o[45 * cs] = dCLy; o[46 * cs] = dCRy;
    }
}

template <typename T, int kPart = 0>
__global__ void __launch_bounds__(kThreads, (trace_minb<T, kPart>()))
k_trace3d(Geo G, const T *__restrict__ Q, const T *__restrict__ Bf, const T *__restrict__ Exa,
          const T *__restrict__ Eya, const T *__restrict__ Eza, T *__restrict__ core, const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.csz) return;
    int i, j, k;
    split3((unsigned)t, G.dCX, G.dCY, i, j, k);
    k += G.kc0;
    const GStencil<T> a{QV<T>{Q, Bf, G}, Exa, Eya, Eza, i, j, k};
    trace3_cell<T, kPart>(a, G, i, S->dt, core + core_base(t, kCore3));
}

// ---------------------------------------------------------------------------
// The 3D trace with its stencil staged in shared memory.  A block of kThreads threads owns a
// tile of kTX x kTY cells in (x, y) and marches along z through kTZ planes of the core index
// space.  Shared memory holds a ring of kRingQ z planes (k-1, k, k+1 and the one being
// fetched) of the tile plus a one-cell halo in x and y, with the primitive variables and
// left-face field components the part reads, and a ring of kRingE planes of the trace's edge
// fields (scheme.f90:1194-1239), which the block computes from the staged planes: edge plane
// k+1 needs the cell planes k and k+1 only.  Planes arrive by cp.async (element copies, so no
// alignment rule applies to the ghosted rows); cell plane k+2 is fetched while plane k is
// computed.  Each stencil read is a shared-memory load at a fixed offset from the thread's
// cell.  The parts (kPart as in trace3_cell) stage only what they read: part 1 the 8
// primitives (its four face-B values come from global memory) and no edge fields, part 2 the
// velocities and the face-B components (for the edge fields), part 0 all of them.
// ---------------------------------------------------------------------------
constexpr int kTX = 32, kTY = kThreads / kTX;
constexpr int kTR = kTX + 2;              // row of a staged plane (halo of one cell each side)
constexpr int kTP = kTR * (kTY + 2);      // one field of a staged plane
constexpr int kRingQ = 4, kRingE = 2;
#ifndef DG_TRACE_KZ
#define DG_TRACE_KZ 16
#endif
constexpr int kTZ = DG_TRACE_KZ;
// staged fields of a cell plane; field v (0-7 primitives, 8-10 face-B components) sits at
// slot position tq_pos(v): part 0 all 11, part 1 the 8 primitives, part 2 u, v, w and the face B
template <int kPart> __host__ __device__ constexpr int tq_count() { return kPart == 0 ? NVAR + 3 : kPart == 1 ? NVAR : 6; }
template <int kPart> __host__ __device__ constexpr int tq_field(int f) {  // the field at slot position f
    return kPart == 2 ? (f < 3 ? IU + f : NVAR + f - 3) : f;
}
template <int kPart> __host__ __device__ constexpr int tq_pos(int v) { return kPart == 2 ? (v < NVAR ? v - IU : v - NVAR + 3) : v; }
template <int kPart> __host__ __device__ constexpr bool t_edges() { return kPart != 1; }
template <typename T, int kPart>
constexpr int trace_tile_smem() {
    return (kRingQ * tq_count<kPart>() + (t_edges<kPart>() ? kRingE * 3 : 0)) * kTP * (int)sizeof(T);
}

template <typename T, int kPart>
struct TStencil {
    const T *p0, *p1, *p2;  // this cell in the staged cell planes k-1, k, k+1
    const T *e0, *e1;       // this cell in the edge planes k, k+1
    const T *bg;            // part 1: this cell's left-face component 0 in global memory ...
    long long sv, sy, sz;   // ... and the strides from it
    __device__ __forceinline__ const T *pl(int dk) const { return dk < 0 ? p0 : (dk > 0 ? p2 : p1); }
    __device__ __forceinline__ T q(int v, int di, int dj, int dk) const {
        if constexpr (kPart == 2) return T(0);  // part 2 evaluates no primitive
        else return pl(dk)[tq_pos<kPart>(v) * kTP + dj * kTR + di];
    }
    __device__ __forceinline__ T bf(int c, int di, int dj, int dk) const {
        if constexpr (kPart == 1) return ld(bg + sv * c + sy * dj + sz * dk + di);
        else return pl(dk)[tq_pos<kPart>(NVAR + c) * kTP + dj * kTR + di];
    }
    __device__ __forceinline__ T ex(int dj, int dk) const {
        if constexpr (kPart == 1) return T(0);  // part 1 reads no edge field
        else return (dk ? e1 : e0)[dj * kTR];
    }
    __device__ __forceinline__ T ey(int di, int dk) const {
        if constexpr (kPart == 1) return T(0);
        else return (dk ? e1 : e0)[kTP + di];
    }
    __device__ __forceinline__ T ez(int di, int dj) const {
        if constexpr (kPart == 1) return T(0);
        else return e0[2 * kTP + dj * kTR + di];
    }
};

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// The positions of a staged plane a thread fetches (kTP <= 2 kThreads: at most two), fixed for
// the whole z march: the cell of position n of plane k is c[n] + (k - k0) sz.
struct FetchPos {
    long long c[2];  // cell index at plane k0
    int q[2];        // position in the plane, or -1
    bool in[2];      // inside the ghosted grid in x and y
    int k0;
};
__device__ __forceinline__ FetchPos fetch_positions(const Geo &G, int i0, int j0, int k0) {
    FetchPos P;
    P.k0 = k0;
#pragma unroll
    for (int n = 0; n < 2; n++) {
        const int q = threadIdx.x + n * kThreads;
        const int ii = q % kTR, jj = q / kTR;
        const int i = i0 - 1 + ii, j = j0 - 1 + jj;
        P.q[n] = q < kTP ? q : -1;
        P.in[n] = q < kTP && i + 2 >= 0 && i + 2 < G.NX && j + G.gy - 1 >= 0 && j + G.gy - 1 < G.NY;
        P.c[n] = P.in[n] ? G.idx(i, j, k0) : 0;
    }
    return P;
}

// fetch the staged fields of cell plane k (tile + halo) into slot s: cp.async element copies,
// or zeros where the cell is outside the ghosted grid
template <typename T, int kPart>
__device__ __forceinline__ void fetch_qplane(const Geo &G, const T *Q, const T *Bf, T *s, const FetchPos &P, int k) {
    const bool kok = k + G.gz - 1 >= 0 && k + G.gz - 1 < G.NZ;
    const long long dk = (long long)(k - P.k0) * G.sz;
#pragma unroll
    for (int n = 0; n < 2; n++) {
        if (P.q[n] < 0) continue;
        T *d = s + P.q[n];
        const long long c = P.c[n] + dk;
#pragma unroll
        for (int f = 0; f < tq_count<kPart>(); f++) {
            const int v = tq_field<kPart>(f);
            const T *src = (v < NVAR ? Q + G.sv * v : Bf + G.sv * (IA + v - NVAR)) + c;
            if (kok && P.in[n] && chk(src, sizeof(T))) {
                const unsigned a = (unsigned)__cvta_generic_to_shared(d + f * kTP);
                if constexpr (sizeof(T) == 4)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(src) : "memory");
                else
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(src) : "memory");
            } else {
                d[f * kTP] = T(0);
            }
        }
    }
}

// the trace's edge fields of plane k (Ex_at, Ey_at, Ez_at on the staged cell planes lo = k-1
// and hi = k) for the edges i0..i0+kTX, j0..j0+kTY, into slot s at the cells' positions
template <typename T, int kPart>
__device__ __forceinline__ void edge_plane(const Geo &G, const T *lo, const T *hi, T *s, int i0) {
    constexpr int pU = tq_pos<kPart>(IU) * kTP, pV = tq_pos<kPart>(IV) * kTP, pW = tq_pos<kPart>(IW) * kTP;
    constexpr int pA = tq_pos<kPart>(NVAR) * kTP, pB = tq_pos<kPart>(NVAR + 1) * kTP, pC = tq_pos<kPart>(NVAR + 2) * kTP;
    const T forth = T(0.25), half = T(0.5);
    const bool shear = (G.omega0 > 0.0) && !G.fargo;
    for (int q = threadIdx.x; q < (kTX + 1) * (kTY + 1); q += kThreads) {
        const int ii = 1 + q % (kTX + 1), jj = 1 + q / (kTX + 1);
        const int o = jj * kTR + ii;                    // edge (i, j) sits at cell (i, j)
        const int ojm = o - kTR, oim = o - 1, oimjm = o - kTR - 1;
        const int i = i0 - 1 + ii;
        // Ex(i, j, k): cells (i, j-1..j, k-1..k)
        {
            T v = forth * (lo[pV + ojm] + hi[pV + ojm] + lo[pV + o] + hi[pV + o]);
            T w = forth * (lo[pW + ojm] + hi[pW + ojm] + lo[pW + o] + hi[pW + o]);
            T B = half * (lo[pB + o] + hi[pB + o]);
            T C = half * (hi[pC + ojm] + hi[pC + o]);
            T e = v * C - w * B;
            if (shear) {
                T sh = (T)(-1.5 * G.omega0 * G.xc(i));
                e = e + sh * C;
            }
            s[o] = e;
        }
        // Ey(i, j, k): cells (i-1..i, j, k-1..k)
        {
            T u = forth * (lo[pU + oim] + hi[pU + oim] + lo[pU + o] + hi[pU + o]);
            T w = forth * (lo[pW + oim] + hi[pW + oim] + lo[pW + o] + hi[pW + o]);
            T A = half * (lo[pA + o] + hi[pA + o]);
            T C = half * (hi[pC + oim] + hi[pC + o]);
            s[kTP + o] = w * A - u * C;
        }
        // Ez(i, j, k): cells (i-1..i, j-1..j, k)
        {
            T u = forth * (hi[pU + oimjm] + hi[pU + oim] + hi[pU + ojm] + hi[pU + o]);
            T v = forth * (hi[pV + oimjm] + hi[pV + oim] + hi[pV + ojm] + hi[pV + o]);
            T A = half * (hi[pA + ojm] + hi[pA + o]);
            T B = half * (hi[pB + oim] + hi[pB + o]);
            T e = u * B - v * A;
            if (shear) {
                T sh = (T)(-1.5 * G.omega0 * 0.5 * (G.xc(i) + G.xc(i - 1)));
                e = e - sh * A;
            }
            s[2 * kTP + o] = e;
        }
    }
}

// resident blocks per SM the tiled trace is compiled for, by arithmetic and part (bounded by
// its shared memory: FP64 82/52/49 KB, FP32 41/26/24 KB per block for parts 0/1/2)
#ifndef DG_TRACET_MINB64
#define DG_TRACET_MINB64 2
#endif
#ifndef DG_TRACET1_MINB64
#define DG_TRACET1_MINB64 4
#endif
#ifndef DG_TRACET2_MINB64
#define DG_TRACET2_MINB64 4
#endif
#ifndef DG_TRACET_MINB32
#define DG_TRACET_MINB32 5
#endif
#ifndef DG_TRACET1_MINB32
#define DG_TRACET1_MINB32 6
#endif
#ifndef DG_TRACET2_MINB32
#define DG_TRACET2_MINB32 8
#endif
template <typename T, int kPart>
constexpr int trace_tile_minb() {
    return sizeof(T) == 8 ? (kPart == 0 ? DG_TRACET_MINB64 : kPart == 1 ? DG_TRACET1_MINB64 : DG_TRACET2_MINB64)
                          : (kPart == 0 ? DG_TRACET_MINB32 : kPart == 1 ? DG_TRACET1_MINB32 : DG_TRACET2_MINB32);
}
template <typename T, int kPart = 0>
__global__ void __launch_bounds__(kThreads, (trace_tile_minb<T, kPart>()))
k_trace3d_tile(Geo G, const T *__restrict__ Q, const T *__restrict__ Bf, T *__restrict__ core, const Scalars *S) {
    extern __shared__ __align__(16) unsigned char tsm[];
    constexpr int kQS = tq_count<kPart>() * kTP;  // one cell-plane slot
    T *ringQ = (T *)tsm;
    T *ringE = ringQ + kRingQ * kQS;
    const int i0 = blockIdx.x * kTX, j0 = blockIdx.y * kTY;
    const int kb = G.kc0 + blockIdx.z * kTZ;
    const int ke = min(kb + kTZ, G.kc0 + G.CZ);  // core planes [kb, ke)
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    const int i = i0 + tx, j = j0 + ty;
    const bool mine = i < G.CX && j < G.CY;
    const int own = (ty + 1) * kTR + (tx + 1);  // this cell in a staged plane
    auto qslot = [&](int k) { return ringQ + ((k - kb + 1) % kRingQ) * kQS; };
    auto eslot = [&](int k) { return ringE + ((k - kb) % kRingE) * (3 * kTP); };
    const double dtd = S->dt;
    const FetchPos P = fetch_positions(G, i0, j0, kb - 1);
    fetch_qplane<T, kPart>(G, Q, Bf, qslot(kb - 1), P, kb - 1);
    fetch_qplane<T, kPart>(G, Q, Bf, qslot(kb), P, kb);
    cp_commit();
    fetch_qplane<T, kPart>(G, Q, Bf, qslot(kb + 1), P, kb + 1);
    cp_commit();
    cp_wait_all();
    __syncthreads();
    if constexpr (t_edges<kPart>()) edge_plane<T, kPart>(G, qslot(kb - 1), qslot(kb), eslot(kb), i0);
    for (int k = kb; k < ke; k++) {
        // cell planes k-1 .. k+1 are in, edge plane k is written; fetch cell plane k+2 into the
        // slot of plane k-2 (read last by the trace of plane k-1, before the barrier ending it)
        if (k + 2 <= ke) fetch_qplane<T, kPart>(G, Q, Bf, qslot(k + 2), P, k + 2);
        cp_commit();
        if constexpr (t_edges<kPart>()) {
            edge_plane<T, kPart>(G, qslot(k), qslot(k + 1), eslot(k + 1), i0);  // into the slot of plane k-1
            __syncthreads();
        }
        if (mine) {
            TStencil<T, kPart> a{qslot(k - 1) + own, qslot(k) + own, qslot(k + 1) + own, nullptr, nullptr,
                                 nullptr, G.sv, G.sy, G.sz};
            if constexpr (t_edges<kPart>()) {
                a.e0 = eslot(k) + own;
                a.e1 = eslot(k + 1) + own;
            }
            if constexpr (kPart == 1) a.bg = Bf + G.sv * IA + G.idx(i, j, k);
            const long long t = (long long)i + (long long)G.CX * ((long long)j + (long long)G.CY * (k - G.kc0));
            trace3_cell<T, kPart>(a, G, i, dtd, core + core_base(t, kCore3));
        }
        cp_wait_all();
        __syncthreads();  // cell plane k+2 is in; every thread is done with planes k-1 (cells, edges)
    }
}

// launch k_trace3d_tile over the core index space (its dynamic shared memory is above the
// default 48 KB limit in FP64: the attribute is set once per device)
template <typename T, int kPart = 0>
cudaError_t launch_trace_tile(const Geo &G, const T *Q, const T *Bf, T *core, const Scalars *S, cudaStream_t s) {
    const int smem = trace_tile_smem<T, kPart>();
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        e = cudaFuncSetAttribute(k_trace3d_tile<T, kPart>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    const dim3 grid((unsigned)((G.CX + kTX - 1) / kTX), (unsigned)((G.CY + kTY - 1) / kTY),
                    (unsigned)((G.CZ + kTZ - 1) / kTZ));
    k_trace3d_tile<T, kPart><<<grid, kThreads, smem, s>>>(G, Q, Bf, core, S);
    return cudaSuccess;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_trace2d(Geo G, const T *__restrict__ Q, const T *__restrict__ Bf,
                                                      const T *__restrict__ Eza, T *__restrict__ core,
                                                      const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.csz) return;
    const int j = (int)fdiv((unsigned)t, G.dCX);
    const int i = (int)((unsigned)t - (unsigned)j * G.dCX.d);
    const int k = 1;
    const QV<T> a{Q, Bf, G};
    const double dtd = S->dt;
    const T half = T(0.5), gamma = (T)G.gamma;
    const T dtdx = (T)(dtd / G.dx), dtdy = (T)(dtd / G.dy);

    const T r = a.q(IR, i, j, k), u = a.q(IU, i, j, k), v = a.q(IV, i, j, k), w = a.q(IW, i, j, k);
    const T p = a.q(IP, i, j, k), A = a.q(IA, i, j, k), B = a.q(IB, i, j, k), C = a.q(IC, i, j, k);
    const T AL = a.bf(0, i, j, k), AR = a.bf(0, i + 1, j, k);
    const T BL = a.bf(1, i, j, k), BR = a.bf(1, i, j + 1, k);
    const T ELL = ld(Eza + G.eidx(i, j, 1)), ELR = ld(Eza + G.eidx(i, j + 1, 1));
    const T ERL = ld(Eza + G.eidx(i + 1, j, 1)), ERR = ld(Eza + G.eidx(i + 1, j + 1, 1));
    T d2[2];
    cell_slopes2(a, IR, i, j, d2); const T drx = half * d2[0], dry = half * d2[1];
    cell_slopes2(a, IU, i, j, d2); const T dux = half * d2[0], duy = half * d2[1];
    cell_slopes2(a, IV, i, j, d2); const T dvx = half * d2[0], dvy = half * d2[1];
    cell_slopes2(a, IW, i, j, d2); const T dwx = half * d2[0], dwy = half * d2[1];
    cell_slopes2(a, IP, i, j, d2); const T dpx = half * d2[0], dpy = half * d2[1];
    cell_slopes2(a, IA, i, j, d2); const T dAy = half * d2[1];
    cell_slopes2(a, IB, i, j, d2); const T dBx = half * d2[0];
    cell_slopes2(a, IC, i, j, d2); const T dCx = half * d2[0], dCy = half * d2[1];
    const T dALy = half * face_slope(a, 0, 1, i, j, k), dARy = half * face_slope(a, 0, 1, i + 1, j, k);
    const T dBLx = half * face_slope(a, 1, 0, i, j, k), dBRx = half * face_slope(a, 1, 0, i, j + 1, k);
    const T dAx = half * (AR - AL), dBy = half * (BR - BL);

    // scheme.f90:946-967
    const T sr0 = (-u * drx - dux * r) * dtdx + (-v * dry - dvy * r) * dtdy;
    const T su0 = (-u * dux - dpx / r - B * dBx / r - C * dCx / r) * dtdx + (-v * duy + B * dAy / r) * dtdy;
    const T sv0 = (-u * dvx + A * dBx / r) * dtdx + (-v * dvy - dpy / r - A * dAy / r - C * dCy / r) * dtdy;
    const T sw0 = (-u * dwx + A * dCx / r) * dtdx + (-v * dwy + B * dCy / r) * dtdy;
    const T sp0 = (-u * dpx - dux * gamma * p) * dtdx + (-v * dpy - dvy * gamma * p) * dtdy;
    const T sA0 = (u * dBy + B * duy - v * dAy - A * dvy) * dtdy;
    const T sB0 = (-u * dBx - B * dux + v * dAx + A * dvx) * dtdx;
    T sC0 = (w * dAx + A * dwx - u * dCx - C * dux) * dtdx + (-v * dCy - C * dvy + w * dBy + B * dwy) * dtdy;
    if (G.omega0 > 0.0) {
        const T Omega0 = (T)G.omega0;
        const T shear = (T)(-1.5 * G.omega0 * G.xc(i));
        sC0 = sC0 + (shear * dAx - T(1.5) * Omega0 * A) * dtdx + shear * dBy * dtdy;
    }
    const T sAL0 = +(ELR - ELL) * half * dtdy;
    const T sAR0 = +(ERR - ERL) * half * dtdy;
    const T sBL0 = -(ERL - ELL) * half * dtdx;
    const T sBR0 = -(ERR - ELR) * half * dtdx;

    T *o = core + core_base(t, kCore2);
    const int cs = kCoreLane;
    if (!chk(o, ((kCore2 - 1) * cs + 1) * sizeof(T))) return;
    o[0 * cs] = r + sr0; o[1 * cs] = u + su0; o[2 * cs] = v + sv0; o[3 * cs] = w + sw0;
    o[4 * cs] = p + sp0; o[5 * cs] = A + sA0; o[6 * cs] = B + sB0; o[7 * cs] = C + sC0;
    o[8 * cs] = drx; o[9 * cs] = dux; o[10 * cs] = dvx; o[11 * cs] = dwx; o[12 * cs] = dpx; o[13 * cs] = dBx; o[14 * cs] = dCx;
    o[15 * cs] = dry; o[16 * cs] = duy; o[17 * cs] = dvy; o[18 * cs] = dwy; o[19 * cs] = dpy; o[20 * cs] = dAy; o[21 * cs] = dCy;
    o[22 * cs] = AL + sAL0; o[23 * cs] = AR + sAR0; o[24 * cs] = BL + sBL0; o[25 * cs] = BR + sBR0;
    o[26 * cs] = dALy; o[27 * cs] = dARy; o[28 * cs] = dBLx; o[29 * cs] = dBRx;
}

// ---------------------------------------------------------------------------
// Riemann fluxes and edge EMFs from the core
// ---------------------------------------------------------------------------
// core field slots, 3D
enum {
    C_R = 0, C_U, C_V, C_W, C_P, C_A, C_B, C_C,
    C_DRX = 8, C_DUX, C_DVX, C_DWX, C_DPX, C_DBX, C_DCX,
    C_DRY = 15, C_DUY, C_DVY, C_DWY, C_DPY, C_DAY, C_DCY,
    C_DRZ = 22, C_DUZ, C_DVZ, C_DWZ, C_DPZ, C_DAZ, C_DBZ,
    C_AL = 29, C_AR, C_BL, C_BR, C_CL, C_CR,
    C_DALY = 35, C_DARY, C_DALZ, C_DARZ, C_DBLX, C_DBRX, C_DBLZ, C_DBRZ, C_DCLX, C_DCRX, C_DCLY, C_DCRY
};
// core field slots, 2D
enum {
    D_R = 0, D_U, D_V, D_W, D_P, D_A, D_B, D_C,
    D_DRX = 8, D_DUX, D_DVX, D_DWX, D_DPX, D_DBX, D_DCX,
    D_DRY = 15, D_DUY, D_DVY, D_DWY, D_DPY, D_DAY, D_DCY,
    D_AL = 22, D_AR, D_BL, D_BR, D_DALY, D_DARY, D_DBLX, D_DBRX
};

// the core in blocks of kCoreLane cells: field f of cell c at core_base(c, nf) + f * kCoreLane,
// so one warp reads one field of 32 consecutive cells as one 128-byte line and all fields of
// a cell sit at small constant offsets from one address
template <typename T>
struct CoreView {
    const T *core;
    int nf;  // fields per cell (kCore3 or kCore2)
    __device__ __forceinline__ T f(int field, long long c) const {
        return ld(core + core_base(c, nf) + field * kCoreLane);
    }
};

// the 15 trace-core fields a cell's face state in direction d on side sgn is built from, in
// the order face_state_v takes them: r u v w p, the 7 slopes of direction d (r u v w p and
// the two transverse field components), the two transverse cell-centred field components,
// and the field on the face itself
__host__ __device__ __forceinline__ void face_fields(int d, int sgn, int ndim, int f[15]) {
    const int base = (d == 0) ? C_DRX : (ndim == 3 ? (d == 1 ? C_DRY : C_DRZ) : D_DRY);
    const int fAL = ndim == 3 ? C_AL : D_AL;
#pragma unroll
    for (int q = 0; q < 5; q++) f[q] = C_R + q;
#pragma unroll
    for (int q = 0; q < 7; q++) f[5 + q] = base + q;
    if (d == 0) { f[12] = C_B; f[13] = C_C; f[14] = sgn > 0 ? fAL + 1 : fAL; }
    else if (d == 1) { f[12] = C_A; f[13] = C_C; f[14] = sgn > 0 ? fAL + 3 : fAL + 2; }
    else { f[12] = C_A; f[13] = C_B; f[14] = sgn > 0 ? C_CR : C_CL; }
}

// face state (uin order r,u,v,w,p,A,B,C) of a cell on its minus (sgn=-1, "qp") or plus
// (sgn=+1, "qm") side in direction d from the values of its face_fields (scheme.f90:1489-1553,
// 1062-1100)
template <typename T>
__device__ __forceinline__ void face_state_v(const T v[15], int d, int sgn, T smallp, T s[8]) {
    const T smallr = T(kSmallr);
    if (sgn > 0) {
        s[IR] = mx(smallr, v[0] + v[5]); s[IU] = v[1] + v[6]; s[IV] = v[2] + v[7]; s[IW] = v[3] + v[8];
        s[IP] = mx(smallp, v[4] + v[9]);
    } else {
        s[IR] = mx(smallr, v[0] - v[5]); s[IU] = v[1] - v[6]; s[IV] = v[2] - v[7]; s[IW] = v[3] - v[8];
        s[IP] = mx(smallp, v[4] - v[9]);
    }
    const T t1 = sgn > 0 ? v[12] + v[10] : v[12] - v[10];
    const T t2 = sgn > 0 ? v[13] + v[11] : v[13] - v[11];
    if (d == 0) { s[IA] = v[14]; s[IB] = t1; s[IC] = t2; }
    else if (d == 1) { s[IA] = t1; s[IB] = v[14]; s[IC] = t2; }
    else { s[IA] = t1; s[IB] = t2; s[IC] = v[14]; }
}

template <typename T>
__device__ __forceinline__ void face_state(const CoreView<T> &cv, long long c, int d, int sgn, int ndim, T smallp,
                                           T s[8]) {
    int f[15];
    face_fields(d, sgn, ndim, f);
    T v[15];
#pragma unroll
    for (int q = 0; q < 15; q++) v[q] = cv.f(f[q], c);
    face_state_v(v, d, sgn, smallp, s);
}

// corner state qXY(c, e) of edge direction e (0 x, 1 y, 2 z); sa/sb = +1/-1 are the
// signs of the first/second transverse directions (R/L and T/B of the reference names:
// RT = (+,+), RB = (+,-), LT = (-,+), LB = (-,-)).  scheme.f90:1555-1697 (3D), 1102-1139 (2D)
template <typename T>
__device__ __forceinline__ void corner_state(const CoreView<T> &cv, long long c, int e, int sa, int sb, int ndim,
                                             T smallp, T s[8]) {
    int b1, b2;
    if (ndim == 2) { b1 = D_DRX; b2 = D_DRY; }
    else if (e == 0) { b1 = C_DRY; b2 = C_DRZ; }
    else if (e == 1) { b1 = C_DRX; b2 = C_DRZ; }
    else { b1 = C_DRX; b2 = C_DRY; }
    T x[5];
#pragma unroll
    for (int n = 0; n < 5; n++) {
        const T d1 = cv.f(b1 + n, c), d2 = cv.f(b2 + n, c);
        const T comb = (sa > 0 ? (sb > 0 ? (+d1 + d2) : (+d1 - d2)) : (sb > 0 ? (-d1 + d2) : (-d1 - d2)));
        x[n] = cv.f(C_R + n, c) + comb;
    }
    s[IR] = mx(T(kSmallr), x[0]); s[IU] = x[1]; s[IV] = x[2]; s[IW] = x[3]; s[IP] = mx(smallp, x[4]);
    if (ndim == 2) {
        // qRT: AR+dARy, BR+dBRx ; qRB: AR-dARy, BL+dBLx ; qLT: AL+dALy, BR-dBRx ; qLB: AL-dALy, BL-dBLx
        const T Af = cv.f(sa > 0 ? D_AR : D_AL, c), dAf = cv.f(sa > 0 ? D_DARY : D_DALY, c);
        const T Bf = cv.f(sb > 0 ? D_BR : D_BL, c), dBf = cv.f(sb > 0 ? D_DBRX : D_DBLX, c);
        s[IA] = Af + (sb > 0 ? +dAf : -dAf);
        s[IB] = Bf + (sa > 0 ? +dBf : -dBf);
        const T C = cv.f(D_C, c), dCx = cv.f(D_DCX, c), dCy = cv.f(D_DCY, c);
        s[IC] = C + (sa > 0 ? (sb > 0 ? (+dCx + dCy) : (+dCx - dCy)) : (sb > 0 ? (-dCx + dCy) : (-dCx - dCy)));
        return;
    }
    if (e == 0) {
        const T A = cv.f(C_A, c), dAy = cv.f(C_DAY, c), dAz = cv.f(C_DAZ, c);
        s[IA] = A + (sa > 0 ? (sb > 0 ? (+dAy + dAz) : (+dAy - dAz)) : (sb > 0 ? (-dAy + dAz) : (-dAy - dAz)));
        const T Bf = cv.f(sa > 0 ? C_BR : C_BL, c), dBf = cv.f(sa > 0 ? C_DBRZ : C_DBLZ, c);
        const T Cf = cv.f(sb > 0 ? C_CR : C_CL, c), dCf = cv.f(sb > 0 ? C_DCRY : C_DCLY, c);
        s[IB] = sb > 0 ? Bf + dBf : Bf - dBf;
        s[IC] = sa > 0 ? Cf + dCf : Cf - dCf;
    } else if (e == 1) {
        const T Af = cv.f(sa > 0 ? C_AR : C_AL, c), dAf = cv.f(sa > 0 ? C_DARZ : C_DALZ, c);
        s[IA] = sb > 0 ? Af + dAf : Af - dAf;
        const T B = cv.f(C_B, c), dBx = cv.f(C_DBX, c), dBz = cv.f(C_DBZ, c);
        s[IB] = B + (sa > 0 ? (sb > 0 ? (+dBx + dBz) : (+dBx - dBz)) : (sb > 0 ? (-dBx + dBz) : (-dBx - dBz)));
        const T Cf = cv.f(sb > 0 ? C_CR : C_CL, c), dCf = cv.f(sb > 0 ? C_DCRX : C_DCLX, c);
        s[IC] = sa > 0 ? Cf + dCf : Cf - dCf;
    } else {
        const T Af = cv.f(sa > 0 ? C_AR : C_AL, c), dAf = cv.f(sa > 0 ? C_DARY : C_DALY, c);
        s[IA] = sb > 0 ? Af + dAf : Af - dAf;
        const T Bf = cv.f(sb > 0 ? C_BR : C_BL, c), dBf = cv.f(sb > 0 ? C_DBRX : C_DBLX, c);
        s[IB] = sa > 0 ? Bf + dBf : Bf - dBf;
        const T C = cv.f(C_C, c), dCx = cv.f(C_DCX, c), dCy = cv.f(C_DCY, c);
        s[IC] = C + (sa > 0 ? (sb > 0 ? (+dCx + dCy) : (+dCx - dCy)) : (sb > 0 ? (-dCx + dCy) : (-dCx - dCy)));
    }
}

// the 1D solver for one interface (solver.f90:163-187); kHLLD: HLLD fixed at compile time, so
// a kernel for the HLLD/HLLD configuration carries no code of the other solvers
template <typename T, bool kHLLD = false>
__device__ __forceinline__ void solve1d(int iriemann, const T *ql, const T *qr, T *f, T &pg, T gamma, T ciso,
                                        int iso, T entho) {
    if constexpr (kHLLD) {
        hlld1d<T>(ql, qr, f, pg, gamma, ciso, iso, entho);
        return;
    }
    switch (iriemann) {
        case DG_RIEMANN_HLLD: hlld1d<T>(ql, qr, f, pg, gamma, ciso, iso, entho); break;
        case DG_RIEMANN_HLL: hll1d<T>(ql, qr, f, gamma, ciso, iso); pg = T(0); break;
        case DG_RIEMANN_LLF: llf1d<T>(ql, qr, f, gamma, ciso, iso); pg = T(0); break;
        default: upwind1d<T>(ql, qr, f, gamma, ciso, iso); pg = T(0); break;
    }
}

// the solver-order interface states of a face from the face states of its two cells (cell
// minus side sm, plus side sp): 0 rho, 1 P, 2 u_n, 3 B_n (face mean), 4 v_t1, 5 B_t1, 6 v_t2,
// 7 B_t2 (solver.f90:116-160)
template <typename T>
__device__ __forceinline__ void face_pair(const T sm[8], const T sp[8], int d, T ql[8], T qr[8]) {
    const T half = T(0.5);
    int ln, lt1, lt2, bn, bt1, bt2;
    if (d == 0) { ln = IU; lt1 = IV; lt2 = IW; bn = IA; bt1 = IB; bt2 = IC; }
    else if (d == 1) { ln = IV; lt1 = IU; lt2 = IW; bn = IB; bt1 = IA; bt2 = IC; }
    else { ln = IW; lt1 = IU; lt2 = IV; bn = IC; bt1 = IA; bt2 = IB; }
    const T bn_mean = half * (sm[bn] + sp[bn]);
    ql[0] = sm[IR]; ql[1] = sm[IP]; ql[2] = sm[ln]; ql[3] = bn_mean; ql[4] = sm[lt1]; ql[5] = sm[bt1]; ql[6] = sm[lt2]; ql[7] = sm[bt2];
    qr[0] = sp[IR]; qr[1] = sp[IP]; qr[2] = sp[ln]; qr[3] = bn_mean; qr[4] = sp[lt1]; qr[5] = sp[bt1]; qr[6] = sp[lt2]; qr[7] = sp[bt2];
}

// solver-order interface states of the face in direction d between cells cl (minus side)
// and cr (plus side)
template <typename T>
__device__ __forceinline__ void face_io(const Geo &G, const CoreView<T> &cv, long long cl, long long cr, int d,
                                        T ql[8], T qr[8]) {
    const T smallp = (T)G.smallp;
    T sm[8], sp[8];
    face_state(cv, cl, d, +1, G.ndim, smallp, sm);
    face_state(cv, cr, d, -1, G.ndim, smallp, sp);
    face_pair(sm, sp, d, ql, qr);
}

// shearing-box upwind terms (solver.f90:199-241) and compflux scaling of solver fluxes f
// (order of ql) and p*_T into the face record (scheme.f90:1740-1753)
template <typename T>
__device__ __forceinline__ void flux_store(const Geo &G, const T *ql, const T *qr, T *f, T pg, int d, int i,
                                           double dtd, T *__restrict__ out, long long fo) {
    const T half = T(0.5), one = T(1);
    const T gamma = (T)G.gamma;
    const T bn_mean = ql[3];
    int ln, lt1, lt2;
    if (d == 0) { ln = IU; lt1 = IV; lt2 = IW; }
    else if (d == 1) { ln = IV; lt1 = IU; lt2 = IW; }
    else { ln = IW; lt1 = IU; lt2 = IV; }
    if (G.ndim == 2) {
        if (G.omega0 > 0.0) {
            double shear = -1.5 * G.omega0 * G.xc(i);
            if (d == 0) shear = -1.5 * G.omega0 * (G.xc(i) + G.xc(i - 1));
            if (d == 1) shear = -1.5 * G.omega0 * G.xc(i);
            f[7] = f[7] + (T)shear * bn_mean;
        }
    } else if ((G.omega0 > 0.0) && (d == 1) && !G.fargo) {
        const T shear = (T)(-1.5 * G.omega0 * G.xc(i));
        const T *qs = (shear > T(0)) ? ql : qr;
        const T rs = qs[0], ps = qs[1], us = qs[2], as = qs[3], vs = qs[4], bs = qs[5], ws = qs[6], cs = qs[7];
        const T Emag = half * (as * as + bs * bs + cs * cs);
        const T Ekin = half * (us * us + vs * vs + ws * ws);
        const T Etot = Ekin + Emag + ps / (gamma - one);
        f[0] = f[0] + shear * rs;
        f[1] = f[1] + shear * (Etot + Emag - bn_mean * bn_mean);
        f[2] = f[2] + shear * rs * us;
        f[4] = f[4] + shear * rs * vs;
        f[6] = f[6] + shear * rs * ws;
    }
    // compflux: flux = fgodunov*ds*dt, reordered to uin variables
    double dsd;
    if (d == 0) dsd = G.dy * G.dz; else if (d == 1) dsd = G.dx * G.dz; else dsd = G.dx * G.dy;
    const T ds = (T)dsd, dt = (T)dtd;
    T o[8];
    o[0] = f[0] * ds * dt;                       // rho
    o[1] = f[1] * ds * dt;                       // E
    o[2 + ln - IU] = f[2] * ds * dt;             // normal momentum
    o[2 + lt1 - IU] = f[4] * ds * dt;            // first tangential momentum
    o[2 + lt2 - IU] = f[6] * ds * dt;            // second tangential momentum
    o[5] = pg;                                   // p*_T (zero unless HLLD)
    if (G.ndim == 3) {
        store6(out + fo * kFluxRec3, o);
    } else {
        o[6] = f[7] * ds * dt;  // B_t2 = B_z
        o[7] = T(0);
        store8(out + fo * kFluxRec2, o);
    }
}

// one face flux in direction d between cells cl (minus side) and cr (plus side);
// writes the compflux-scaled fluxes in uin order plus p*_T (solver.f90:116-262, scheme.f90:1740-1753)
template <typename T, bool kHLLD = false>
__device__ void face_flux(const Geo &G, const CoreView<T> &cv, long long cl, long long cr, int d, int i, double dtd,
                          T *__restrict__ out, long long fo) {
    T ql[8], qr[8];
    face_io(G, cv, cl, cr, d, ql, qr);
    T f[8], pg = T(0);
    solve1d<T, kHLLD>(G.iriemann, ql, qr, f, pg, (T)G.gamma, (T)G.ciso, G.iso, (T)G.entho);
    flux_store(G, ql, qr, f, pg, d, i, dtd, out, fo);
}

// one edge EMF (riemann_solver_magnetic, solver_magnetic.f90:79-230); e = edge direction
template <typename T, bool kHLLD = false>
__device__ T edge_emf(const Geo &G, const CoreView<T> &cv, long long cLL, long long cRL, long long cLR, long long cRR,
                      int e, int i, double dtd) {
    const T half = T(0.5);
    const T smallp = (T)G.smallp;
    T sLL[8], sRL[8], sLR[8], sRR[8];
    int lt1, lt2, bn, bt1, bt2;
    if (e == 0) {
        // qLL <- qRT(i,j-1,k-1), qRL <- qLT(i,j,k-1), qLR <- qRB(i,j-1,k), qRR <- qLB(i,j,k)
        corner_state(cv, cLL, 0, +1, +1, G.ndim, smallp, sLL);
        corner_state(cv, cRL, 0, -1, +1, G.ndim, smallp, sRL);
        corner_state(cv, cLR, 0, +1, -1, G.ndim, smallp, sLR);
        corner_state(cv, cRR, 0, -1, -1, G.ndim, smallp, sRR);
        lt1 = IV; lt2 = IW; bn = IA; bt1 = IB; bt2 = IC;
    } else if (e == 1) {
        // call site passes (qRT, qLT, qRB, qLB): qLL <- qRT(i-1,j,k-1), qRL <- qRB(i-1,j,k),
        // qLR <- qLT(i,j,k-1), qRR <- qLB(i,j,k)
        corner_state(cv, cLL, 1, +1, +1, G.ndim, smallp, sLL);
        corner_state(cv, cRL, 1, +1, -1, G.ndim, smallp, sRL);
        corner_state(cv, cLR, 1, -1, +1, G.ndim, smallp, sLR);
        corner_state(cv, cRR, 1, -1, -1, G.ndim, smallp, sRR);
        lt1 = IW; lt2 = IU; bn = IB; bt1 = IC; bt2 = IA;
    } else {
        // qLL <- qRT(i-1,j-1,k), qRL <- qLT(i,j-1,k), qLR <- qRB(i-1,j,k), qRR <- qLB(i,j,k)
        corner_state(cv, cLL, 2, +1, +1, G.ndim, smallp, sLL);
        corner_state(cv, cRL, 2, -1, +1, G.ndim, smallp, sRL);
        corner_state(cv, cLR, 2, +1, -1, G.ndim, smallp, sLR);
        corner_state(cv, cRR, 2, -1, -1, G.ndim, smallp, sRR);
        lt1 = IU; lt2 = IV; bn = IC; bt1 = IA; bt2 = IB;
    }
    T qLL[8], qRL[8], qLR[8], qRR[8];
    qLL[0] = sLL[IR]; qRL[0] = sRL[IR]; qLR[0] = sLR[IR]; qRR[0] = sRR[IR];
    if (G.iso) {
        const T c2 = (T)(G.ciso * G.ciso);
        qLL[1] = qLL[0] * c2; qRL[1] = qRL[0] * c2; qLR[1] = qLR[0] * c2; qRR[1] = qRR[0] * c2;
    } else {
        qLL[1] = sLL[IP]; qRL[1] = sRL[IP]; qLR[1] = sLR[IP]; qRR[1] = sRR[IP];
    }
    qLL[2] = sLL[lt1]; qRL[2] = sRL[lt1]; qLR[2] = sLR[lt1]; qRR[2] = sRR[lt1];
    qLL[3] = sLL[lt2]; qRL[3] = sRL[lt2]; qLR[3] = sLR[lt2]; qRR[3] = sRR[lt2];
    qLL[4] = half * (sLL[bt1] + sRL[bt1]);
    qRL[4] = half * (sLL[bt1] + sRL[bt1]);
    qLR[4] = half * (sLR[bt1] + sRR[bt1]);
    qRR[4] = half * (sLR[bt1] + sRR[bt1]);
    qLL[5] = half * (sLL[bt2] + sLR[bt2]);
    qRL[5] = half * (sRL[bt2] + sRR[bt2]);
    qLR[5] = half * (sLL[bt2] + sLR[bt2]);
    qRR[5] = half * (sRL[bt2] + sRR[bt2]);
    qLL[6] = sLL[bn]; qRL[6] = sRL[bn]; qLR[6] = sLR[bn]; qRR[6] = sRR[bn];
    qLL[7] = qLL[2] * qLL[5] - qLL[3] * qLL[4];
    qRL[7] = qRL[2] * qRL[5] - qRL[3] * qRL[4];
    qLR[7] = qLR[2] * qLR[5] - qLR[3] * qLR[4];
    qRR[7] = qRR[2] * qRR[5] - qRR[3] * qRR[4];
    Corners<T> c;
    c.rLL = qLL[0]; c.uLL = qLL[2]; c.ALL = qLL[4]; c.CLL = qLL[6];
    c.rRL = qRL[0]; c.uRL = qRL[2]; c.ARL = qRL[4]; c.CRL = qRL[6];
    c.rLR = qLR[0]; c.uLR = qLR[2]; c.ALR = qLR[4]; c.CLR = qLR[6];
    c.rRR = qRR[0]; c.uRR = qRR[2]; c.ARR = qRR[4]; c.CRR = qRR[6];
    c.pLL = qLL[1]; c.vLL = qLL[3]; c.BLL = qLL[5]; c.ELL = qLL[7];
    c.pRL = qRL[1]; c.vRL = qRL[3]; c.BRL = qRL[5]; c.ERL = qRL[7];
    c.pLR = qLR[1]; c.vLR = qLR[3]; c.BLR = qLR[5]; c.ELR = qLR[7];
    c.pRR = qRR[1]; c.vRR = qRR[3]; c.BRR = qRR[5]; c.ERR = qRR[7];
    const T dt = (T)dtd, gamma = (T)G.gamma;
    T emf;
    if constexpr (kHLLD) emf = hlld2d<T>(c, dt, gamma);
    else switch (G.iriemann2d) {
        case DG_RIEMANN_HLLD: emf = hlld2d<T>(c, dt, gamma); break;
        case DG_RIEMANN_LLF: emf = llf2d<T>(c, dt, gamma, (T)G.ciso, G.iso); break;
        case DG_RIEMANN_HLLA: emf = hlla2d<T>(c, dt); break;
        default: emf = upwind2d<T>(c, dt); break;
    }
    if ((G.omega0 > 0.0) && !G.fargo) {
        if (e == 0) {
            const T shear = (T)(-1.5 * G.omega0 * G.xc(i));
            if (shear > T(0)) emf = emf + shear * c.BLL * dt;
            else emf = emf + shear * c.BRR * dt;
        } else if (e == 2) {
            const T shear = (T)(-1.5 * G.omega0 * 0.5 * (G.xc(i) + G.xc(i - 1)));
            if (shear > T(0)) emf = emf - shear * c.ALL * dt;
            else emf = emf - shear * c.ARR * dt;
        }
    }
    return emf;
}

template <typename T, bool kHLLD>
__global__ void __launch_bounds__(kThreads, (sizeof(T) == 8 ? DG_RIEMANN_MINB64 : DG_RIEMANN_MINB32)) k_riemann3d(Geo G, const T *__restrict__ core, T *__restrict__ fx,
                                                           T *__restrict__ fy, T *__restrict__ fz, T *__restrict__ ex,
                                                           T *__restrict__ ey, T *__restrict__ ez, const Scalars *S,
                                                           int faces) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    int i, j, k;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    const double dt = S->dt;
    const CoreView<T> cv{core, kCore3};
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const long long c = G.cidx(i, j, k);
    if (faces) {  // faces = 0: the face fluxes come from the learned flux and its HLLD fallback list
        if (j <= ny && k <= nz) face_flux<T, kHLLD>(G, cv, G.cidx(i - 1, j, k), c, 0, i, dt, fx, t);
        if (i <= nx && k <= nz) face_flux<T, kHLLD>(G, cv, G.cidx(i, j - 1, k), c, 1, i, dt, fy, t);
        if (i <= nx && j <= ny) face_flux<T, kHLLD>(G, cv, G.cidx(i, j, k - 1), c, 2, i, dt, fz, t);
    }
    if (k <= nz)
        ez[t] = edge_emf<T, kHLLD>(G, cv, G.cidx(i - 1, j - 1, k), G.cidx(i, j - 1, k), G.cidx(i - 1, j, k), c, 2, i, dt);
    if (j <= ny)
        ey[t] = edge_emf<T, kHLLD>(G, cv, G.cidx(i - 1, j, k - 1), G.cidx(i - 1, j, k), G.cidx(i, j, k - 1), c, 1, i, dt);
    if (i <= nx)
        ex[t] = edge_emf<T, kHLLD>(G, cv, G.cidx(i, j - 1, k - 1), G.cidx(i, j, k - 1), G.cidx(i, j - 1, k), c, 0, i, dt);
}

// The same work split in two passes over the face index space: the face fluxes (1D solves)
// and the edge EMFs (2D solves), each compiled for its own register budget.  A thread
// holds the live values of one kind of solve only, so more warps fit an SM; the trace core
// is read twice (once per pass).  Every solve is the same function of the same core values
// as in k_riemann3d, so the results are identical.
#ifndef DG_RFACE_MINB64
#define DG_RFACE_MINB64 4
#endif
#ifndef DG_REDGE_MINB64
#define DG_REDGE_MINB64 4
#endif
#ifndef DG_RFACE_MINB32
#define DG_RFACE_MINB32 8
#endif
#ifndef DG_REDGE_MINB32
#define DG_REDGE_MINB32 8
#endif
// kDir: the one direction this launch solves (0, 1, 2), or -1 for all three
template <typename T, bool kHLLD, int kDir = -1>
__global__ void __launch_bounds__(kThreads, (sizeof(T) == 8 ? DG_RFACE_MINB64 : DG_RFACE_MINB32))
k_faces3d(Geo G, const T *__restrict__ core, T *__restrict__ fx, T *__restrict__ fy, T *__restrict__ fz,
          const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    int i, j, k;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    const double dt = S->dt;
    const CoreView<T> cv{core, kCore3};
    const long long c = G.cidx(i, j, k);
    if ((kDir < 0 || kDir == 0) && j <= G.ny && k <= G.nz) face_flux<T, kHLLD>(G, cv, G.cidx(i - 1, j, k), c, 0, i, dt, fx, t);
    if ((kDir < 0 || kDir == 1) && i <= G.nx && k <= G.nz) face_flux<T, kHLLD>(G, cv, G.cidx(i, j - 1, k), c, 1, i, dt, fy, t);
    if ((kDir < 0 || kDir == 2) && i <= G.nx && j <= G.ny) face_flux<T, kHLLD>(G, cv, G.cidx(i, j, k - 1), c, 2, i, dt, fz, t);
}

template <typename T, bool kHLLD, int kDir = -1>
__global__ void __launch_bounds__(kThreads, (sizeof(T) == 8 ? DG_REDGE_MINB64 : DG_REDGE_MINB32))
k_edges3d(Geo G, const T *__restrict__ core, T *__restrict__ ex, T *__restrict__ ey, T *__restrict__ ez,
          const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    int i, j, k;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    const double dt = S->dt;
    const CoreView<T> cv{core, kCore3};
    const long long c = G.cidx(i, j, k);
    if ((kDir < 0 || kDir == 2) && k <= G.nz)
        ez[t] = edge_emf<T, kHLLD>(G, cv, G.cidx(i - 1, j - 1, k), G.cidx(i, j - 1, k), G.cidx(i - 1, j, k), c, 2, i, dt);
    if ((kDir < 0 || kDir == 1) && j <= G.ny)
        ey[t] = edge_emf<T, kHLLD>(G, cv, G.cidx(i - 1, j, k - 1), G.cidx(i - 1, j, k), G.cidx(i, j, k - 1), c, 1, i, dt);
    if ((kDir < 0 || kDir == 0) && i <= G.nx)
        ex[t] = edge_emf<T, kHLLD>(G, cv, G.cidx(i, j - 1, k - 1), G.cidx(i, j, k - 1), G.cidx(i, j - 1, k), c, 0, i, dt);
}

// ---------------------------------------------------------------------------
// NDIM = 1: slope, trace1d, riemann_solver and update along x only (scheme.f90:289-316,
// 661-805; solver.f90:116-262; scheme.f90:1764-1936).  The core of a cell is its predicted
// state (8: rho, u, v, w, P, B_x cell-centred and unchanged, B_y, B_z) and its 7 half slopes
// (rho, u, v, w, P, B_y, B_z), at core index i (cells 0 .. nx+1).
// ---------------------------------------------------------------------------
constexpr int kCore1 = 15;
template <typename T>
__global__ void __launch_bounds__(kThreads) k_trace1d(Geo G, const T *__restrict__ Q, T *__restrict__ core,
                                                      const Scalars *S) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.CX) return;
    const int i = (int)t;
    const long long c = G.idx(i, 1, 1);
    const double dtd = S->dt;
    const T half = T(0.5), gamma = (T)G.gamma, dtdx = (T)(dtd / G.dx);
    const T st = (T)G.slope_type;  // 1 or 2 (dg_init refuses 3 with ndim = 1)
    T qv[8], d[8];
#pragma unroll
    for (int v = 0; v < 8; v++) {
        qv[v] = ld(Q + G.sv * v + c);
        d[v] = G.slope_type == 0 ? T(0) : limit1(st, ld(Q + G.sv * v + c - 1), qv[v], ld(Q + G.sv * v + c + 1));
    }
    const T r = qv[IR], u = qv[IU], v = qv[IV], w = qv[IW], p = qv[IP], A = qv[IA], B = qv[IB], C = qv[IC];
    const T drx = half * d[IR], dux = half * d[IU], dvx = half * d[IV], dwx = half * d[IW], dpx = half * d[IP];
    const T dBx = half * d[IB], dCx = half * d[IC];
    // source terms, scheme.f90:717-727 (the rotation term of :777-781 changes only the local
    // sC0 after its last use)
    T sr0 = -u * drx - r * dux;                   sr0 = sr0 * dtdx;
    T su0 = -u * dux - (dpx + B * dBx + C * dCx) / r; su0 = su0 * dtdx;
    T sv0 = -u * dvx + (A * dBx) / r;              sv0 = sv0 * dtdx;
    T sw0 = -u * dwx + (A * dCx) / r;              sw0 = sw0 * dtdx;
    T sp0 = -u * dpx - gamma * p * dux;            sp0 = sp0 * dtdx;
    T sB0 = -u * dBx + A * dvx - B * dux;          sB0 = sB0 * dtdx;
    T sC0 = -u * dCx + A * dwx - C * dux;          sC0 = sC0 * dtdx;
    T *o = core + core_base(t, kCore1);
    const int cs = kCoreLane;
    if (!chk(o, ((kCore1 - 1) * cs + 1) * sizeof(T))) return;
    o[0 * cs] = r + sr0; o[1 * cs] = u + su0; o[2 * cs] = v + sv0; o[3 * cs] = w + sw0;
    o[4 * cs] = p + sp0; o[5 * cs] = A;       o[6 * cs] = B + sB0; o[7 * cs] = C + sC0;
    o[8 * cs] = drx; o[9 * cs] = dux; o[10 * cs] = dvx; o[11 * cs] = dwx; o[12 * cs] = dpx;
    o[13 * cs] = dBx; o[14 * cs] = dCx;
}

// the x faces i = 1 .. nx+1: qm of cell i-1 (state + slope) against qp of cell i (state - slope),
// the density floored, the pressure not (trace1d, scheme.f90:783-801); record per face: the
// compflux-scaled fluxes of rho, E, rho u, rho v, rho w, then p*_T, then those of B_x, B_y, B_z
template <typename T, bool kHLLD>
__global__ void __launch_bounds__(kThreads) k_riemann1d(Geo G, const T *__restrict__ core, T *__restrict__ fx,
                                                        const Scalars *S) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.FX) return;
    const int i = (int)t + 1;
    const T half = T(0.5), smallr = T(kSmallr);
    auto side = [&](long long cc, int sgn, T s[8]) {
        const CoreView<T> cv{core, kCore1};
        const T pr = cv.f(0, cc), pu = cv.f(1, cc), pv = cv.f(2, cc), pw = cv.f(3, cc), pp = cv.f(4, cc);
        const T pA = cv.f(5, cc), pB = cv.f(6, cc), pC = cv.f(7, cc);
        const T dr = cv.f(8, cc), du = cv.f(9, cc), dv = cv.f(10, cc), dw = cv.f(11, cc), dp = cv.f(12, cc);
        const T dB = cv.f(13, cc), dC = cv.f(14, cc);
        if (sgn > 0) {
            s[IR] = mx(smallr, pr + dr); s[IU] = pu + du; s[IV] = pv + dv; s[IW] = pw + dw; s[IP] = pp + dp;
            s[IA] = pA; s[IB] = pB + dB; s[IC] = pC + dC;
        } else {
            s[IR] = mx(smallr, pr - dr); s[IU] = pu - du; s[IV] = pv - dv; s[IW] = pw - dw; s[IP] = pp - dp;
            s[IA] = pA; s[IB] = pB - dB; s[IC] = pC - dC;
        }
    };
    T sm[8], sp[8];
    side(i - 1, +1, sm);
    side(i, -1, sp);
    const T bn_mean = half * (sm[IA] + sp[IA]);
    T ql[8] = {sm[IR], sm[IP], sm[IU], bn_mean, sm[IV], sm[IB], sm[IW], sm[IC]};
    T qr[8] = {sp[IR], sp[IP], sp[IU], bn_mean, sp[IV], sp[IB], sp[IW], sp[IC]};
    T f[8], pg = T(0);
    solve1d<T, kHLLD>(G.iriemann, ql, qr, f, pg, (T)G.gamma, (T)G.ciso, G.iso, (T)G.entho);
    if (G.omega0 > 0.0) {  // solver.f90:201-207
        const T shear = (T)(-1.5 * G.omega0 * (G.xc(i) + G.xc(i - 1)));
        f[7] = f[7] + shear * bn_mean;
    }
    // compflux, scheme.f90:1740-1753: ds = dy dz
    const T ds = (T)(G.dy * G.dz), dt = (T)S->dt;
    T *o = fx + t * kFluxRec1;
    if (!chk(o, kFluxRec1 * sizeof(T))) return;
    o[0] = f[0] * ds * dt; o[1] = f[1] * ds * dt; o[2] = f[2] * ds * dt; o[3] = f[4] * ds * dt;
    o[4] = f[6] * ds * dt; o[5] = pg; o[6] = f[3] * ds * dt; o[7] = f[5] * ds * dt; o[8] = f[7] * ds * dt;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_riemann2d(Geo G, const T *__restrict__ core, T *__restrict__ fx,
                                                        T *__restrict__ fy, T *__restrict__ ez, const Scalars *S,
                                                        int faces) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    const int j = (int)fdiv((unsigned)t, G.dFX) + 1;
    const int i = (int)((unsigned)t - (unsigned)(j - 1) * G.dFX.d) + 1;
    const double dt = S->dt;
    const CoreView<T> cv{core, kCore2};
    const long long c = G.cidx(i, j, 1);
    if (faces && j <= G.ny) face_flux(G, cv, G.cidx(i - 1, j, 1), c, 0, i, dt, fx, t);
    if (faces && i <= G.nx) face_flux(G, cv, G.cidx(i, j - 1, 1), c, 1, i, dt, fy, t);
    ez[t] = edge_emf(G, cv, G.cidx(i - 1, j - 1, 1), G.cidx(i, j - 1, 1), G.cidx(i - 1, j, 1), c, 2, i, dt);
}

// ---------------------------------------------------------------------------
// update + constrained transport
// ---------------------------------------------------------------------------
struct ShearRemap {
    double epsi;
    int jp;
};
// shear offset of the x boundaries at time itime (shearingbox.f90:34-37)
__device__ __forceinline__ ShearRemap shear_offset(const Geo &G, double itime) {
    double deltay = 1.5 * G.omega0 * (G.xmax - G.xmin) * itime;
    deltay = fmod(deltay, (G.ymax - G.ymin));
    ShearRemap s;
    s.epsi = fmod(deltay, G.dy);
    s.jp = (int)(deltay / G.dy);
    return s;
}

// Any y index into [1, n].  Equal to the reference's single "+/- ny" wrap whenever
// that wrap lands inside the active range; the reference reads a ghost row or
// unallocated memory otherwise (a shift of a full box or more), which this guard
// keeps inside the array.
__device__ __forceinline__ int wrap1(int j, int n) {
    if (j >= 1 && j <= n) return j;
    int m = (j - 1) % n;
    return (m < 0 ? m + n : m) + 1;
}

// shear offset at time + frac*dt, computed once per step phase instead of per thread
__global__ void k_shear_offset(Geo G, Scalars *S, double frac) {
    const ShearRemap r = shear_offset(G, S->time + frac * S->dt);
    S->sh_jp = r.jp;
    S->sh_epsi = r.epsi;
}

// shearing_flux / shearing_emf average of a face quantity on the inner (side 0)
// or outer (side 1) x boundary (shearingbox.f90:250-280, 339-380)
template <typename T>
__device__ __forceinline__ T shear_avg(const Geo &G, const ShearRemap &sr, const T *a, int stride, int side, int j,
                                       int k) {
    auto at = [&](int ii, int jj) { return ld(a + G.fidx(ii, jj, k) * stride); };
    const int ny = G.ny;
    const T one = T(1), half = T(0.5);
    if (side == 0) {
        int jremap = j - sr.jp - 1, jremapp = jremap + 1;
        if (jremap <= 0) jremap = jremap + ny;
        if (jremapp <= 0) jremapp = jremapp + ny;
        jremap = wrap1(jremap, ny);
        jremapp = wrap1(jremapp, ny);
        const T eps = (T)(1.0 - sr.epsi / G.dy);
        T v = at(1, j) + (one - eps) * at(G.nx + 1, jremap) + eps * at(G.nx + 1, jremapp);
        return half * v;
    } else {
        int jremap = j + sr.jp, jremapp = jremap + 1;
        if (jremap > ny) jremap = jremap - ny;
        if (jremapp > ny) jremapp = jremapp - ny;
        jremap = wrap1(jremap, ny);
        jremapp = wrap1(jremapp, ny);
        const T eps = (T)(sr.epsi / G.dy);
        T v = at(G.nx + 1, j) + (one - eps) * at(1, jremap) + eps * at(1, jremapp);
        return half * v;
    }
}

// ---------------------------------------------------------------------------
// boundary: every ghost value written from active values in one pass
// ---------------------------------------------------------------------------
__device__ __forceinline__ int map_bc(int type, int i, int n) {
    if (i >= 1 && i <= n) return i;
    if (type == DG_BC_ZERO_GRADIENT) return i < 1 ? 1 : n;
    // periodic (and y/z of the shearing box)
    return i < 1 ? i + n : i - n;
}

// number of ghost cells: the z-ghost planes, the y-ghost rows of the active planes and
// the x-ghost cells of the active rows
__host__ __device__ __forceinline__ long long ghost_cells(const Geo &G) {
    const long long nA = (G.ndim == 3) ? 6LL * G.NX * G.NY : 0;
    const long long nB = (G.ndim > 1) ? 6LL * G.NX * (G.ndim == 3 ? G.nz : 1) : 0;
    const long long nC = 6LL * G.ny * (G.ndim == 3 ? G.nz : 1);
    return nA + nB + nC;
}

constexpr int kMaxVars = 10;  // stored state variables: 8, plus the frozen right-face B (z in 2D, y and z in 1D)
template <class Store>
__global__ void __launch_bounds__(kThreads) k_boundary(Geo G, Store U, int nv, const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= ghost_cells(G)) return;
    // the ghost counts of any grid that fits a GPU are far below 2^32: 32-bit index arithmetic
    const unsigned NX = G.NX, NY = G.NY;
    const unsigned nA = (G.ndim == 3) ? 6u * NX * NY : 0u;
    const unsigned nB = (G.ndim > 1) ? 6u * NX * (G.ndim == 3 ? (unsigned)G.nz : 1u) : 0u;
    auto ghost = [](int g, int n) { return g < 3 ? g - 2 : n + g - 2; };  // 0..5 -> -2,-1,0,n+1,n+2,n+3
    int i, j, k;
    const unsigned u0 = (unsigned)t;
    if (u0 < nA) {
        i = (int)(u0 % NX) - 2;
        const unsigned r = u0 / NX;
        j = (int)(r % NY) - 2;
        k = ghost((int)(r / NY), G.nz);
        // a z slab's ghost planes on a neighbour's side come from its halo (dg_halo_unpack)
        if ((k < 1 ? G.bcz_lo : G.bcz_hi) == kBcHalo) return;
    } else if (u0 - nA < nB) {
        const unsigned u = u0 - nA;
        i = (int)(u % NX) - 2;
        const unsigned r = u / NX;
        j = ghost((int)(r % 6u), G.ny);
        k = (G.ndim == 3) ? (int)(r / 6u) + 1 : 1;
    } else {
        const unsigned u = u0 - nA - nB;
        i = ghost((int)(u % 6u), G.nx);
        const unsigned r = u / 6u;
        j = (int)(r % (unsigned)G.ny) + 1;
        k = (G.ndim == 3) ? (int)(r / (unsigned)G.ny) + 1 : 1;
    }
    const bool gx = (i < 1 || i > G.nx);
    const int jj = (G.ndim > 1) ? map_bc(G.bc[1], j, G.ny) : 1;
    const int kk = (G.ndim == 3) ? map_bc(k < 1 ? G.bcz_lo : G.bcz_hi, k, G.nz) : 1;
    const long long c = G.idx(i, j, k);
    // every value is read (from active cells, or the outer x face that no thread writes)
    // before the first store, so the loads of all variables are in flight together
    double out[kMaxVars];
    if (!gx || G.bc[0] != DG_BC_SHEARINGBOX) {
        const long long src = G.idx(map_bc(G.bc[0], i, G.nx), jj, kk);
#pragma unroll
        for (int v = 0; v < kMaxVars; v++)
            if (v < nv) out[v] = U.get(G, v, src);
#pragma unroll
        for (int v = 0; v < kMaxVars; v++)
            if (v < nv) U.set(G, v, c, out[v]);
        return;
    }
    // shear-periodic x ghost (only with ndim = 3; shearingbox.f90:62-147): the remapped rows,
    // eps and lambda are the same for every variable; offset for time+dt from k_shear_offset
    const ShearRemap sr{S->sh_epsi, S->sh_jp};
    const int nx = G.nx, ny = G.ny;
    const double one = 1.0, half = 0.5;
    const bool lower = i < 1;
    const int src = lower ? nx + i : i - nx;  // outer(1:3) = uin(nx-2:nx) / inner(1:3) = uin(1:3)
    int jr, jrp;
    double eps;
    if (lower) {
        jr = jj - sr.jp - 1;
        jrp = jr + 1;
        if (jr <= 0) jr = jr + ny;
        if (jrp <= 0) jrp = jrp + ny;
        eps = one - sr.epsi / G.dy;
    } else {
        jr = jj + sr.jp;
        jrp = jr + 1;
        if (jr > ny) jr = jr - ny;
        if (jrp > ny) jrp = jrp - ny;
        eps = sr.epsi / G.dy;
    }
    const double lambda = half * eps * (eps - one);
    const int st = mn(G.slope_type, 2);
    auto row = [&](int r) { return G.idx(src, map_bc(G.bc[1], r, ny), kk); };
    // rows of the two values and of shearing_slope at each (shearingbox.f90:415-430, 493-499)
    const long long cm = row(jr - 1), c0 = row(jr), cp = row(jr + 1);
    const long long dm = row(jrp - 1), d0 = row(jrp), dp = row(jrp + 1);
    // the outer face keeps its own (CT-updated) value; ghost j/k copy it
    const bool outer = (i == nx + 1);
    const bool keep_a = outer && jj == j && kk == k;
    const long long ca = G.idx(i, jj, kk);
#pragma unroll
    for (int v = 0; v < kMaxVars; v++) {
        if (v >= nv) continue;
        if (v == IA && outer) {
            out[v] = U.get(G, v, ca);
        } else if (v == IB) {  // By: one-sided slope
            const double a0 = U.get(G, v, c0), a1 = U.get(G, v, cp);
            out[v] = a0 + eps * (st == 0 ? 0.0 : a1 - a0);
        } else {
            const double am = U.get(G, v, cm), a0 = U.get(G, v, c0), ap = U.get(G, v, cp);
            const double bm = U.get(G, v, dm), b0 = U.get(G, v, d0), bp = U.get(G, v, dp);
            const double sa = st == 0 ? 0.0 : limit1<double>((double)st, am, a0, ap);
            const double sb = st == 0 ? 0.0 : limit1<double>((double)st, bm, b0, bp);
            out[v] = (one - eps) * a0 + eps * b0 + lambda * (lower ? sa - sb : sb - sa);
        }
    }
#pragma unroll
    for (int v = 0; v < kMaxVars; v++)
        if (v < nv && !(v == IA && keep_a)) U.set(G, v, c, out[v]);
}

// right-face B (uin vars 9-11) of the reference layout, from the stored left faces
template <class Store>
__global__ void k_right_faces(Geo G, Store U, double *__restrict__ out) {
    const long long n = (long long)G.NX * G.NY * G.NZ;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % G.NX);
    const long long r = t / G.NX;
    const int j = (int)(r % G.NY);
    const int k = (int)(r / G.NY);
    // last layer of each direction: no neighbour, keep the left-face value
    out[t] = (i + 1 < G.NX) ? U.get(G, IA, t + 1) : U.get(G, IA, t);
    // ndim = 1: the right y and z faces are never refreshed by the reference (stored planes 8, 9);
    // ndim = 2: the right z face (plane 8)
    if (G.ndim == 1) out[n + t] = U.get(G, 8, t);
    else out[n + t] = (j + 1 < G.NY) ? U.get(G, IB, t + G.sy) : U.get(G, IB, t);
    if (G.ndim == 3) out[2 * n + t] = (k + 1 < G.NZ) ? U.get(G, IC, t + G.sz) : U.get(G, IC, t);
    else out[2 * n + t] = U.get(G, G.ndim == 1 ? 9 : 8, t);
}

// state <-> FP64 planes (upload/download of the compensated state)
template <class Store>
__global__ void k_state_to_f64(Geo G, Store U, int nv, double *__restrict__ out) {
    const long long n = G.sv * nv;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    out[t] = U.get(G, (int)(t / G.sv), t % G.sv);
}
template <class Store>
__global__ void k_f64_to_state(Geo G, const double *__restrict__ in, int nv, Store U) {
    const long long n = G.sv * nv;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    U.set(G, (int)(t / G.sv), t % G.sv, in[t]);
}

// ---------------------------------------------------------------------------
// FARGO, fargo.f90:17-288, FP64 (the FP32 path remaps with FP32 increments instead)
// ---------------------------------------------------------------------------
struct FargoShift {
    double vK, eps;
    int nshft;
};
__device__ __forceinline__ FargoShift fargo_shift(const Geo &G, double xpos, double dt) {
    FargoShift f;
    f.vK = -1.5 * G.omega0 * xpos;
    // whole cells of the shift; a shift of a box length or more (a step far beyond the CFL
    // limit, or a non-finite dt) is held at ny, so the loops over the shifted cells stay bounded
    const double cells = fabs(f.vK * dt) / G.dy;
    f.nshft = cells < (double)G.ny ? (int)cells : G.ny;
    f.eps = fmod(fabs(f.vK * dt), G.dy);
    f.eps = f.eps / G.dy;
    return f;
}

// uin_slope of variable v at (i, j, k) with y wrap (fargo.f90:266-280)
template <class Store>
__device__ __forceinline__ double fslope(const Geo &G, const Store &U, int v, int i, int j, int k) {
    const int st = mn(G.slope_type, 2);
    if (st == 0) return 0.0;
    auto val = [&](int jj) { return U.getr(G, v, G.idx(i, map_bc(G.bc[1], jj, G.ny), k)); };
    return limit1<double>((double)st, val(j - 1), val(j), val(j + 1));
}

// FARGO line layout: one thread per (i, k) face column and per segment of kFargoSeg faces
// along y; consecutive threads take consecutive i (coalesced), and a thread slides a
// window of source values along its segment so each source value is read once
#ifndef DG_FARGO_SEG
#define DG_FARGO_SEG 16
#endif
constexpr int kFargoSeg = DG_FARGO_SEG;
constexpr int kFargoChunk = 4;  // rows of the CT part whose loads are issued together
__host__ __device__ __forceinline__ long long fargo_line_threads(const Geo &G) {
    return (long long)G.FX * G.FZ * ((G.FY + kFargoSeg - 1) / kFargoSeg);
}
struct FargoLine {
    int i, k, jb, je;  // face column and the segment [jb, je] of y faces
};
__device__ __forceinline__ bool fargo_line(const Geo &G, long long t, FargoLine &L) {
    const int nseg = (G.FY + kFargoSeg - 1) / kFargoSeg;
    if (t >= 2147483647LL) return false;
    int sg;
    split3((unsigned)t, G.dFX, G.dFZ, L.i, L.k, sg);
    L.i++; L.k++;
    if (sg >= nseg) return false;
    L.jb = (int)sg * kFargoSeg + 1;
    L.je = mn(L.jb + kFargoSeg - 1, G.FY);
    return true;
}
// donor row js of row j for the column's shift, fargo.f90:63-77
__device__ __forceinline__ int fargo_src(const FargoShift &f, int j, int ny) {
    int js;
    if (f.vK > 0.0) {
        js = j - f.nshft - 1;
        if (js < 1) js = js + ny;
    } else {
        js = j + f.nshft;
        if (js > ny) js = js - ny;
    }
    return wrap1(js, ny);
}
__device__ __forceinline__ int next_row(int j, int ny) { return j + 1 > ny ? j + 1 - ny : j + 1; }
// The z plane that FARGO's EMFs read for face plane k (1..nz+1).  The reference refreshes the
// z ghosts first (fargo.f90:36-49), so plane nz+1 holds its boundary copy: plane 1 when
// periodic, plane nz when zero-gradient.  In a z slab the reference exchanges that plane with
// the upper neighbour (boundary_z); the top face plane this slab's godunov updated holds the
// same values (its EMFs come from the neighbour's halo cells), so the slab reads it directly.
__device__ __forceinline__ int fargo_zplane(const Geo &G, int k) {
    if (k > G.nz && G.bcz_hi == kBcHalo) return k;
    return map_bc(G.bc[2], k, G.nz);
}

// emfx (i in 1..nx, k in 1..nz+1) and emfz (i in 1..nx+1, k in 1..nz) over j in 1..ny+1,
// along y lines (fargo_line): per column the shift is computed once and the donor field and
// its two neighbours (for uin_slope) slide along the segment
template <class Store>
__global__ void __launch_bounds__(kThreads) k_fargo_emf(Geo G, Store U, double *__restrict__ fex,
                                                        double *__restrict__ fez, const Scalars *S) {
    FargoLine L;
    if (!fargo_line(G, blockIdx.x * (long long)blockDim.x + threadIdx.x, L)) return;
    const int i = L.i, k = L.k;
    const double dt = S->dt, dy = G.dy, half = 0.5, one = 1.0;
    const int ny = G.ny, st = mn(G.slope_type, 2);
    const int kw = fargo_zplane(G, k);
    auto lim = [&](double m, double c, double p) { return st == 0 ? 0.0 : limit1<double>((double)st, m, c, p); };
    // one component: get_emfx (v = IC, sign +1, fargo.f90:146-177) or get_emfz (v = IA, sign -1, :204-235)
    auto line = [&](int v, double sgn, const FargoShift &f, double *out) {
        auto B = [&](int jj) { return U.getr(G, v, G.idx(i, jj, kw)); };
        int js = fargo_src(f, L.jb, ny);
        double w0 = B(js - 1 < 1 ? js - 1 + ny : js - 1), w1 = B(js), w2 = B(next_row(js, ny));
        for (int j = L.jb; j <= L.je; j++) {
            if (j > L.jb) {  // slide by one row
                js = next_row(js, ny);
                w0 = w1;
                w1 = w2;
                w2 = B(next_row(js, ny));
            }
            double e = 0.0;
            if (f.vK > 0.0) {
                const double lambda = half * f.eps * (one - f.eps);
                for (int jj = 1; jj <= f.nshft; jj++) {
                    int jr = j - jj;
                    if (jr < 1) jr = jr + ny;
                    e = sgn > 0.0 ? e + B(wrap1(jr, ny)) * dy : e - B(wrap1(jr, ny)) * dy;
                }
                const double demf = f.eps * w1 + lambda * lim(w0, w1, w2);
                e = sgn > 0.0 ? e + demf * dy : e - demf * dy;
            } else {
                const double lambda = half * f.eps * (f.eps - one);
                for (int jj = 0; jj <= f.nshft - 1; jj++) {
                    int jr = j + jj;
                    if (jr > ny) jr = jr - ny;
                    e = sgn > 0.0 ? e - B(wrap1(jr, ny)) * dy : e + B(wrap1(jr, ny)) * dy;
                }
                const double demf = -f.eps * w1 - lambda * lim(w0, w1, w2);
                e = sgn > 0.0 ? e + demf * dy : e - demf * dy;
            }
            out[G.fidx(i, j, k)] = e;
        }
    };
    if (i <= G.nx) line(IC, 1.0, fargo_shift(G, G.xc(i), dt), fex);
    if (k <= G.nz) line(IA, -1.0, fargo_shift(G, half * (G.xc(i) + G.xc(i - 1)), dt), fez);
}

// remap of rho, rho v, E (fargo.f90:59-93) and CT of the face B (fargo.f90:100-119).
// Per row: val = a(js) eps + a(jsp) (1-eps) (or mirrored) + the two slope terms, with
// slope(js) = limit(a(js-1), a(js), a(jsp)) and slope(jsp) = limit(a(js), a(jsp), a(jsp+1))
// (periodic y, the only y boundary FARGO runs with); the row after shares slope(jsp).
// Every value a row needs is loaded before the row's stores (the compiler cannot move a
// load of U across a store to Un): the donor window of the whole segment per variable, and
// the face B and EMFs of kFargoChunk rows at a time for the CT part.
// 3 resident blocks (168 registers): the window stays in registers; timed best at 256^3
#ifndef DG_FARGO_MINB64
#define DG_FARGO_MINB64 3
#endif
template <class Store>
__global__ void __launch_bounds__(kThreads, DG_FARGO_MINB64) k_fargo_update(Geo G, Store U, Store Un, const double *__restrict__ fex,
                                                           const double *__restrict__ fez, const Scalars *S) {
    FargoLine L;
    if (!fargo_line(G, blockIdx.x * (long long)blockDim.x + threadIdx.x, L)) return;
    const int i = L.i, k = L.k;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const double dt = S->dt, half = 0.5, forth = 0.25, one = 1.0;
    if (i <= nx && k <= nz && L.jb <= ny) {
        const FargoShift f = fargo_shift(G, G.xc(i), dt);
        const double hme = half - f.eps;
        const int st = mn(G.slope_type, 2);
        auto lim = [&](double m, double c, double p) { return st == 0 ? 0.0 : limit1<double>((double)st, m, c, p); };
        const int js = fargo_src(f, L.jb, ny);
        const int j0 = js - 1 < 1 ? js - 1 + ny : js - 1;  // the window starts one row below the first donor
        for (int v = IR; v <= IP; v++) {
            // rows js-1 .. js+kFargoSeg+1 (periodic y); rows past the segment's end are loaded but unused
            double wn[kFargoSeg + 3];
            int row = j0;
#pragma unroll
            for (int m = 0; m < kFargoSeg + 3; m++) {
                wn[m] = U.getr(G, v, G.idx(i, row, k));
                row = next_row(row, ny);
            }
            double s0 = lim(wn[0], wn[1], wn[2]);
#pragma unroll
            for (int m = 0; m < kFargoSeg; m++) {
                const int j = L.jb + m;
                if (j > L.je || j > ny) break;
                const double s1 = lim(wn[m + 1], wn[m + 2], wn[m + 3]);
                const double w1 = wn[m + 1], w2 = wn[m + 2];
                double val = (f.vK > 0.0) ? w1 * f.eps + w2 * (one - f.eps) : w1 * (one - f.eps) + w2 * f.eps;
                val = val + half * s0 * (forth - hme * hme) + half * s1 * (hme * hme - forth);
                Un.set(G, v, G.idx(i, j, k), val);
                s0 = s1;
            }
        }
    }
    const double dx = G.dx, dy = G.dy, dz = G.dz;
    // face indices clamped into the EMF arrays; a clamped value is never used
    auto EX = [&](int ii, int jj, int kk) { return ld(fex + G.fidx(ii, mn(jj, G.FY), mn(kk, G.FZ))); };
    auto EZ = [&](int ii, int jj, int kk) { return (ii <= nx + 1) ? ld(fez + G.fidx(ii, mn(jj, G.FY), kk)) : 0.0; };
    for (int jb = L.jb; jb <= L.je; jb += kFargoChunk) {
        double a[kFargoChunk], b[kFargoChunk], cz[kFargoChunk];
        double ezj[kFargoChunk + 1], exj[kFargoChunk + 1], ezr[kFargoChunk], exu[kFargoChunk];
#pragma unroll
        for (int m = 0; m <= kFargoChunk; m++) {
            ezj[m] = EZ(i, jb + m, k);
            exj[m] = EX(i, jb + m, k);
            if (m < kFargoChunk) {
                const int j = mn(jb + m, L.je);
                const long long c = G.idx(i, j, k);
                a[m] = U.getr(G, IA, c);
                b[m] = U.getr(G, IB, c);
                cz[m] = U.getr(G, IC, c);
                ezr[m] = EZ(i + 1, j, k);
                exu[m] = EX(i, j, k + 1);
            }
        }
#pragma unroll
        for (int m = 0; m < kFargoChunk; m++) {
            const int j = jb + m;
            if (j > L.je) break;
            const long long c = G.idx(i, j, k);
            if (j <= ny && k <= nz) Un.set(G, IA, c, a[m] + (ezj[m + 1] - ezj[m]) / dy);
            if (i <= nx && k <= nz) Un.set(G, IB, c, b[m] - (ezr[m] - ezj[m]) / dx + (exu[m] - exj[m]) / dz);
            if (i <= nx && j <= ny) Un.set(G, IC, c, cz[m] - (exj[m + 1] - exj[m]) / dy);
        }
    }
}

// ---------------------------------------------------------------------------
// dissipation (physics.f90:272-664): after boundary when nu > 0 or eta > 0
// (dumses.f90:104); resistivity, then viscosity, then boundary again
// ---------------------------------------------------------------------------
// one thread per point of the face index space [1, nx+1] x [1, ny+1] x [1, nz+1]
__device__ __forceinline__ bool face_point(const Geo &G, long long t, int &i, int &j, int &k) {
    if (t >= G.fsz) return false;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    return true;
}

// resistivity edge EMFs -eta J dt (physics.f90:310-345), J from the face B of the
// state (in 2D only emfz, the one the CT reads).  The resistive energy flux of :350-451 never
// reaches the state in the reference (dissipation zeroes the flux array before
// viscosity and godunov overwrites it), so it is not computed.
template <class Store>
__global__ void __launch_bounds__(kThreads) k_resist_emf(Geo G, Store U, typename Store::T *__restrict__ ex,
                                                         typename Store::T *__restrict__ ey,
                                                         typename Store::T *__restrict__ ez, const Scalars *S) {
    using T = typename Store::T;
    int i, j, k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!face_point(G, t, i, j, k)) return;
    const T dx = (T)G.dx, dy = (T)G.dy, dz = (T)G.dz, eta = (T)G.eta, dt = (T)S->dt, zero = T(0);
    auto B = [&](int v, int ii, int jj, int kk) { return (T)U.getr(G, v, G.idx(ii, jj, kk)); };
    T dBxdy = zero, dBxdz = zero, dBydz = zero, dBzdy = zero, jx = zero;
    const T dBydx = (B(IB, i, j, k) - B(IB, i - 1, j, k)) / dx;
    const T dBzdx = (B(IC, i, j, k) - B(IC, i - 1, j, k)) / dx;
    if (G.ndim > 1) {
        dBxdy = (B(IA, i, j, k) - B(IA, i, j - 1, k)) / dy;
        dBzdy = (B(IC, i, j, k) - B(IC, i, j - 1, k)) / dy;
    }
    if (G.ndim == 3) {
        dBxdz = (B(IA, i, j, k) - B(IA, i, j, k - 1)) / dz;
        dBydz = (B(IB, i, j, k) - B(IB, i, j, k - 1)) / dz;
    }
    if (G.ndim > 1) jx = dBzdy - dBydz;
    const T jy = dBxdz - dBzdx, jz = dBydx - dBxdy;
    if (G.ndim == 3) {  // emfx and emfy enter only the ndim = 3 terms of the CT
        ex[t] = -eta * jx * dt;
        ey[t] = -eta * jy * dt;
    }
    ez[t] = -eta * jz * dt;
}

// constrained_transport (scheme.f90:1940-1993) of the resistive EMFs, in place, on the
// faces that the following boundary keeps: B_x on i = 1..nx+1 (the outer x face is the
// shearing box's own), B_y and B_z of the active cells.  The two loop nests of the
// reference (the ndim >= 2 terms, then the ndim = 3 terms) become two increments.
template <class Store>
__global__ void __launch_bounds__(kThreads) k_ct(Geo G, Store U, const typename Store::T *__restrict__ ex,
                                                 const typename Store::T *__restrict__ ey,
                                                 const typename Store::T *__restrict__ ez) {
    using T = typename Store::T;
    int i, j, k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!face_point(G, t, i, j, k)) return;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const T dx = (T)G.dx, dy = (T)G.dy, dz = (T)G.dz;
    auto E = [&](const T *e, int ii, int jj, int kk) { return ld(e + G.fidx(ii, jj, kk)); };
    const long long c = G.idx(i, j, k);
    if (j <= ny && k <= nz) {
        auto a = U.load(G, IA, c);
        Store::inc(a, (E(ez, i, j + 1, k) - E(ez, i, j, k)) / dy);
        if (G.ndim == 3) Store::inc(a, -((E(ey, i, j, k + 1) - E(ey, i, j, k)) / dz));
        U.store(G, IA, c, a);
    }
    if (i <= nx && k <= nz) {
        auto b = U.load(G, IB, c);
        Store::inc(b, -((E(ez, i + 1, j, k) - E(ez, i, j, k)) / dx));
        if (G.ndim == 3) Store::inc(b, (E(ex, i, j, k + 1) - E(ex, i, j, k)) / dz);
        U.store(G, IB, c, b);
    }
    if (G.ndim == 3 && i <= nx && j <= ny) {
        auto z = U.load(G, IC, c);
        Store::inc(z, (E(ey, i + 1, j, k) - E(ey, i, j, k)) / dx);
        Store::inc(z, -((E(ex, i, j + 1, k) - E(ex, i, j, k)) / dy));
        U.store(G, IC, c, z);
    }
}

// the velocities m / rho of every cell of the ghosted grid, once: each is the quotient the
// reference forms again at every use, so the flux kernel reads them instead
template <class Store>
__global__ void __launch_bounds__(kThreads) k_visc_vel(Geo G, Store U, typename Store::T *__restrict__ vel) {
    using T = typename Store::T;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= G.sv) return;
    const T r = (T)U.getr(G, IR, c);
#pragma unroll
    for (int m = 0; m < 3; m++) vel[G.sv * m + c] = (T)U.getr(G, IU + m, c) / r;
}

// viscous fluxes of momentum and energy (physics.f90:481-643) on the faces the update
// reads: four values per face (rho v_x, rho v_y, rho v_z, E), already x dt/dx_d.
// As in the reference, dudx of the first direction divides the momentum of cell i-1
// by the density of cell i (:494-496).
template <class Store>
__global__ void __launch_bounds__(kThreads) k_visc_flux(Geo G, Store U, const typename Store::T *__restrict__ vel,
                                                        typename Store::T *__restrict__ f0,
                                                        typename Store::T *__restrict__ f1,
                                                        typename Store::T *__restrict__ f2, const Scalars *S) {
    using T = typename Store::T;
    int i, j, k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!face_point(G, t, i, j, k)) return;
    const int nx = G.nx, ny = G.ny, nz = G.nz, nd = G.ndim;
    const T dx = (T)G.dx, dy = (T)G.dy, dz = (T)G.dz, nu = (T)G.nu, dt = (T)S->dt;
    const T zero = T(0), half = T(0.5), forth = T(0.25), two = T(2), two3rd = T(0.66666666666666667);
    auto R = [&](int ii, int jj, int kk) { return (T)U.getr(G, IR, G.idx(ii, jj, kk)); };
    auto M = [&](int m, int ii, int jj, int kk) { return (T)U.getr(G, IR + m, G.idx(ii, jj, kk)); };
    auto V = [&](int m, int ii, int jj, int kk) { return ld(vel + G.sv * (m - 1) + G.idx(ii, jj, kk)); };
    // (d_a u_m) centred on the face: forth ((u(+a) + u(+a,-n)) - (u(-a) + u(-a,-n))) / h_a
    auto cross = [&](int m, int ai, int aj, int ak, int ni, int nj, int nk, T h) {
        const T uR = V(m, i + ai, j + aj, k + ak) + V(m, i + ai - ni, j + aj - nj, k + ak - nk);
        const T uL = V(m, i - ai, j - aj, k - ak) + V(m, i - ai - ni, j - aj - nj, k - ak - nk);
        return forth * (uR - uL) / h;
    };
    T dudx[4], dudy[4], dudz[4];
    if (j <= ny && k <= nz) {  // first direction
        const T rho = half * (R(i, j, k) + R(i - 1, j, k));
        for (int m = 1; m <= 3; m++) dudx[m] = (V(m, i, j, k) - M(m, i - 1, j, k) / R(i, j, k)) / dx;
        if (nd > 1) { dudy[1] = cross(1, 0, 1, 0, 1, 0, 0, dy); dudy[2] = cross(2, 0, 1, 0, 1, 0, 0, dy); }
        if (nd == 3) { dudz[1] = cross(1, 0, 0, 1, 1, 0, 0, dz); dudz[3] = cross(3, 0, 0, 1, 1, 0, 0, dz); }
        else dudz[1] = dudz[3] = zero;
        const T txx = -two3rd * nu * rho * (two * dudx[1] - dudy[2] - dudz[3]);
        const T txy = -nu * rho * (dudy[1] + dudx[2]);
        const T txz = -nu * rho * (dudz[1] + dudx[3]);
        T *f = f0 + t * 4;
        f[0] = txx * dt / dx;
        f[1] = txy * dt / dx;
        f[2] = txz * dt / dx;
        f[3] = zero;
        if (!G.iso) {
            const T u = half * (V(1, i, j, k) + V(1, i - 1, j, k)), v = half * (V(2, i, j, k) + V(2, i - 1, j, k));
            const T w = half * (V(3, i, j, k) + V(3, i - 1, j, k));
            f[3] = (u * txx + v * txy + w * txz) * dt / dx;
        }
    }
    if (nd > 1 && i <= nx && k <= nz) {  // second direction
        const T rho = half * (R(i, j, k) + R(i, j - 1, k));
        for (int m = 1; m <= 3; m++) dudy[m] = (V(m, i, j, k) - V(m, i, j - 1, k)) / dy;
        dudx[1] = cross(1, 1, 0, 0, 0, 1, 0, dx);
        dudx[2] = cross(2, 1, 0, 0, 0, 1, 0, dx);
        if (nd == 3) { dudz[2] = cross(2, 0, 0, 1, 0, 1, 0, dz); dudz[3] = cross(3, 0, 0, 1, 0, 1, 0, dz); }
        else dudz[2] = dudz[3] = zero;
        const T tyy = -two3rd * nu * rho * (two * dudy[2] - dudx[1] - dudz[3]);
        const T txy = -nu * rho * (dudy[1] + dudx[2]);
        const T tyz = -nu * rho * (dudz[2] + dudy[3]);
        T *f = f1 + t * 4;
        f[0] = txy * dt / dy;
        f[1] = tyy * dt / dy;
        f[2] = tyz * dt / dy;
        f[3] = zero;
        if (!G.iso) {
            const T u = half * (V(1, i, j, k) + V(1, i, j - 1, k)), v = half * (V(2, i, j, k) + V(2, i, j - 1, k));
            const T w = half * (V(3, i, j, k) + V(3, i, j - 1, k));
            f[3] = (u * txy + v * tyy + w * tyz) * dt / dy;
        }
    }
    if (nd == 3 && i <= nx && j <= ny) {  // third direction
        const T rho = half * (R(i, j, k) + R(i, j, k - 1));
        for (int m = 1; m <= 3; m++) dudz[m] = (V(m, i, j, k) - V(m, i, j, k - 1)) / dz;
        dudx[1] = cross(1, 1, 0, 0, 0, 0, 1, dx);
        dudx[3] = cross(3, 1, 0, 0, 0, 0, 1, dx);
        dudy[2] = cross(2, 0, 1, 0, 0, 0, 1, dy);
        dudy[3] = cross(3, 0, 1, 0, 0, 0, 1, dy);
        const T tzz = -two3rd * nu * rho * (two * dudz[3] - dudx[1] - dudy[2]);
        const T txz = -nu * rho * (dudz[1] + dudx[3]);
        const T tyz = -nu * rho * (dudz[2] + dudy[3]);
        T *f = f2 + t * 4;
        f[0] = txz * dt / dz;
        f[1] = tyz * dt / dz;
        f[2] = tzz * dt / dz;
        f[3] = zero;
        if (!G.iso) {
            const T u = half * (V(1, i, j, k) + V(1, i, j, k - 1)), v = half * (V(2, i, j, k) + V(2, i, j, k - 1));
            const T w = half * (V(3, i, j, k) + V(3, i, j, k - 1));
            f[3] = (u * txz + v * tyz + w * tzz) * dt / dz;
        }
    }
}

// conservative update of momentum and energy with the viscous fluxes (physics.f90:647-663),
// directions in the order 1, 2, 3
template <class Store>
__global__ void __launch_bounds__(kThreads) k_visc_update(Geo G, Store U, const typename Store::T *__restrict__ f0,
                                                          const typename Store::T *__restrict__ f1,
                                                          const typename Store::T *__restrict__ f2) {
    int i, j, k;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (!face_point(G, t, i, j, k) || i > G.nx || j > G.ny || k > G.nz) return;
    const long long c = G.idx(i, j, k);
    const typename Store::T *F[3] = {f0, f1, f2};
    const long long R[3] = {G.fidx(i + 1, j, k), G.fidx(i, j + 1, k), G.fidx(i, j, k + 1)};
#pragma unroll
    for (int m = 0; m < 4; m++) {
        auto u = U.load(G, IU + m, c);
        for (int d = 0; d < G.ndim; d++) Store::inc(u, ld(F[d] + t * 4 + m) - ld(F[d] + R[d] * 4 + m));
        U.store(G, IU + m, c, u);
    }
}

// ---------------------------------------------------------------------------
// History sums, FP64: the MRI problem's (src/problem/mri/history.f90:60-125) and the default
// routine's of the other problems (src/subroutines/history.f90:57-125); they differ in the
// second velocity of the Reynolds stress (iv2: v_y, v_z) and the second face component of the
// Maxwell stress (ib2: B_y, B_z)
// ---------------------------------------------------------------------------
// pass 1: per-x-column yz sums of vx and the second velocity (compute_yz_mean)
template <class Store>
// raw = 1: the column sums themselves (a z slab's share, summed over the slabs by the caller)
__global__ void k_hist_yzmean(Geo G, Store U, double *__restrict__ m, int raw = 0, int iv2 = IV) {
    const int i = blockIdx.x + 1;
    double a = 0.0, b = 0.0;
    const long long n = (long long)G.ny * G.nz;
    for (long long t = threadIdx.x; t < n; t += blockDim.x) {
        const int j = (int)(t % G.ny) + 1, k = (int)(t / G.ny) + 1;
        const long long c = G.idx(i, j, k);
        const double d = U.get(G, IR, c);
        a += U.get(G, IU, c) / d;
        b += U.get(G, iv2, c) / d;
    }
    __shared__ double sa[256], sb[256];
    sa[threadIdx.x] = a; sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sa[threadIdx.x] += sa[threadIdx.x + s]; sb[threadIdx.x] += sb[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        m[2 * (i - 1)] = raw ? sa[0] : sa[0] / G.ny / G.nz;
        m[2 * (i - 1) + 1] = raw ? sb[0] : sb[0] / G.ny / G.nz;
    }
}

// pass 2: per-block partial sums of the 9 quantities
template <class Store>
__global__ void k_hist_sums(Geo G, Store U, const double *__restrict__ m, double *__restrict__ part, int iv2 = IV,
                            int ib2 = IB) {
    const long long n = (long long)G.nx * G.ny * G.nz;
    const double forth = 0.25;
    const double dtau = G.dx * G.dy * G.dz / (G.xmax - G.xmin) / (G.ymax - G.ymin) / (G.zmax - G.zmin);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // mass, magp, maxwell, Bx, By, Bz, reynolds, divB
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % G.nx) + 1;
        const long long r = t / G.nx;
        const int j = (int)(r % G.ny) + 1, k = (int)(r / G.ny) + 1;
        const long long c = G.idx(i, j, k);
        const double bxl = U.get(G, IA, c), bxr = U.get(G, IA, c + 1);
        const double byl = U.get(G, IB, c), byr = U.get(G, IB, c + G.sy);
        const double bzl = U.get(G, IC, c), bzr = U.get(G, IC, c + G.sz);
        const double bxc = bxl + bxr, byc = byl + byr, bzc = bzl + bzr;
        const double d = U.get(G, IR, c);
        acc[0] += d;
        acc[1] += forth * (bxc * bxc) + forth * (byc * byc) + forth * (bzc * bzc);
        acc[2] += -(forth * bxc * (ib2 == IB ? byc : bzc));
        acc[3] += bxl; acc[4] += byl; acc[5] += bzl;
        acc[6] += d * dtau * (U.get(G, IU, c) / d - m[2 * (i - 1)]) * (U.get(G, iv2, c) / d - m[2 * (i - 1) + 1]);
        acc[7] += (bxr - bxl) / G.dx + (byr - byl) / G.dy + (bzr - bzl) / G.dz;
    }
    __shared__ double sh[8][256];
    for (int q = 0; q < 8; q++) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int q = 0; q < 8; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 8; q++) part[8 * blockIdx.x + q] = sh[q][0];
}

__global__ void k_hist_final(Geo G, const double *__restrict__ part, int nb, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < nb; b++)
        for (int q = 0; q < 8; q++) s[q] += part[8 * b + q];
    const double dtau = G.dx * G.dy * G.dz / (G.xmax - G.xmin) / (G.ymax - G.ymin) / (G.zmax - G.zmin);
    const double mass = s[0] * dtau, magp = 0.5 * s[1] * dtau, maxwell = s[2] * dtau;
    out[0] = mass; out[1] = maxwell; out[2] = s[6]; out[3] = maxwell + s[6]; out[4] = magp;
    out[5] = s[3] * dtau; out[6] = s[4] * dtau; out[7] = s[5] * dtau; out[8] = s[7];
}

}  // namespace
}  // namespace DG_NS
}  // namespace dg
