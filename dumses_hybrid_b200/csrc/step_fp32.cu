// FP32 mixed path: the step kernels of step_impl.cuh instantiated for T = float on a
// compensated FP32 (hi, lo) state, compiled with fast FP32 math.
//
// FP64 is used only where it carries accuracy: turning the state into primitive
// variables (pressure from total energy, which cancels in low-beta zones), the CFL
// reduction, FARGO's remap of the state and the history sums.  Trace, Riemann
// solvers, fluxes, EMFs and the constrained-transport increments are FP32; the
// state update adds each FP32 increment to the (hi, lo) pair with an error-free
// two-sum, so the state carries about 48 significant bits across steps.
#define DG_NS f32
#include "step_impl.cuh"

namespace dg {
namespace f32 {
namespace {

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

__device__ __forceinline__ void apply(const StoreHL &U, const StoreHL &Un, const Geo &G, int v, long long c, float inc) {
    float h = U.hi[G.sv * v + c], l = U.lo[G.sv * v + c];
    add_hl(h, l, inc);
    Un.hi[G.sv * v + c] = h;
    Un.lo[G.sv * v + c] = l;
}

// update + constrained_transport (scheme.f90:1764-1993) as FP32 increments on the compensated state
__global__ void __launch_bounds__(kThreads) k_update3d_hl(Geo G, StoreHL U, StoreHL Un, const float *__restrict__ fx,
                                                          const float *__restrict__ fy, const float *__restrict__ fz,
                                                          const float *__restrict__ ex, const float *__restrict__ ey,
                                                          const float *__restrict__ ez, const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    const int i = (int)(t % G.FX) + 1;
    const long long r = t / G.FX;
    const int j = (int)(r % G.FY) + 1;
    const int k = (int)(r / G.FY) + 1;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const double dtd = S->dt;
    const float dt = (float)dtd;
    const long long fs = G.fsz;
    const long long c = G.idx(i, j, k);
    const bool shear = G.shearing != 0;
    ShearRemap sr{0.0, 0};
    if (shear) sr = shear_offset(G, S->time + 0.5 * dtd);

    if (i <= nx && j <= ny && k <= nz) {
        const float dvloc = (float)(1.0 / (G.dx * G.dy * G.dz));
        const float Om = (float)G.omega0;
        float dr = 0.f, du = 0.f, dv = 0.f, dw = 0.f, dp = 0.f;
        float opl = 1.f;
        if (G.omega0 > 0.0) {
            // Crank-Nicolson Coriolis, ratio - 1 = -2 lambda / (1 + lambda)
            const double lam = 0.25 * (G.omega0 * dtd) * (G.omega0 * dtd);
            opl = (float)(1.0 + lam);
            const float rm1 = (float)(-2.0 * lam / (1.0 + lam));
            const float uu = U.hi[G.sv * IU + c], uv = U.hi[G.sv * IV + c];
            du += uu * rm1 + 2.f * Om * dt * uv / opl;
            dv += uv * rm1 - 0.5f * Om * dt * uu / opl;
        }
        const long long FR[3] = {G.fidx(i + 1, j, k), G.fidx(i, j + 1, k), G.fidx(i, j, k + 1)};
        const float *FA[3] = {fx, fy, fz};
        const float ds[3] = {(float)(G.dy * G.dz), (float)(G.dx * G.dz), (float)(G.dx * G.dy)};
        float pre[3];
        for (int d = 0; d < 3; d++) {
            const float *F = FA[d];
            float rl = ld(F + t), rr = ld(F + FR[d]);
            if (d == 0 && shear) {
                if (i == 1) rl = shear_avg(G, sr, fx, 0, 0, j, k);
                if (i == nx) rr = shear_avg(G, sr, fx, 0, 1, j, k);
            }
            pre[d] = -(ld(F + 5 * fs + FR[d]) * ds[d] - ld(F + 5 * fs + t) * ds[d]) * dt;
            dr += (rl - rr) * dvloc;
            dw += (ld(F + 4 * fs + t) - ld(F + 4 * fs + FR[d])) * dvloc;
            dp += (ld(F + 1 * fs + t) - ld(F + 1 * fs + FR[d])) * dvloc;
            if (G.omega0 > 0.0) {
                float dfn2 = (ld(F + 2 * fs + t) - ld(F + 2 * fs + FR[d])) * dvloc;
                if (d == 0) dfn2 = dfn2 + pre[0] * dvloc;
                float dfn3 = (ld(F + 3 * fs + t) - ld(F + 3 * fs + FR[d])) * dvloc;
                if (d == 1) dfn3 = dfn3 + pre[1] * dvloc;
                du += dfn2 / opl + Om * dt / opl * dfn3;
                dv += dfn3 / opl - 0.25f * Om * dt / opl * dfn2;
            } else {
                du += (ld(F + 2 * fs + t) - ld(F + 2 * fs + FR[d])) * dvloc;
                dv += (ld(F + 3 * fs + t) - ld(F + 3 * fs + FR[d])) * dvloc;
            }
        }
        if (G.omega0 == 0.0) {
            du += pre[0] * dvloc;
            dv += pre[1] * dvloc;
        }
        dw += pre[2] * dvloc;
        apply(U, Un, G, IR, c, dr);
        apply(U, Un, G, IU, c, du);
        apply(U, Un, G, IV, c, dv);
        apply(U, Un, G, IW, c, dw);
        apply(U, Un, G, IP, c, dp);
    }
    auto EYc = [&](int ii, int jj, int kk) -> float {
        if (shear && (ii == 1 || ii == nx + 1) && jj <= ny && kk <= nz + 1)
            return shear_avg(G, sr, ey, 0, ii == 1 ? 0 : 1, jj, kk);
        return ld(ey + G.fidx(ii, jj, kk));
    };
    const float rdx = (float)(1.0 / G.dx), rdy = (float)(1.0 / G.dy), rdz = (float)(1.0 / G.dz);
    const bool ct = G.ndim_act > 1;
    if (j <= ny && k <= nz) {
        float inc = 0.f;
        if (ct) inc = (ld(ez + G.fidx(i, j + 1, k)) - ld(ez + t)) * rdy - (EYc(i, j, k + 1) - EYc(i, j, k)) * rdz;
        apply(U, Un, G, IA, c, inc);
    }
    if (i <= nx && k <= nz) {
        float inc = 0.f;
        if (ct) inc = -(ld(ez + G.fidx(i + 1, j, k)) - ld(ez + t)) * rdx + (ld(ex + G.fidx(i, j, k + 1)) - ld(ex + t)) * rdz;
        apply(U, Un, G, IB, c, inc);
    }
    if (i <= nx && j <= ny) {
        float inc = 0.f;
        if (ct) inc = (EYc(i + 1, j, k) - EYc(i, j, k)) * rdx - (ld(ex + G.fidx(i, j + 1, k)) - ld(ex + t)) * rdy;
        apply(U, Un, G, IC, c, inc);
    }
}

__global__ void __launch_bounds__(kThreads) k_update2d_hl(Geo G, StoreHL U, StoreHL Un, const float *__restrict__ fx,
                                                          const float *__restrict__ fy, const float *__restrict__ ez,
                                                          const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    const int i = (int)(t % G.FX) + 1;
    const int j = (int)(t / G.FX) + 1;
    const int k = 1;
    const int nx = G.nx, ny = G.ny;
    const double dtd = S->dt;
    const float dt = (float)dtd;
    const long long fs = G.fsz;
    const long long c = G.idx(i, j, k);
    if (i <= nx && j <= ny) {
        const float dvloc = (float)(1.0 / (G.dx * G.dy * G.dz));
        const float Om = (float)G.omega0;
        float dr = 0.f, du = 0.f, dv = 0.f, dw = 0.f, dp = 0.f, dc = 0.f;
        float opl = 1.f;
        if (G.omega0 > 0.0) {
            const double lam = 0.25 * (G.omega0 * dtd) * (G.omega0 * dtd);
            opl = (float)(1.0 + lam);
            const float rm1 = (float)(-2.0 * lam / (1.0 + lam));
            const float uu = U.hi[G.sv * IU + c], uv = U.hi[G.sv * IV + c];
            du += uu * rm1 + 2.f * Om * dt * uv / opl;
            dv += uv * rm1 - 0.5f * Om * dt * uu / opl;
        }
        const long long FR[2] = {G.fidx(i + 1, j, k), G.fidx(i, j + 1, k)};
        const float *FA[2] = {fx, fy};
        const float ds[2] = {(float)(G.dy * G.dz), (float)(G.dx * G.dz)};
        float pre[2];
        for (int d = 0; d < 2; d++) {
            const float *F = FA[d];
            pre[d] = -(ld(F + 5 * fs + FR[d]) * ds[d] - ld(F + 5 * fs + t) * ds[d]) * dt;
            dr += (ld(F + t) - ld(F + FR[d])) * dvloc;
            dw += (ld(F + 4 * fs + t) - ld(F + 4 * fs + FR[d])) * dvloc;
            dp += (ld(F + 1 * fs + t) - ld(F + 1 * fs + FR[d])) * dvloc;
            dc += (ld(F + 6 * fs + t) - ld(F + 6 * fs + FR[d])) * dvloc;
            if (G.omega0 > 0.0) {
                float dfn2 = (ld(F + 2 * fs + t) - ld(F + 2 * fs + FR[d])) * dvloc;
                if (d == 0) dfn2 = dfn2 + pre[0] * dvloc;
                float dfn3 = (ld(F + 3 * fs + t) - ld(F + 3 * fs + FR[d])) * dvloc;
                if (d == 1) dfn3 = dfn3 + pre[1] * dvloc;
                du += dfn2 / opl + Om * dt / opl * dfn3;
                dv += dfn3 / opl - 0.25f * Om * dt / opl * dfn2;
            } else {
                du += (ld(F + 2 * fs + t) - ld(F + 2 * fs + FR[d])) * dvloc;
                dv += (ld(F + 3 * fs + t) - ld(F + 3 * fs + FR[d])) * dvloc;
            }
        }
        if (G.omega0 == 0.0) {
            du += pre[0] * dvloc;
            dv += pre[1] * dvloc;
        }
        apply(U, Un, G, IR, c, dr);
        apply(U, Un, G, IU, c, du);
        apply(U, Un, G, IV, c, dv);
        apply(U, Un, G, IW, c, dw);
        apply(U, Un, G, IP, c, dp);
        apply(U, Un, G, IC, c, dc);
    }
    const bool ct = G.ndim_act > 1;
    const float rdx = (float)(1.0 / G.dx), rdy = (float)(1.0 / G.dy);
    if (j <= ny) {
        float inc = ct ? (ld(ez + G.fidx(i, j + 1, k)) - ld(ez + t)) * rdy : 0.f;
        apply(U, Un, G, IA, c, inc);
    }
    if (i <= nx) {
        float inc = ct ? -(ld(ez + G.fidx(i + 1, j, k)) - ld(ez + t)) * rdx : 0.f;
        apply(U, Un, G, IB, c, inc);
    }
}

StoreHL st(const Bufs &B, int b) {
    float *base = (float *)B.U[b];
    return StoreHL{base, base + (size_t)B.nv * (size_t)B.sv};
}

}  // namespace

#define TIMED(slot, st, launch)                          \
    do {                                                 \
        if (g_timer) g_timer->begin(slot, st);           \
        launch;                                          \
        if (g_timer) g_timer->end(slot, st);             \
    } while (0)

int launch_set_scalars(const Bufs &B, double dt, double time, int set_dt, int set_time, cudaStream_t s) {
    TIMED(KS_SCALARS, s, (k_set_scalars<<<1, 1, 0, s>>>(B.S, dt, time, set_dt, set_time)));
    return 1;
}

int launch_advance_time(const Bufs &B, cudaStream_t s) {
    TIMED(KS_SCALARS, s, (k_advance_time<<<1, 1, 0, s>>>(B.S)));
    return 1;
}

int launch_dt(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    TIMED(KS_DT, s, (k_dt_reset<<<1, 1, 0, s>>>(G, B.S)));
    const long long n = (long long)G.nx * G.ny * G.nz;
    long long nb = (n + kThreads - 1) / kThreads;
    if (nb > 148 * 16) nb = 148 * 16;
    TIMED(KS_DT, s, (k_dt<StoreHL><<<(unsigned)nb, kThreads, 0, s>>>(G, st(B, cur), B.S)));
    TIMED(KS_DT, s, (k_dt_final<<<1, 1, 0, s>>>(G, B.S)));
    return 3;
}

int launch_godunov(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreHL U = st(B, cur), Un = st(B, cur ^ 1);
    float *Q = (float *)B.Q, *core = (float *)B.core;
    float *E0 = (float *)B.E[0], *E1 = (float *)B.E[1], *E2 = (float *)B.E[2];
    float *fx = (float *)B.flx[0], *fy = (float *)B.flx[1], *fz = (float *)B.flx[2];
    float *ex = (float *)B.emf[0], *ey = (float *)B.emf[1], *ez = (float *)B.emf[2];
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    TIMED(KS_PRIM, s, (k_prim<float, StoreHL><<<nblocks((long long)ni * nj * nk, kThreads), kThreads, 0, s>>>(G, U, Q, B.S)));
    if (G.ndim == 3) {
        TIMED(KS_EFIELD, s, (k_efield3d<float><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2)));
        TIMED(KS_TRACE, s, (k_trace3d<float><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2, core, B.S)));
        TIMED(KS_RIEMANN, s, (k_riemann3d<float><<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, core, fx, fy, fz, ex, ey, ez, B.S)));
        TIMED(KS_UPDATE, s, (k_update3d_hl<<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, U, Un, fx, fy, fz, ex, ey, ez, B.S)));
    } else {
        TIMED(KS_EFIELD, s, (k_efield2d<float><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E2)));
        TIMED(KS_TRACE, s, (k_trace2d<float><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E2, core, B.S)));
        TIMED(KS_RIEMANN, s, (k_riemann2d<float><<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, core, fx, fy, ez, B.S)));
        TIMED(KS_UPDATE, s, (k_update2d_hl<<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, U, Un, fx, fy, ez, B.S)));
    }
    return 5;
}

int launch_fargo(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    TIMED(KS_FARGO_EMF, s, (k_fargo_emf<StoreHL><<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, st(B, cur), B.femf[0], B.femf[1], B.S)));
    TIMED(KS_FARGO_UPDATE, s, (k_fargo_update<StoreHL><<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, st(B, cur), st(B, cur ^ 1), B.femf[0], B.femf[1], B.S)));
    return 2;
}

int launch_boundary(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const long long n = (long long)G.NX * G.NY * G.NZ;
    TIMED(KS_BOUNDARY, s, (k_boundary<StoreHL><<<nblocks(n, kThreads), kThreads, 0, s>>>(G, st(B, cur), B.nv, B.S)));
    return 1;
}

int launch_right_faces(const Geo &G, const Bufs &B, int cur, double *out, cudaStream_t s) {
    const long long n = (long long)G.NX * G.NY * G.NZ;
    TIMED(KS_RIGHT_FACES, s, (k_right_faces<StoreHL><<<nblocks(n, 256), 256, 0, s>>>(G, st(B, cur), out)));
    return 1;
}

int launch_state_to_f64(const Geo &G, const Bufs &B, int cur, double *out, cudaStream_t s) {
    TIMED(KS_RIGHT_FACES, s, (k_state_to_f64<StoreHL><<<nblocks(G.sv * B.nv, 256), 256, 0, s>>>(G, st(B, cur), B.nv, out)));
    return 1;
}

int launch_f64_to_state(const Geo &G, const Bufs &B, int b, const double *in, int nv, cudaStream_t s) {
    TIMED(KS_RIGHT_FACES, s, (k_f64_to_state<StoreHL><<<nblocks(G.sv * nv, 256), 256, 0, s>>>(G, in, nv, st(B, b))));
    return 1;
}

int launch_history(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const int nb = 296;
    TIMED(KS_HISTORY, s, (k_hist_yzmean<StoreHL><<<G.nx, 256, 0, s>>>(G, st(B, cur), B.part)));
    TIMED(KS_HISTORY, s, (k_hist_sums<StoreHL><<<nb, 256, 0, s>>>(G, st(B, cur), B.part, B.part + 2 * G.nx)));
    TIMED(KS_HISTORY, s, (k_hist_final<<<1, 32, 0, s>>>(G, B.part + 2 * G.nx, nb, B.hist)));
    return 3;
}

}  // namespace f32
}  // namespace dg
