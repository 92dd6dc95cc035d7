// FP64 plain path: the step kernels of step_impl.cuh instantiated for T = double
// on an FP64 state, compiled with --fmad=false.  Bit-identical to the reference
// arithmetic (see dg_common.cuh).
#define DG_NS f64
#include "step_impl.cuh"

namespace dg {
namespace f64 {
namespace {

// update + constrained_transport of the FP64 state (scheme.f90:1764-1993), in the
// reference's statement order
// 8 resident blocks (64 registers), chosen by timing at 256^3
#ifndef DG_UPDATE_MINB64
#define DG_UPDATE_MINB64 8
#endif
#if DG_UPDATE_MINB64 > 0
__global__ void __launch_bounds__(kThreads, DG_UPDATE_MINB64) k_update3d(
#else
__global__ void __launch_bounds__(kThreads) k_update3d(
#endif
    Geo G, const double *__restrict__ U, double *__restrict__ Un,
                                                       const double *__restrict__ fx, const double *__restrict__ fy,
                                                       const double *__restrict__ fz, const double *__restrict__ ex,
                                                       const double *__restrict__ ey, const double *__restrict__ ez,
                                                       const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    int i, j, k;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    const long long fxy = (long long)G.FX * G.FY;  // face index steps: +1 (x), +FX (y), +fxy (z)
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const double dt = S->dt;
    const double one = 1.0, two = 2.0, half = 0.5;
    const long long sv = G.sv;
    const long long c = G.idx(i, j, k);
    if (!chk(Un + c, 8) || !chk(Un + sv * IC + c, 8)) return;  // the planes this thread writes
    const bool shear = G.shearing != 0;
    ShearRemap sr{0.0, 0};
    if (shear) sr = ShearRemap{S->sh_epsi, S->sh_jp};  // time + dt/2, from k_shear_offset

    if (i <= nx && j <= ny && k <= nz) {
        // hydro update, scheme.f90:1783-1907
        const double Omega0 = G.omega0;
        double lambda = 0.0, ratio = 0.0;
        if (Omega0 > 0.0) {
            lambda = Omega0 * dt; lambda = 2.5e-1 * lambda * lambda;
            ratio = (one - lambda) / (one + lambda);
        }
        const double dvloc = G.dvloc;  // one / (dx dy dz)
        double ur = ld(U + c), uu = ld(U + sv * IU + c), uv = ld(U + sv * IV + c), uw = ld(U + sv * IW + c);
        double up = ld(U + sv * IP + c);
        if (Omega0 > 0.0) {
            const double dsx = two * Omega0 * dt * uv / (one + lambda);
            const double dsy = -(half * Omega0 * dt * uu) / (one + lambda);
            uu = uu * ratio + dsx;
            uv = uv * ratio + dsy;
        }
        const long long f0 = t;
        const long long fxr = (t + 1), fyr = (t + G.FX), fzr = (t + fxy);
        const double *FA[3] = {fx, fy, fz};
        const long long FR[3] = {fxr, fyr, fzr};
        double pre[3];
        for (int d = 0; d < 3; d++) {
            double L[6], R[6];
            load6(FA[d] + f0 * kFluxRec3, L);
            load6(FA[d] + FR[d] * kFluxRec3, R);
            double rl = L[0], rr = R[0];
            if (d == 0 && shear) {
                if (i == 1) rl = shear_avg(G, sr, fx, kFluxRec3, 0, j, k);
                if (i == nx) rr = shear_avg(G, sr, fx, kFluxRec3, 1, j, k);
            }
            const double ds = (d == 0) ? G.dy * G.dz : (d == 1 ? G.dx * G.dz : G.dx * G.dy);
            pre[d] = -(R[5] * ds - L[5] * ds) * dt;
            ur = ur + (rl - rr) * dvloc;
            uw = uw + (L[4] * one - R[4] * one) * dvloc / one;
            up = up + (L[1] - R[1]) * dvloc;
            if (Omega0 > 0.0) {
                double dfn2 = (L[2] - R[2]) * dvloc;
                if (d == 0) dfn2 = dfn2 + pre[0] * dvloc;
                double dfn3 = (L[3] - R[3]) * dvloc;
                if (d == 1) dfn3 = dfn3 + pre[1] * dvloc;
                uu = uu + dfn2 / (one + lambda) + Omega0 * dt / (one + lambda) * dfn3;
                uv = uv + dfn3 / (one + lambda) - 2.5e-1 * Omega0 * dt / (one + lambda) * dfn2;
            } else {
                uu = uu + (L[2] * one - R[2] * one) * dvloc / one;
                uv = uv + (L[3] * one - R[3] * one) * dvloc / one;
            }
        }
        if (Omega0 == 0.0) {
            uu = uu + pre[0] * dvloc;
            uv = uv + pre[1] * dvloc;
        }
        uw = uw + pre[2] * dvloc;
        Un[c] = ur; Un[sv * IU + c] = uu; Un[sv * IV + c] = uv; Un[sv * IW + c] = uw; Un[sv * IP + c] = up;
    }
    // constrained transport of the left faces, scheme.f90:1957-1993 (ranges 1..n+1)
    auto EYc = [&](int ii, int jj, int kk) -> double {
        if (shear && (ii == 1 || ii == nx + 1) && jj <= ny && kk <= nz + 1)
            return shear_avg(G, sr, ey, 1, ii == 1 ? 0 : 1, jj, kk);
        return ld(ey + G.fidx(ii, jj, kk));
    };
    const bool ct = G.ndim_act > 1;
    if (j <= ny && k <= nz) {  // B_x at face i (i = 1..nx+1)
        double b = ld(U + sv * IA + c);
        if (ct) {
            b = b + G.per_dy(ld(ez + (t + G.FX)) - ld(ez + t));
            b = b - G.per_dz(EYc(i, j, k + 1) - EYc(i, j, k));
        }
        Un[sv * IA + c] = b;
    }
    if (i <= nx && k <= nz) {  // B_y at face j
        double b = ld(U + sv * IB + c);
        if (ct) {
            b = b - G.per_dx(ld(ez + (t + 1)) - ld(ez + t));
            b = b + G.per_dz(ld(ex + (t + fxy)) - ld(ex + t));
        }
        Un[sv * IB + c] = b;
    }
    if (i <= nx && j <= ny) {  // B_z at face k
        double b = ld(U + sv * IC + c);
        if (ct) b = b + G.per_dx(EYc(i + 1, j, k) - EYc(i, j, k)) - G.per_dy(ld(ex + (t + G.FX)) - ld(ex + t));
        Un[sv * IC + c] = b;
    }
}

// update of the FP64 state with ndim = 1 (scheme.f90:1764-1936): every field from its x fluxes,
// no constrained transport (ndim_act = 1), in the reference's statement order
__global__ void __launch_bounds__(kThreads) k_update1d(Geo G, const double *__restrict__ U, double *__restrict__ Un,
                                                       const double *__restrict__ fx, const Scalars *S) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.nx) return;
    const int i = (int)t + 1;
    const double dt = S->dt;
    const double one = 1.0, two = 2.0, half = 0.5;
    const long long sv = G.sv, c = G.idx(i, 1, 1);
    if (!chk(Un + c, 8) || !chk(Un + sv * IC + c, 8)) return;
    const double Omega0 = G.omega0;
    double lambda = 0.0, ratio = 0.0;
    if (Omega0 > 0.0) {
        lambda = Omega0 * dt; lambda = 2.5e-1 * lambda * lambda;
        ratio = (one - lambda) / (one + lambda);
    }
    const double dvloc = G.dvloc;  // one / dv
    double ur = ld(U + c), uu = ld(U + sv * IU + c), uv = ld(U + sv * IV + c), uw = ld(U + sv * IW + c);
    double up = ld(U + sv * IP + c), ua = ld(U + sv * IA + c), ub = ld(U + sv * IB + c), uc = ld(U + sv * IC + c);
    if (Omega0 > 0.0) {
        const double dsx = two * Omega0 * dt * uv / (one + lambda);
        const double dsy = -(half * Omega0 * dt * uu) / (one + lambda);
        uu = uu * ratio + dsx;
        uv = uv * ratio + dsy;
    }
    const double *L = fx + t * kFluxRec1, *R = fx + (t + 1) * kFluxRec1;  // faces i and i+1
    const double ds = G.dy * G.dz;
    const double pre = -(ld(R + 5) * ds - ld(L + 5) * ds) * dt;  // fgodunov_pre, solver.f90:246-262
    ur = ur + (ld(L) - ld(R)) * dvloc;
    uw = uw + (ld(L + 4) * one - ld(R + 4) * one) * dvloc / one;
    up = up + (ld(L + 1) - ld(R + 1)) * dvloc;
    ua = ua + (ld(L + 6) - ld(R + 6)) * dvloc;
    ub = ub + (ld(L + 7) - ld(R + 7)) * dvloc;
    uc = uc + (ld(L + 8) - ld(R + 8)) * dvloc;
    if (Omega0 > 0.0) {
        double dfn2 = (ld(L + 2) - ld(R + 2)) * dvloc;
        dfn2 = dfn2 + pre * dvloc;
        const double dfn3 = (ld(L + 3) - ld(R + 3)) * dvloc;
        uu = uu + dfn2 / (one + lambda) + Omega0 * dt / (one + lambda) * dfn3;
        uv = uv + dfn3 / (one + lambda) - 2.5e-1 * Omega0 * dt / (one + lambda) * dfn2;
    } else {
        uu = uu + (ld(L + 2) * one - ld(R + 2) * one) * dvloc / one;
        uv = uv + (ld(L + 3) * one - ld(R + 3) * one) * dvloc / one;
        uu = uu + pre * dvloc;
    }
    Un[c] = ur; Un[sv * IU + c] = uu; Un[sv * IV + c] = uv; Un[sv * IW + c] = uw; Un[sv * IP + c] = up;
    Un[sv * IA + c] = ua; Un[sv * IB + c] = ub; Un[sv * IC + c] = uc;
}

__global__ void __launch_bounds__(kThreads) k_update2d(Geo G, const double *__restrict__ U, double *__restrict__ Un,
                                                       const double *__restrict__ fx, const double *__restrict__ fy,
                                                       const double *__restrict__ ez, const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    const int j = (int)fdiv((unsigned)t, G.dFX) + 1;
    const int i = (int)((unsigned)t - (unsigned)(j - 1) * G.dFX.d) + 1;
    const int k = 1;
    const int nx = G.nx, ny = G.ny;
    const double dt = S->dt;
    const double one = 1.0, two = 2.0, half = 0.5;
    const long long sv = G.sv;
    const long long c = G.idx(i, j, k);
    if (i <= nx && j <= ny) {
        const double Omega0 = G.omega0;
        double lambda = 0.0, ratio = 0.0;
        if (Omega0 > 0.0) {
            lambda = Omega0 * dt; lambda = 2.5e-1 * lambda * lambda;
            ratio = (one - lambda) / (one + lambda);
        }
        const double dv = G.dx * G.dy * G.dz;
        const double dvloc = one / dv;
        double ur = ld(U + c), uu = ld(U + sv * IU + c), uv = ld(U + sv * IV + c), uw = ld(U + sv * IW + c);
        double up = ld(U + sv * IP + c), uc = ld(U + sv * IC + c);
        if (Omega0 > 0.0) {
            const double dsx = two * Omega0 * dt * uv / (one + lambda);
            const double dsy = -(half * Omega0 * dt * uu) / (one + lambda);
            uu = uu * ratio + dsx;
            uv = uv * ratio + dsy;
        }
        const long long FR[2] = {G.fidx(i + 1, j, k), G.fidx(i, j + 1, k)};
        const double *FA[2] = {fx, fy};
        double pre[2];
        for (int d = 0; d < 2; d++) {
            double L[8], R[8];
            load8(FA[d] + t * kFluxRec2, L);
            load8(FA[d] + FR[d] * kFluxRec2, R);
            const double ds = (d == 0) ? G.dy * G.dz : G.dx * G.dz;
            pre[d] = -(R[5] * ds - L[5] * ds) * dt;
            ur = ur + (L[0] - R[0]) * dvloc;
            uw = uw + (L[4] * one - R[4] * one) * dvloc / one;
            up = up + (L[1] - R[1]) * dvloc;
            uc = uc + (L[6] - R[6]) * dvloc;
            if (Omega0 > 0.0) {
                double dfn2 = (L[2] - R[2]) * dvloc;
                if (d == 0) dfn2 = dfn2 + pre[0] * dvloc;
                double dfn3 = (L[3] - R[3]) * dvloc;
                if (d == 1) dfn3 = dfn3 + pre[1] * dvloc;
                uu = uu + dfn2 / (one + lambda) + Omega0 * dt / (one + lambda) * dfn3;
                uv = uv + dfn3 / (one + lambda) - 2.5e-1 * Omega0 * dt / (one + lambda) * dfn2;
            } else {
                uu = uu + (L[2] * one - R[2] * one) * dvloc / one;
                uv = uv + (L[3] * one - R[3] * one) * dvloc / one;
            }
        }
        if (Omega0 == 0.0) {
            uu = uu + pre[0] * dvloc;
            uv = uv + pre[1] * dvloc;
        }
        Un[c] = ur; Un[sv * IU + c] = uu; Un[sv * IV + c] = uv; Un[sv * IW + c] = uw; Un[sv * IP + c] = up;
        Un[sv * IC + c] = uc;
    }
    const bool ct = G.ndim_act > 1;
    if (j <= ny) {
        double b = ld(U + sv * IA + c);
        if (ct) b = b + (ld(ez + G.fidx(i, j + 1, k)) - ld(ez + t)) / G.dy;
        Un[sv * IA + c] = b;
    }
    if (i <= nx) {
        double b = ld(U + sv * IB + c);
        if (ct) b = b - (ld(ez + G.fidx(i + 1, j, k)) - ld(ez + t)) / G.dx;
        Un[sv * IB + c] = b;
    }
}


StoreD st(const Bufs &B, int b) { return StoreD{(double *)B.U[b]}; }

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

// compute_dt; the pass also leaves primitive(0) in Q for the godunov that follows (B.q_fresh)
int launch_dt(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    TIMED(KS_DT, s, (k_dt_reset<<<1, 1, 0, s>>>(G, B.S)));
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    TIMED(KS_DT, s, (k_prim_dt<StoreD><<<nblocks((long long)ni * nj * nk, kThreads), kThreads, 0, s>>>(G, st(B, cur), (double *)B.Q, B.S)));
    TIMED(KS_DT, s, (k_dt_final<<<1, 1, 0, s>>>(G, B.S)));
    return 3;
}

// the rotation half-kick of primitive(dt) on Q = primitive(0), as prim_cell applies it
// (scheme.f90:78-85): one thread per element of the velocity planes
__global__ void __launch_bounds__(kThreads) k_kick64(Geo G, double *__restrict__ Q, const Scalars *S) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= G.sv) return;
    const double half = 0.5, two = 2.0, dt = S->dt;
    const double u = Q[G.sv * IU + c], v = Q[G.sv * IV + c];
    const double dvx = two * G.omega0 * v;
    const double dvy = -(half * G.omega0 * u);
    Q[G.sv * IU + c] = u + dvx * dt * half;
    Q[G.sv * IV + c] = v + dvy * dt * half;
}

// 3D trace as two kernels: cell fields (5 blocks per SM, 96 registers), then face fields
// (6 blocks per SM); 3.03 against 3.68 ms at 256^3 for the single kernel, which spills at 128
#ifndef DG_TRACE_SPLIT64
#define DG_TRACE_SPLIT64 1
#endif
constexpr bool kTraceSplit64 = DG_TRACE_SPLIT64 != 0;
// 3D trace with its stencil staged in shared memory (k_trace3d_tile)
#ifndef DG_TRACE_TILE64
#define DG_TRACE_TILE64 1
#endif
constexpr bool kTraceTile64 = DG_TRACE_TILE64 != 0;

// 3D Riemann work as two kernels (faces, then edges) instead of one
#ifndef DG_RIEMANN_SPLIT64
#define DG_RIEMANN_SPLIT64 1
#endif
constexpr bool kRiemannSplit64 = DG_RIEMANN_SPLIT64 != 0;
// HLLD/HLLD: one kernel per direction for the faces and for the edges (six launches; each
// kernel's code is a third of the two-kernel form's, and 7.57 against 8.22 ms at 256^3)
#ifndef DG_RIEMANN_PERDIR64
#define DG_RIEMANN_PERDIR64 1
#endif
constexpr bool kRiemannPerDir64 = DG_RIEMANN_PERDIR64 != 0;

int launch_godunov(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreD U = st(B, cur);
    double *Un = (double *)B.U[cur ^ 1];
    double *Q = (double *)B.Q, *core = (double *)B.core;
    double *E0 = (double *)B.E[0], *E1 = (double *)B.E[1], *E2 = (double *)B.E[2];
    double *fx = (double *)B.flx[0], *fy = (double *)B.flx[1], *fz = (double *)B.flx[2];
    double *ex = (double *)B.emf[0], *ey = (double *)B.emf[1], *ez = (double *)B.emf[2];
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    int n = 4 + (G.shearing ? 1 : 0);
    if (!B.q_fresh) {
        TIMED(KS_PRIM, s, (k_prim<double, StoreD><<<nblocks((long long)ni * nj * nk, kThreads), kThreads, 0, s>>>(G, U, Q, B.S)));
        n++;
    } else if (G.omega0 > 0.0) {  // Q = primitive(0) of this state from launch_dt: add the half-kick
        TIMED(KS_PRIM, s, (k_kick64<<<nblocks(G.sv, kThreads), kThreads, 0, s>>>(G, Q, B.S)));
        n++;
    }
    if (G.shearing) TIMED(KS_SCALARS, s, (k_shear_offset<<<1, 1, 0, s>>>(G, B.S, 0.5)));
    if (G.ndim == 3) {
        // the tiled trace computes its edge fields itself
        if (kTraceTile64) n--;
        else TIMED(KS_EFIELD, s, (k_efield3d<double><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.p, E0, E1, E2)));
        if (kTraceTile64 && kTraceSplit64) {
            TIMED(KS_TRACE, s, (launch_trace_tile<double, 1>(G, Q, U.p, core, B.S, s)));
            TIMED(KS_TRACE, s, (launch_trace_tile<double, 2>(G, Q, U.p, core, B.S, s)));
            n++;
        } else if (kTraceTile64) {
            TIMED(KS_TRACE, s, (launch_trace_tile<double>(G, Q, U.p, core, B.S, s)));
        } else if (kTraceSplit64) {
            TIMED(KS_TRACE, s, (k_trace3d<double, 1><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.p, E0, E1, E2, core, B.S)));
            TIMED(KS_TRACE, s, (k_trace3d<double, 2><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.p, E0, E1, E2, core, B.S)));
            n++;
        } else {
            TIMED(KS_TRACE, s, (k_trace3d<double><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.p, E0, E1, E2, core, B.S)));
        }
        // HLLD/HLLD (the reference's default and every benchmark) runs kernels without the other solvers
        const unsigned nb = nblocks(G.fsz, kThreads);
        if (kRiemannPerDir64 && G.iriemann == DG_RIEMANN_HLLD && G.iriemann2d == DG_RIEMANN_HLLD) {
            TIMED(KS_RIEMANN, s, (k_faces3d<double, true, 0><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
            TIMED(KS_RIEMANN, s, (k_faces3d<double, true, 1><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
            TIMED(KS_RIEMANN, s, (k_faces3d<double, true, 2><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
            TIMED(KS_RIEMANN, s, (k_edges3d<double, true, 0><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
            TIMED(KS_RIEMANN, s, (k_edges3d<double, true, 1><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
            TIMED(KS_RIEMANN, s, (k_edges3d<double, true, 2><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
            n += 5;
        } else if (kRiemannSplit64) {
            if (G.iriemann == DG_RIEMANN_HLLD && G.iriemann2d == DG_RIEMANN_HLLD) {
                TIMED(KS_RIEMANN, s, (k_faces3d<double, true><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
                TIMED(KS_RIEMANN, s, (k_edges3d<double, true><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
            } else {
                TIMED(KS_RIEMANN, s, (k_faces3d<double, false><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
                TIMED(KS_RIEMANN, s, (k_edges3d<double, false><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
            }
            n++;
        } else if (G.iriemann == DG_RIEMANN_HLLD && G.iriemann2d == DG_RIEMANN_HLLD) {
            TIMED(KS_RIEMANN, s, (k_riemann3d<double, true><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, ex, ey, ez, B.S, 1)));
        } else {
            TIMED(KS_RIEMANN, s, (k_riemann3d<double, false><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, ex, ey, ez, B.S, 1)));
        }
        TIMED(KS_UPDATE, s, (k_update3d<<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, U.p, Un, fx, fy, fz, ex, ey, ez, B.S)));
    } else if (G.ndim == 1) {
        // trace1d, the x solves, update: no edge fields and no EMFs
        const bool hlld = G.iriemann == DG_RIEMANN_HLLD;
        TIMED(KS_TRACE, s, (k_trace1d<double><<<nblocks(G.CX, kThreads), kThreads, 0, s>>>(G, Q, core, B.S)));
        if (hlld) TIMED(KS_RIEMANN, s, (k_riemann1d<double, true><<<nblocks(G.FX, kThreads), kThreads, 0, s>>>(G, core, fx, B.S)));
        else TIMED(KS_RIEMANN, s, (k_riemann1d<double, false><<<nblocks(G.FX, kThreads), kThreads, 0, s>>>(G, core, fx, B.S)));
        TIMED(KS_UPDATE, s, (k_update1d<<<nblocks(G.nx, kThreads), kThreads, 0, s>>>(G, U.p, Un, fx, B.S)));
        n--;
    } else {
        TIMED(KS_EFIELD, s, (k_efield2d<double><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.p, E2)));
        TIMED(KS_TRACE, s, (k_trace2d<double><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.p, E2, core, B.S)));
        TIMED(KS_RIEMANN, s, (k_riemann2d<double><<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, core, fx, fy, ez, B.S, 1)));
        TIMED(KS_UPDATE, s, (k_update2d<<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, U.p, Un, fx, fy, ez, B.S)));
    }
    return n;
}

int launch_fargo(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    TIMED(KS_FARGO_EMF, s, (k_fargo_emf<StoreD><<<nblocks(fargo_line_threads(G), kThreads), kThreads, 0, s>>>(G, st(B, cur), B.femf[0], B.femf[1], B.S)));
    TIMED(KS_FARGO_UPDATE, s, (k_fargo_update<StoreD><<<nblocks(fargo_line_threads(G), kThreads), kThreads, 0, s>>>(G, st(B, cur), st(B, cur ^ 1), B.femf[0], B.femf[1], B.S)));
    return 2;
}

int launch_boundary(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    int n = 1;
    if (G.shearing) {
        TIMED(KS_SCALARS, s, (k_shear_offset<<<1, 1, 0, s>>>(G, B.S, 1.0)));
        n++;
    }
    TIMED(KS_BOUNDARY, s, (k_boundary<StoreD><<<nblocks(ghost_cells(G), kThreads), kThreads, 0, s>>>(G, st(B, cur), B.nv, B.S)));
    return n;
}

int launch_right_faces(const Geo &G, const Bufs &B, int cur, double *out, cudaStream_t s) {
    const long long n = (long long)G.NX * G.NY * G.NZ;
    TIMED(KS_RIGHT_FACES, s, (k_right_faces<StoreD><<<nblocks(n, 256), 256, 0, s>>>(G, st(B, cur), out)));
    return 1;
}

int launch_state_to_f64(const Geo &G, const Bufs &B, int cur, double *out, cudaStream_t s) {
    TIMED(KS_RIGHT_FACES, s, (k_state_to_f64<StoreD><<<nblocks(G.sv * B.nv, 256), 256, 0, s>>>(G, st(B, cur), B.nv, out)));
    return 1;
}

int launch_f64_to_state(const Geo &G, const Bufs &B, int b, const double *in, int nv, cudaStream_t s) {
    TIMED(KS_RIGHT_FACES, s, (k_f64_to_state<StoreD><<<nblocks(G.sv * nv, 256), 256, 0, s>>>(G, in, nv, st(B, b))));
    return 1;
}

constexpr int kHistBlocks = 296;

long long history_scratch_doubles(const Geo &G) { return 2LL * G.nx + 8LL * kHistBlocks; }

int launch_history_ptrs(const Geo &G, const double *U, double *scratch, double *out, cudaStream_t s, int variant) {
    // every scratch entry read below is written earlier in the same launch sequence
    const StoreD S{(double *)U};
    const int iv2 = variant == DG_HISTORY_DEFAULT ? IW : IV, ib2 = variant == DG_HISTORY_DEFAULT ? IC : IB;
    TIMED(KS_HISTORY, s, (k_hist_yzmean<StoreD><<<G.nx, 256, 0, s>>>(G, S, scratch, 0, iv2)));
    TIMED(KS_HISTORY, s, (k_hist_sums<StoreD><<<kHistBlocks, 256, 0, s>>>(G, S, scratch, scratch + 2 * G.nx, iv2, ib2)));
    TIMED(KS_HISTORY, s, (k_hist_final<<<1, 32, 0, s>>>(G, scratch + 2 * G.nx, kHistBlocks, out)));
    return 3;
}

// dissipation (physics.f90:272-291): resistive EMFs + CT, viscous fluxes + update, in
// place on U[cur], then boundary; the step's EMF and flux arrays are free at this point
int launch_dissipation(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreD U = st(B, cur);
    double *e0 = (double *)B.emf[0], *e1 = (double *)B.emf[1], *e2 = (double *)B.emf[2];
    double *f0 = (double *)B.flx[0], *f1 = (double *)B.flx[1], *f2 = G.ndim == 3 ? (double *)B.flx[2] : f0;
    if (G.ndim == 2) e0 = e1 = e2;  // 2D: only emfz is allocated and used
    const unsigned nb = nblocks(G.fsz, kThreads);
    int n = 0;
    if (G.eta > 0.0) {
        TIMED(KS_DISSIPATION, s, (k_resist_emf<StoreD><<<nb, kThreads, 0, s>>>(G, U, e0, e1, e2, B.S)));
        TIMED(KS_DISSIPATION, s, (k_ct<StoreD><<<nb, kThreads, 0, s>>>(G, U, e0, e1, e2)));
        n += 2;
    }
    if (G.nu > 0.0) {
        // the velocities go to the primitive-variable buffer, which the next step recomputes
        double *vel = (double *)B.Q;
        TIMED(KS_DISSIPATION, s, (k_visc_vel<StoreD><<<nblocks(G.sv, kThreads), kThreads, 0, s>>>(G, U, vel)));
        TIMED(KS_DISSIPATION, s, (k_visc_flux<StoreD><<<nb, kThreads, 0, s>>>(G, U, vel, f0, f1, f2, B.S)));
        TIMED(KS_DISSIPATION, s, (k_visc_update<StoreD><<<nb, kThreads, 0, s>>>(G, U, f0, f1, f2)));
        n += 3;
    }
    return n + launch_boundary(G, B, cur, s);
}

__global__ void k_history_1d(Geo G, const double *__restrict__ U, double *__restrict__ out) {
    // do ipos = 1, nx: exit at the first x(ipos) >= 1/2 (the loop's exit value nx+1 if none)
    int ipos = 1;
    for (ipos = 1; ipos <= G.nx; ipos++)
        if (G.xc(ipos) >= 0.5) break;
    const long long c = G.idx(ipos, 1, 1);
    out[0] = ld(U + c);
    out[1] = ld(U + G.sv * IU + c);
    out[2] = ld(U + G.sv * IP + c);
    for (int q = 3; q < 9; q++) out[q] = 0.0;
}

int launch_history_1d(const Geo &G, const double *U, double *out, cudaStream_t s) {
    TIMED(KS_HISTORY, s, (k_history_1d<<<1, 1, 0, s>>>(G, U, out)));
    return 1;
}

int launch_history(const Geo &G, const Bufs &B, int cur, cudaStream_t s, int variant) {
    return launch_history_ptrs(G, (const double *)B.U[cur], B.part, B.hist, s, variant);
}

int launch_history_columns(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    TIMED(KS_HISTORY, s, (k_hist_yzmean<StoreD><<<G.nx, 256, 0, s>>>(G, st(B, cur), B.part, 1)));
    return 1;
}

int launch_history_share(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreD S = st(B, cur);
    TIMED(KS_HISTORY, s, (k_hist_sums<StoreD><<<kHistBlocks, 256, 0, s>>>(G, S, B.part, B.part + 2 * G.nx)));
    TIMED(KS_HISTORY, s, (k_hist_final<<<1, 32, 0, s>>>(G, B.part + 2 * G.nx, kHistBlocks, B.hist)));
    return 2;
}

#include "debug_bounds.cuh"

}  // namespace f64
}  // namespace dg
