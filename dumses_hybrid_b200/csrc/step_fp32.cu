// FP32 mixed path: the step kernels of step_impl.cuh instantiated for T = float on a
// compensated FP32 (hi, lo) state, compiled with fast FP32 math.
//
// FP64 is used only where it carries accuracy: the gas pressure from the total
// energy (which cancels in low-beta zones), the minimum of the CFL time steps, the
// orbital-advection shift of each x column and the history sums.  Signal speeds,
// trace, Riemann solvers, fluxes, EMFs, FARGO's remap and the constrained-transport
// increments are FP32; every update adds an FP32 increment to a (hi, lo) pair with
// an error-free two-sum, so the state carries about 48 significant bits across steps.
#define DG_NS f32
#include "step_impl.cuh"
#include "nn_features.cuh"
#include "nn_umma.cuh"

namespace dg {
namespace f32 {
namespace {

__device__ __forceinline__ void apply(const StoreHL &U, const StoreHL &Un, const Geo &G, int v, long long c, float inc) {
    float h = U.hi[G.sv * v + c], l = U.lo[G.sv * v + c];
    add_hl(h, l, inc);
    Un.hi[G.sv * v + c] = h;
    Un.lo[G.sv * v + c] = l;
}
// the same on a pair loaded beforehand: a kernel loads every pair it updates before its
// first store, since the compiler cannot move a load of U across a store to Un
__device__ __forceinline__ void put(const StoreHL &Un, const Geo &G, int v, long long c, float h, float l, float inc) {
    if (!chk(Un.hi + G.sv * v + c, 4) || !chk(Un.lo + G.sv * v + c, 4)) return;
    add_hl(h, l, inc);
    Un.hi[G.sv * v + c] = h;
    Un.lo[G.sv * v + c] = l;
}

// update + constrained_transport (scheme.f90:1764-1993) as FP32 increments on the compensated state
// 10 resident blocks (48 registers): timed best at 256^3 against 12 (40, with spills), 8 and 6
#ifndef DG_UPDATE_MINB32
#define DG_UPDATE_MINB32 10
#endif
__global__ void __launch_bounds__(kThreads, DG_UPDATE_MINB32) k_update3d_hl(Geo G, StoreHL U, StoreHL Un, const float *__restrict__ fx,
                                                          const float *__restrict__ fy, const float *__restrict__ fz,
                                                          const float *__restrict__ ex, const float *__restrict__ ey,
                                                          const float *__restrict__ ez, const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    int i, j, k;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    const long long fxy = (long long)G.FX * G.FY;  // face index steps: +1 (x), +FX (y), +fxy (z)
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const double dtd = S->dt;
    const float dt = (float)dtd;
    const long long c = G.idx(i, j, k);
    const bool shear = G.shearing != 0;
    ShearRemap sr{0.0, 0};
    if (shear) sr = ShearRemap{S->sh_epsi, S->sh_jp};  // time + dt/2, from k_shear_offset
    // the 8 pairs of the cell (c lies inside the ghosted grid for every face cell)
    float uh[8], ul[8];
#pragma unroll
    for (int v = 0; v < 8; v++) {
        uh[v] = ld(U.hi + G.sv * v + c);
        ul[v] = ld(U.lo + G.sv * v + c);
    }

    if (i <= nx && j <= ny && k <= nz) {
        const float dvloc = (float)G.dvloc;
        const float Om = (float)G.omega0;
        float dr = 0.f, du = 0.f, dv = 0.f, dw = 0.f, dp = 0.f;
        float opl = 1.f;
        if (G.omega0 > 0.0) {
            // Crank-Nicolson Coriolis, ratio - 1 = -2 lambda / (1 + lambda)
            const double lam = 0.25 * (G.omega0 * dtd) * (G.omega0 * dtd);
            opl = (float)(1.0 + lam);
            const float rm1 = (float)(-2.0 * lam / (1.0 + lam));
            const float uu = uh[IU], uv = uh[IV];
            du += uu * rm1 + 2.f * Om * dt * uv / opl;
            dv += uv * rm1 - 0.5f * Om * dt * uu / opl;
        }
        const long long FR[3] = {(t + 1), (t + G.FX), (t + fxy)};
        const float *FA[3] = {fx, fy, fz};
        const float ds[3] = {(float)(G.dy * G.dz), (float)(G.dx * G.dz), (float)(G.dx * G.dy)};
        float pre[3];
        for (int d = 0; d < 3; d++) {
            float L[6], R[6];
            load6(FA[d] + t * kFluxRec3, L);
            load6(FA[d] + FR[d] * kFluxRec3, R);
            float rl = L[0], rr = R[0];
            if (d == 0 && shear) {
                if (i == 1) rl = shear_avg(G, sr, fx, kFluxRec3, 0, j, k);
                if (i == nx) rr = shear_avg(G, sr, fx, kFluxRec3, 1, j, k);
            }
            pre[d] = -(R[5] * ds[d] - L[5] * ds[d]) * dt;
            dr += (rl - rr) * dvloc;
            dw += (L[4] - R[4]) * dvloc;
            dp += (L[1] - R[1]) * dvloc;
            if (G.omega0 > 0.0) {
                float dfn2 = (L[2] - R[2]) * dvloc;
                if (d == 0) dfn2 = dfn2 + pre[0] * dvloc;
                float dfn3 = (L[3] - R[3]) * dvloc;
                if (d == 1) dfn3 = dfn3 + pre[1] * dvloc;
                du += dfn2 / opl + Om * dt / opl * dfn3;
                dv += dfn3 / opl - 0.25f * Om * dt / opl * dfn2;
            } else {
                du += (L[2] - R[2]) * dvloc;
                dv += (L[3] - R[3]) * dvloc;
            }
        }
        if (G.omega0 == 0.0) {
            du += pre[0] * dvloc;
            dv += pre[1] * dvloc;
        }
        dw += pre[2] * dvloc;
        put(Un, G, IR, c, uh[IR], ul[IR], dr);
        put(Un, G, IU, c, uh[IU], ul[IU], du);
        put(Un, G, IV, c, uh[IV], ul[IV], dv);
        put(Un, G, IW, c, uh[IW], ul[IW], dw);
        put(Un, G, IP, c, uh[IP], ul[IP], dp);
    }
    auto EYc = [&](int ii, int jj, int kk) -> float {
        if (shear && (ii == 1 || ii == nx + 1) && jj <= ny && kk <= nz + 1)
            return shear_avg(G, sr, ey, 1, ii == 1 ? 0 : 1, jj, kk);
        return ld(ey + G.fidx(ii, jj, kk));
    };
    const float rdx = (float)G.rdx, rdy = (float)G.rdy, rdz = (float)G.rdz;
    const bool ct = G.ndim_act > 1;
    if (j <= ny && k <= nz) {
        float inc = 0.f;
        if (ct) inc = (ld(ez + (t + G.FX)) - ld(ez + t)) * rdy - (EYc(i, j, k + 1) - EYc(i, j, k)) * rdz;
        put(Un, G, IA, c, uh[IA], ul[IA], inc);
    }
    if (i <= nx && k <= nz) {
        float inc = 0.f;
        if (ct) inc = -(ld(ez + (t + 1)) - ld(ez + t)) * rdx + (ld(ex + (t + fxy)) - ld(ex + t)) * rdz;
        put(Un, G, IB, c, uh[IB], ul[IB], inc);
    }
    if (i <= nx && j <= ny) {
        float inc = 0.f;
        if (ct) inc = (EYc(i + 1, j, k) - EYc(i, j, k)) * rdx - (ld(ex + (t + G.FX)) - ld(ex + t)) * rdy;
        put(Un, G, IC, c, uh[IC], ul[IC], inc);
    }
}

__global__ void __launch_bounds__(kThreads) k_update2d_hl(Geo G, StoreHL U, StoreHL Un, const float *__restrict__ fx,
                                                          const float *__restrict__ fy, const float *__restrict__ ez,
                                                          const Scalars *S) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= G.fsz) return;
    const int j = (int)fdiv((unsigned)t, G.dFX) + 1;
    const int i = (int)((unsigned)t - (unsigned)(j - 1) * G.dFX.d) + 1;
    const int k = 1;
    const int nx = G.nx, ny = G.ny;
    const double dtd = S->dt;
    const float dt = (float)dtd;
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
            float L[8], R[8];
            load8(FA[d] + t * kFluxRec2, L);
            load8(FA[d] + FR[d] * kFluxRec2, R);
            pre[d] = -(R[5] * ds[d] - L[5] * ds[d]) * dt;
            dr += (L[0] - R[0]) * dvloc;
            dw += (L[4] - R[4]) * dvloc;
            dp += (L[1] - R[1]) * dvloc;
            dc += (L[6] - R[6]) * dvloc;
            if (G.omega0 > 0.0) {
                float dfn2 = (L[2] - R[2]) * dvloc;
                if (d == 0) dfn2 = dfn2 + pre[0] * dvloc;
                float dfn3 = (L[3] - R[3]) * dvloc;
                if (d == 1) dfn3 = dfn3 + pre[1] * dvloc;
                du += dfn2 / opl + Om * dt / opl * dfn3;
                dv += dfn3 / opl - 0.25f * Om * dt / opl * dfn2;
            } else {
                du += (L[2] - R[2]) * dvloc;
                dv += (L[3] - R[3]) * dvloc;
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

// primitive variables (scheme.f90:44-86) of one cell from the compensated state,
// without the rotation half-kick: velocities and cell-centred B in FP32, the pressure
// in FP64 as (gamma-1) (E - emag - rho eken), which is (gamma-1) rho eint of the
// reference without its division when rho >= smallr
__device__ __forceinline__ void prim_hl(const Geo &G, const StoreHL &U, long long c, float q[8]) {
    auto f = [&](int v, long long cc) { return ld(U.hi + G.sv * v + cc) + ld(U.lo + G.sv * v + cc); };
    const double d = (double)ld(U.hi + G.sv * IR + c) + (double)ld(U.lo + G.sv * IR + c);
    const float ri = 1.0f / (float)d;
    q[IR] = (float)mx(d, kSmallr);
    q[IU] = f(IU, c) * ri;
    q[IV] = f(IV, c) * ri;
    q[IW] = f(IW, c) * ri;
    q[IA] = 0.5f * (f(IA, c) + f(IA, c + 1));
    q[IB] = 0.5f * (f(IB, c) + f(IB, c + G.sy));
    q[IC] = 0.5f * (f(IC, c) + ((G.ndim == 3) ? f(IC, c + G.sz) : f(8, c)));
    if (G.iso) {
        q[IP] = (float)(d * (G.ciso * G.ciso));
    } else {
        const double E = (double)ld(U.hi + G.sv * IP + c) + (double)ld(U.lo + G.sv * IP + c);
        const double emag = 0.5 * ((double)q[IA] * q[IA] + (double)q[IB] * q[IB] + (double)q[IC] * q[IC]);
        const double eken = 0.5 * ((double)q[IU] * q[IU] + (double)q[IV] * q[IV] + (double)q[IW] * q[IW]);
        double pe = (G.gamma - 1.0) * (E - emag - d * eken);
        if (d < kSmallr) pe = pe * (kSmallr / d);
        q[IP] = (float)mx(pe, G.smallp);
    }
}

__global__ void __launch_bounds__(kThreads) k_prim_hl(Geo G, StoreHL U, float *__restrict__ Q, const Scalars *S) {
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
    float q[8];
    prim_hl(G, U, c, q);
    if (G.omega0 > 0.0) {  // rotation half-kick, scheme.f90:78-85
        const float om = (float)G.omega0, hdt = 0.5f * (float)S->dt;
        const float dvx = 2.0f * om * q[IV], dvy = -(0.5f * om * q[IU]);
        q[IU] = q[IU] + dvx * hdt;
        q[IV] = q[IV] + dvy * hdt;
    }
#pragma unroll
    for (int v = 0; v < 8; v++) Q[G.sv * v + c] = q[v];
}

// compute_dt fused with the primitive variables of the next godunov: one pass over the
// ghosted grid writes Q without the rotation half-kick (prim_hl) and reduces the CFL time
// step over the active cells (FP32 signal speeds from prim_hl, the minimum of the per-cell
// time steps taken on their bit patterns); k_kick adds the half-kick once dt is known
__global__ void __launch_bounds__(kThreads) k_prim_dt_hl(Geo G, StoreHL U, float *__restrict__ Q, Scalars *S) {
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    const long long n = (long long)ni * nj * nk;
    const float gamma = (float)G.gamma;
    const float rdx = (float)G.rdx, rdy = (float)G.rdy, rdz = (float)G.rdz;
    const float vsh = ((G.omega0 > 0.0) && !G.fargo) ? (float)(1.5 * G.omega0 * (G.xmax - G.xmin) * 0.5) : 0.0f;
    float best = __int_as_float(0x7f800000);  // +inf
    int bad = 0;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) {
        int i, j, k;
        split3((unsigned)t, G.dPX, G.dPY, i, j, k);
        i -= 2;
        j = (G.ndim > 1) ? j - 2 : 1;
        k = (G.ndim == 3) ? k - 2 : 1;
        const long long c = G.idx(i, j, k);
        float q[8];
        prim_hl(G, U, c, q);
#pragma unroll
        for (int v = 0; v < 8; v++) Q[G.sv * v + c] = q[v];
        if (i >= 1 && i <= G.nx && j >= 1 && j <= G.ny && k >= 1 && k <= G.nz) {
            const float ir = 1.0f / q[IR];
            float sum = 0.0f;
            if (G.nx != 1) sum += (cfast_r(gamma, q[IP], ir, q[IA], q[IB], q[IC]) + fabsf(q[IU])) * rdx;
            if (G.ny != 1) sum += (cfast_r(gamma, q[IP], ir, q[IB], q[IC], q[IA]) + fabsf(q[IV]) + vsh) * rdy;
            if (G.ndim == 3 && G.nz != 1) sum += (cfast_r(gamma, q[IP], ir, q[IC], q[IA], q[IB]) + fabsf(q[IW])) * rdz;
            const float cdt = 1.0f / sum;
            if (!(cdt > 0.0f)) bad = 1;  // NaN or non-positive
            else best = fminf(best, cdt);
        }
    }
    unsigned long long b = (unsigned long long)__double_as_longlong((double)best);
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

// rotation half-kick (scheme.f90:78-85) on the primitive velocities of the ghosted grid:
// one thread per element of the velocity planes, the never-read outer ghost layer included,
// so no cell index is decomposed
__global__ void __launch_bounds__(kThreads) k_kick(Geo G, float *__restrict__ Q, const Scalars *S) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= G.sv) return;
    const float om = (float)G.omega0, hdt = 0.5f * (float)S->dt;
    const float u = Q[G.sv * IU + c], v = Q[G.sv * IV + c];
    const float dvx = 2.0f * om * v, dvy = -(0.5f * om * u);
    Q[G.sv * IU + c] = u + dvx * hdt;
    Q[G.sv * IV + c] = v + dvy * hdt;
}

// ---------------------------------------------------------------------------
// FARGO (fargo.f90:17-288) on the compensated state: the shift of each x column is
// computed in FP64 exactly as in the FP64 path; the remapped value is written as the
// donor cell's (hi, lo) plus an FP32 increment, and the face-B CT as FP32 increments.
// ---------------------------------------------------------------------------
struct HL {
    float h, l;
};
__device__ __forceinline__ HL hl_at(const Geo &G, const StoreHL &U, int v, long long c) {
    return HL{ld(U.hi + G.sv * v + c), ld(U.lo + G.sv * v + c)};
}
// a - b from two (hi, lo) pairs; the hi difference is exact for nearby values
__device__ __forceinline__ float hl_diff(HL a, HL b) { return (a.h - b.h) + (a.l - b.l); }

// uin_slope (fargo.f90:266-280) from the (hi, lo) values at j-1, j, j+1, on differences
__device__ __forceinline__ float slope_hl(int ist, HL m, HL c, HL p) {
    if (ist == 0) return 0.0f;
    const float sl = (float)ist;
    const float dlft = sl * hl_diff(c, m), drgt = sl * hl_diff(p, c);
    const float dcen = 0.5f * (dlft + drgt) / sl;
    const float dlim = (dlft * drgt <= 0.0f) ? 0.0f : fminf(fabsf(dlft), fabsf(drgt));
    return copysignf(fminf(dlim, fabsf(dcen)), dcen);
}
// emfx (i in 1..nx, k in 1..nz+1) and emfz (i in 1..nx+1, k in 1..nz) over j in 1..ny+1,
// along y lines as the FP64 kernel does (shift once per column, sliding donor window)
__global__ void __launch_bounds__(kThreads) k_fargo_emf_hl(Geo G, StoreHL U, float *__restrict__ fex,
                                                           float *__restrict__ fez, const Scalars *S) {
    FargoLine L;
    if (!fargo_line(G, blockIdx.x * (long long)blockDim.x + threadIdx.x, L)) return;
    const int i = L.i, k = L.k;
    const double dt = S->dt;
    const float dy = (float)G.dy;
    const int ny = G.ny, ist = mn(G.slope_type, 2);
    const int kw = fargo_zplane(G, k);
    // the sum over the shifted-through cells and the fractional donor (get_emfx / get_emfz)
    auto line = [&](int v, float sgn, const FargoShift &f, float *out) {
        auto A = [&](int jj) { return hl_at(G, U, v, G.idx(i, jj, kw)); };
        const float eps = (float)f.eps;
        int js = fargo_src(f, L.jb, ny);
        HL w0 = A(js - 1 < 1 ? js - 1 + ny : js - 1), w1 = A(js), w2 = A(next_row(js, ny));
        for (int j = L.jb; j <= L.je; j++) {
            if (j > L.jb) {  // slide by one row
                js = next_row(js, ny);
                w0 = w1;
                w1 = w2;
                w2 = A(next_row(js, ny));
            }
            float e = 0.0f;
            if (f.vK > 0.0) {
                const float lambda = 0.5f * eps * (1.0f - eps);
                for (int jj = 1; jj <= f.nshft; jj++) {
                    int jr = j - jj;
                    if (jr < 1) jr = jr + ny;
                    const HL b = A(wrap1(jr, ny));
                    e += (b.h + b.l) * dy;
                }
                e += (eps * (w1.h + w1.l) + lambda * slope_hl(ist, w0, w1, w2)) * dy;
            } else {
                const float lambda = 0.5f * eps * (eps - 1.0f);
                for (int jj = 0; jj <= f.nshft - 1; jj++) {
                    int jr = j + jj;
                    if (jr > ny) jr = jr - ny;
                    const HL b = A(wrap1(jr, ny));
                    e -= (b.h + b.l) * dy;
                }
                e += (-eps * (w1.h + w1.l) - lambda * slope_hl(ist, w0, w1, w2)) * dy;
            }
            out[G.fidx(i, j, k)] = sgn * e;
        }
    };
    if (i <= G.nx) line(IC, 1.0f, fargo_shift(G, G.xc(i), dt), fex);                         // fargo.f90:146-177
    if (k <= G.nz) line(IA, -1.0f, fargo_shift(G, 0.5 * (G.xc(i) + G.xc(i - 1)), dt), fez);  // fargo.f90:204-235
}

// remap of rho, rho v, E (fargo.f90:59-93) and CT of the face B (fargo.f90:100-119), along
// y lines as the FP64 kernel does (one thread per face column and segment). Every value a
// row needs is loaded before the row's stores: the donor window of a whole segment per
// variable, and the face B and EMFs of kFargoChunk rows at a time for the CT part.
// 3 resident blocks (168 registers): the window stays in registers; timed best at 256^3
#ifndef DG_FARGO_MINB32
#define DG_FARGO_MINB32 3
#endif
__global__ void __launch_bounds__(kThreads, DG_FARGO_MINB32) k_fargo_update_hl(Geo G, StoreHL U, StoreHL Un,
                                                              const float *__restrict__ fex,
                                                              const float *__restrict__ fez, const Scalars *S) {
    FargoLine L;
    if (!fargo_line(G, blockIdx.x * (long long)blockDim.x + threadIdx.x, L)) return;
    const int i = L.i, k = L.k;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    if (i <= nx && k <= nz && L.jb <= ny) {
        const FargoShift f = fargo_shift(G, G.xc(i), S->dt);
        const float eps = (float)f.eps;
        const float w = (f.vK > 0.0) ? 1.0f - eps : eps;  // weight of the upper donor
        const float hme = 0.5f - eps;
        const float q = 0.5f * (0.25f - hme * hme);
        const int ist = mn(G.slope_type, 2);
        const int js = fargo_src(f, L.jb, ny);
        const int j0 = js - 1 < 1 ? js - 1 + ny : js - 1;  // the window starts one row below the first donor
        for (int v = IR; v <= IP; v++) {
            // rows js-1 .. js+kFargoSeg+1 (periodic y); rows past the segment's end are loaded but unused
            HL wn[kFargoSeg + 3];
            int row = j0;
#pragma unroll
            for (int m = 0; m < kFargoSeg + 3; m++) {
                wn[m] = hl_at(G, U, v, G.idx(i, row, k));
                row = next_row(row, ny);
            }
            float s0 = slope_hl(ist, wn[0], wn[1], wn[2]);
#pragma unroll
            for (int m = 0; m < kFargoSeg; m++) {
                const int j = L.jb + m;
                if (j > L.je || j > ny) break;
                const float s1 = slope_hl(ist, wn[m + 1], wn[m + 2], wn[m + 3]);
                HL a0 = wn[m + 1];
                add_hl(a0.h, a0.l, hl_diff(wn[m + 2], wn[m + 1]) * w + (s0 - s1) * q);
                const long long c = G.idx(i, j, k);
                if (!chk(Un.hi + G.sv * v + c, 4) || !chk(Un.lo + G.sv * v + c, 4)) continue;
                Un.hi[G.sv * v + c] = a0.h;
                Un.lo[G.sv * v + c] = a0.l;
                s0 = s1;
            }
        }
    }
    const float rdx = (float)G.rdx, rdy = (float)G.rdy, rdz = (float)G.rdz;
    // face indices clamped into the EMF arrays; a clamped value is never used
    auto EX = [&](int ii, int jj, int kk) { return ld(fex + G.fidx(ii, mn(jj, G.FY), mn(kk, G.FZ))); };
    auto EZ = [&](int ii, int jj, int kk) { return (ii <= nx + 1) ? ld(fez + G.fidx(ii, mn(jj, G.FY), kk)) : 0.0f; };
    for (int jb = L.jb; jb <= L.je; jb += kFargoChunk) {
        HL a[kFargoChunk], b[kFargoChunk], cz[kFargoChunk];
        float ezj[kFargoChunk + 1], exj[kFargoChunk + 1], ezr[kFargoChunk], exu[kFargoChunk];
#pragma unroll
        for (int m = 0; m <= kFargoChunk; m++) {
            ezj[m] = EZ(i, jb + m, k);
            exj[m] = EX(i, jb + m, k);
            if (m < kFargoChunk) {
                const int j = mn(jb + m, L.je);
                const long long c = G.idx(i, j, k);
                a[m] = hl_at(G, U, IA, c);
                b[m] = hl_at(G, U, IB, c);
                cz[m] = hl_at(G, U, IC, c);
                ezr[m] = EZ(i + 1, j, k);
                exu[m] = EX(i, j, k + 1);
            }
        }
#pragma unroll
        for (int m = 0; m < kFargoChunk; m++) {
            const int j = jb + m;
            if (j > L.je) break;
            const long long c = G.idx(i, j, k);
            if (j <= ny && k <= nz) put(Un, G, IA, c, a[m].h, a[m].l, (ezj[m + 1] - ezj[m]) * rdy);
            if (i <= nx && k <= nz)
                put(Un, G, IB, c, b[m].h, b[m].l, -(ezr[m] - ezj[m]) * rdx + (exu[m] - exj[m]) * rdz);
            if (i <= nx && j <= ny) put(Un, G, IC, c, cz[m].h, cz[m].l, -(exj[m + 1] - exj[m]) * rdy);
        }
    }
}

// ---------------------------------------------------------------------------
// learned face flux
// ---------------------------------------------------------------------------
// cells on either side of face (i, j, k) of direction d
__device__ __forceinline__ void face_cells(const Geo &G, int d, int i, int j, int k, long long &cl, long long &cr) {
    cr = G.cidx(i, j, k);
    cl = (d == 0) ? G.cidx(i - 1, j, k) : (d == 1 ? G.cidx(i, j - 1, k) : G.cidx(i, j, k - 1));
}

// interfaces of direction d in harvest order: x fastest over the faces of that direction
__host__ __device__ __forceinline__ void harvest_extent(const Geo &G, int d, int &ex, int &ey, int &ez) {
    ex = G.nx + (d == 0);
    ey = G.ny + (d == 1);
    ez = (G.ndim == 3) ? G.nz + (d == 2) : 1;
}

__global__ void __launch_bounds__(kThreads) k_nn_harvest(Geo G, const float *__restrict__ core, int d, int stride,
                                                         float *__restrict__ xs, float *__restrict__ ts,
                                                         long long first, long long count) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= count) return;
    int ex, ey, ez;
    harvest_extent(G, d, ex, ey, ez);
    const long long idx = s * stride;
    const int i = (int)(idx % ex) + 1;
    const long long r = idx / ex;
    const int j = (int)(r % ey) + 1, k = (int)(r / ey) + 1;
    const CoreView<float> cv{core, G.ndim == 3 ? kCore3 : kCore2};
    long long cl, cr;
    face_cells(G, d, i, j, k, cl, cr);
    float ql[8], qr[8], x[nn::kIn];
    face_io(G, cv, cl, cr, d, ql, qr);
    const float gamma = (float)G.gamma, ciso = (float)G.ciso;
    const nn::FaceUnits u = nn::face_inputs(ql, qr, gamma, ciso, G.iso, x);
    double qld[8], qrd[8], t[nn::kOut], b[nn::kOut];
#pragma unroll
    for (int n = 0; n < 8; n++) { qld[n] = ql[n]; qrd[n] = qr[n]; }
    nn::hlld_targets(qld, qrd, G.gamma, G.ciso, G.iso, t);
    double dis[nn::kOut];
    nn::base_fluxes<double>(qld, qrd, G.gamma, G.ciso, G.iso, b, dis);
    float *xo = xs + (first + s) * nn::kIn;
    float *to = ts + (first + s) * nn::kOut;
#pragma unroll
    for (int n = 0; n < nn::kIn; n++) xo[n] = x[n];
#pragma unroll
    for (int n = 0; n < nn::kOut; n++)
        to[n] = (u.jump > nn::kTinyJump) ? (float)((t[n] - b[n]) / ((double)nn::out_scale(u, n) * (double)u.jump)) : 0.0f;
}

// shared-memory plan of the face-network kernel (bytes): the kNL weight tiles, the kNHid
// hidden-layer bias operands and the all-ones A operand they are multiplied by, then per
// warpgroup one activation tile (its first 8 KB hold the input tile of layer 1), the output
// layer's biases and the barriers
// warpgroups per CTA, each with kHid TMEM columns (a build option, DG_NN_WG; the whole
// register file is shared between them, one CTA per SM): eight up to width 64 (64 registers,
// with some spills: still faster than six at 80 or five at 94), four at width 128 (the tensor
// memory's 512 columns)
#ifndef DG_NN_WG
#define DG_NN_WG (DG_NN_WIDTH > 64 ? 4 : 8)
#endif
constexpr int kNWG = DG_NN_WG;
constexpr int kNTmemUsed = kNWG * nn::kHid;
constexpr int kNTmem = kNTmemUsed <= 32 ? 32 : kNTmemUsed <= 64 ? 64 : kNTmemUsed <= 128 ? 128
                     : kNTmemUsed <= 256 ? 256 : 512;  // an allocation is a power of two from 32 to 512
static_assert(kNTmemUsed <= 512 && kNWG >= 1 && kNWG <= 8, "warpgroups x width exceeds tensor memory");
constexpr int kNBtsz = nn::kBiasK * nn::kHid * 2;
// bytes of the weight tile of layer l: [K_l / 8][N_l][8] BF16
__host__ __device__ constexpr int net_wbytes(int l) {
    return (l == 0 ? nn::kInPad : nn::kHid) * (l == nn::kNHid ? nn::kOutPad : nn::kHid) * 2;
}
__host__ __device__ constexpr int net_woff(int l) { return l == 0 ? 0 : net_woff(l - 1) + net_wbytes(l - 1); }
// per warpgroup a staging area for the trace-core values of its next tile (kNStF per face,
// [value][face] floats), when it fits beside the rest (width 64 with up to six warpgroups; not
// in the checked build)
constexpr int kNStF = 30, kNStsz = kNStF * 128 * 4;
#ifdef DG_CHECK_BOUNDS
constexpr bool kNChecked = true;
#else
constexpr bool kNChecked = false;
#endif
constexpr int kNBt = net_woff(nn::kNL), kNOne = kNBt + nn::kNHid * kNBtsz, kNH0 = kNOne + nn::kBiasK * 128 * 2,
              kNHsz = 128 * nn::kHid * 2, kNSt0 = kNH0 + kNWG * kNHsz;
#ifndef DG_NN_STAGE
#define DG_NN_STAGE 1
#endif
constexpr bool kNStage = DG_NN_STAGE && !kNChecked && kNSt0 + kNWG * kNStsz + 192 <= 232448;
constexpr int kNBias = kNSt0 + (kNStage ? kNWG * kNStsz : 0), kNBar = kNBias + 64, kNSmem = kNBar + 128;
static_assert(kNSmem <= 232448, "face-network kernel exceeds the shared memory of one CTA");

__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory"); }

// element copies (cp.async) of the trace-core values face t of direction d is made of into
// this thread's column of a staging area: the 15 face_fields of its minus-side cell, then
// those of its plus-side cell.  Invalid faces copy nothing.
__device__ __forceinline__ void stage_face(const Geo &G, const float *__restrict__ core, int nf, int d, long long t,
                                           float *st) {
    if (t >= G.fsz) return;
    int i, j, k;
    split3((unsigned)t, G.dFX, G.dFY, i, j, k);
    i++; j++; k++;
    const bool valid = (d == 0) ? (j <= G.ny && (G.ndim == 2 || k <= G.nz))
                     : (d == 1) ? (i <= G.nx && (G.ndim == 2 || k <= G.nz)) : (i <= G.nx && j <= G.ny);
    if (!valid) return;
    long long c[2];
    face_cells(G, d, i, j, k, c[0], c[1]);
#pragma unroll
    for (int side = 0; side < 2; side++) {
        int f[15];
        face_fields(d, side == 0 ? +1 : -1, G.ndim, f);
        const float *src = core + core_base(c[side], nf);
#pragma unroll
        for (int q = 0; q < 15; q++) {
            const unsigned a = (unsigned)__cvta_generic_to_shared(st + (side * 15 + q) * 128);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(src + f[q] * kCoreLane) : "memory");
        }
    }
}

// Four warpgroups per CTA, each taking 128-face tiles in turn: the faces' interface states,
// inputs and gates, the kNL layers as tcgen05 MMAs (weights resident in shared memory,
// each warpgroup with its own kHid TMEM columns; a hidden layer's bias enters its accumulator
// as one more K step, activations go through TMEM -> SmeLU -> shared memory), then the gated
// flux or a mark for HLLD.
__global__ void __launch_bounds__(128 * kNWG, 1) k_nn_faces(Geo G, const float *__restrict__ core,
                                                            float *__restrict__ flux, int *__restrict__ fallback,
                                                            int d, nn::NetView nv, const Scalars *S,
                                                            unsigned long long *cnt, int *err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    using bf16 = __nv_bfloat16;
    const int tid = threadIdx.x, wg = tid >> 7, wt = tid & 127, warp = tid >> 5, lane = tid & 31;
    // weight tile and bias operand of layer l
    auto W = [&](int l) { return (bf16 *)(sm + net_woff(l)); };
    auto Bt = [&](int l) { return (bf16 *)(sm + kNBt + l * kNBtsz); };
    bf16 *One = (bf16 *)(sm + kNOne);
    bf16 *Hs = (bf16 *)(sm + kNH0 + wg * kNHsz), *Xs = Hs;
    float *stg = (float *)(sm + kNSt0 + wg * kNStsz) + wt;  // this thread's staging column (kNStage)
    float *bias = (float *)(sm + kNBias);  // output layer
    uint64_t *wbar = (uint64_t *)(sm + kNBar);
    uint64_t *mbar = (uint64_t *)(sm + kNBar + 8 + 8 * wg);
    uint32_t *tslot = (uint32_t *)(sm + kNBar + 8 + 8 * kNWG);
    int *flags = (int *)(sm + kNBar + 16 + 8 * kNWG);
    int *flag = flags + wg;
    if (tid == 0) {
        nn::mbar_init(wbar, 1);
        for (int g = 0; g < kNWG; g++) {
            nn::mbar_init((uint64_t *)(sm + kNBar + 8 + 8 * g), 1);
            flags[g] = 1;
        }
        nn::mbar_fence_init();
    }
    if (tid < nn::kOut) bias[tid] = nv.b[nn::kNHid][tid];
    // the A operand of the bias step: columns 0 and 1 of every row are 1
    for (int q = tid; q < nn::kBiasK * 128; q += 128 * kNWG) {
        const int r = q / nn::kBiasK, c = q % nn::kBiasK;
        One[nn::blk_off(r, c, nn::kBiasK, 128)] = __float2bfloat16_rn(c < 2 ? 1.0f : 0.0f);
    }
    nn::fence_async_smem();
    if (warp == 0) nn::tmem_alloc(tslot, kNTmem);
    nn::tc_fence_before();
    __syncthreads();
    nn::tc_fence_after();
    const uint32_t tmem = *tslot + (uint32_t)(wg * nn::kHid);
    const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    if (tid == 0) {
        nn::mbar_expect_tx(wbar, net_woff(nn::kNL) + nn::kNHid * kNBtsz);
#pragma unroll
        for (int l = 0; l < nn::kNL; l++) nn::bulk_g2s(W(l), nv.wt[l], net_wbytes(l), wbar);
#pragma unroll
        for (int l = 0; l < nn::kNHid; l++) nn::bulk_g2s(Bt(l), nv.bt[l], kNBtsz, wbar);
        if (!nn::mbar_wait(wbar, 0)) {
            nn::mbar_wait(wbar, 0);
            for (int g = 0; g < kNWG; g++) flags[g] = 0;
        }
    }
    __syncthreads();
    const CoreView<float> cv{core, G.ndim == 3 ? kCore3 : kCore2};
    const float gamma = (float)G.gamma, ciso = (float)G.ciso;
    const double dt = S->dt;
    unsigned ph = 0;
    unsigned long long nface = 0, nfall = 0;
    const bool weights_ok = *flag != 0;  // set before the block-wide barrier above
    const long long tstride = (long long)kNWG * gridDim.x;
    if constexpr (kNStage) {
        if (weights_ok) stage_face(G, core, cv.nf, d, ((long long)kNWG * blockIdx.x + wg) * 128 + wt, stg);
        cp_commit();
    }
    for (long long tile = (long long)kNWG * blockIdx.x + wg; weights_ok && tile * 128 < G.fsz; tile += tstride) {
        const long long t = tile * 128 + wt;
        int i = 0, j = 0, k = 1;
        bool valid = t < G.fsz;
        if (valid) {
            split3((unsigned)t, G.dFX, G.dFY, i, j, k);
            i++; j++; k++;
            valid = (d == 0) ? (j <= G.ny && (G.ndim == 2 || k <= G.nz))
                  : (d == 1) ? (i <= G.nx && (G.ndim == 2 || k <= G.nz)) : (i <= G.nx && j <= G.ny);
        }
        float ql[8], qr[8], x[nn::kInPad], base[nn::kOut], dis[nn::kOut];
        nn::FaceUnits u{1.0f, 1.0f, 1.0f, 0.0f};
        bool use = false;
#pragma unroll
        for (int n = 0; n < nn::kInPad; n++) x[n] = 0.0f;
        if constexpr (kNStage) cp_wait_all();  // this thread's copies of this tile's values
        if (valid) {
            if constexpr (kNStage) {
                const float smallp = (float)G.smallp;
                float v[15], fm[8], fp[8];
#pragma unroll
                for (int q = 0; q < 15; q++) v[q] = stg[q * 128];
                face_state_v(v, d, +1, smallp, fm);
#pragma unroll
                for (int q = 0; q < 15; q++) v[q] = stg[(15 + q) * 128];
                face_state_v(v, d, -1, smallp, fp);
                face_pair(fm, fp, d, ql, qr);
            } else {
                long long cl, cr;
                face_cells(G, d, i, j, k, cl, cr);
                face_io(G, cv, cl, cr, d, ql, qr);
            }
            u = nn::face_inputs(ql, qr, gamma, ciso, G.iso, x);
            use = nn::gate_inputs(nv.gates, ql, qr, ciso, G.iso, u, x);
            nn::base_fluxes<float>(ql, qr, gamma, ciso, G.iso, base, dis);
        }
        if constexpr (kNStage) {  // the next tile's values, in flight while this tile's layers run
            stage_face(G, core, cv.nf, d, (tile + tstride) * 128 + wt, stg);
            cp_commit();
        }
#pragma unroll
        for (int n = 0; n < nn::kIn; n++) x[n] = use ? (x[n] - nv.sc.xmu[n]) * nv.sc.xisd[n] : 0.0f;
#pragma unroll
        for (int cg = 0; cg < nn::kInPad / 8; cg++) {
            __align__(16) bf16 h[8];
#pragma unroll
            for (int q = 0; q < 8; q++) h[q] = __float2bfloat16_rn(x[cg * 8 + q]);
            *(uint4 *)(Xs + (cg * 128 + wt) * 8) = *(const uint4 *)h;
        }
        nn::fence_async_smem();
        nn::tc_fence_before();  // this warpgroup's TMEM reads of the previous tile come before the next MMA
        wg_sync(wg);
        if (!*flag) break;  // read right after a barrier, so the whole warpgroup agrees
        float y[nn::kOut];
        bool tile_ok = true;
        for (int l = 0; l < nn::kNL; l++) {
            if (wt == 0) {
                nn::tc_fence_after();
                nn::mma_tiles(tmem, l == 0 ? Xs : Hs, W(l), l == nn::kNHid ? nn::kOutPad : nn::kHid,
                              (l == 0 ? nn::kInPad : nn::kHid) / 16, 0);
                if (l < nn::kNHid) nn::mma_extra_step(tmem, One, Bt(l), nn::kHid);  // + bias
                nn::mma_commit(mbar);
            }
            // every thread observes the MMA's completion itself; the warp agrees on the outcome
            bool ok = nn::mbar_wait(mbar, ph & 1);
            if (!ok) {
                nn::mbar_wait(mbar, ph & 1);  // let the MMA finish before this warp moves on
                *flag = 0;
            }
            ok = __all_sync(0xffffffffu, ok);
            tile_ok = tile_ok && ok;
            ph++;
            nn::tc_fence_after();
            if (l < nn::kNHid) {
                if (ok) {
                    // one 32-column chunk at a time (chunks interleaved by the compiler took the
                    // kernel to its 128-register limit, with spills, and 2% more time)
#pragma unroll 1
                    for (int cc = 0; cc < nn::kHid / 32; cc++) {
                        float v[32];
                        nn::tmem_ld32(taddr + cc * 32, v);
#pragma unroll
                        for (int hh = 0; hh < 4; hh++) {
                            const float *w = v + hh * 8;
                            *(uint4 *)(Hs + ((cc * 4 + hh) * 128 + wt) * 8) =
                                make_uint4(nn::smelu2_bf16(w[0], w[1]), nn::smelu2_bf16(w[2], w[3]),
                                           nn::smelu2_bf16(w[4], w[5]), nn::smelu2_bf16(w[6], w[7]));
                        }
                    }
                }
                nn::fence_async_smem();
                nn::tc_fence_before();
                wg_sync(wg);  // the next layer's MMA reads every warp's activations
                nn::tc_fence_after();
                if (!*flag) break;
            } else if (ok) {
                float v[16];
                nn::tmem_ld16(taddr, v);
#pragma unroll
                for (int q = 0; q < nn::kOut; q++) y[q] = (v[q] + bias[q]) * nv.sc.ysd[q];
            }
        }
        if (!tile_ok || !*flag) valid = false;  // a failed tile writes nothing (the error word reports it)
        if (valid) {
            bool acc = use;
            float F[nn::kOut], dn[nn::kOut];
#pragma unroll
            for (int c = 0; c < nn::kOut; c++) {
                acc = acc && fabsf(y[c]) <= 1.5f * nv.gates.ymax;  // confidence: inside the training range
                const float sj = nn::out_scale(u, c) * u.jump;
                F[c] = base[c] + sj * y[c];
                dn[c] = (sj > 0.0f) ? dis[c] / sj : 0.0f;
                acc = acc && isfinite(F[c]);
            }
            acc = acc && F[7] > 0.0f;                      // positive star pressure
            acc = acc && nn::gate_dissipation(y, dn);    // no anti-diffusion, no more than LLF's
            if (acc) {
                float f[8] = {F[0], F[1], F[2] - F[7], 0.0f, F[3], F[4], F[5], F[6]};
                flux_store(G, ql, qr, f, F[7], d, i, dt, flux, t);
            }
            if (!acc) fallback[atomicAdd(&cnt[3 + d], 1ULL)] = (int)t;  // HLLD for this face
            nface++;
            nfall += acc ? 0 : 1;
        }
    }
    if constexpr (kNStage) cp_wait_all();  // no copy into shared memory outlives the loop
    if (!*flag && wt == 0) atomicOr(err, nn::NN_ERR_WAIT);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nface += __shfl_xor_sync(0xffffffffu, nface, o);
        nfall += __shfl_xor_sync(0xffffffffu, nfall, o);
    }
    if (lane == 0) {
        atomicAdd(&cnt[0], nface);
        atomicAdd(&cnt[1], nfall);
    }
    nn::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        nn::tc_fence_after();
        nn::tmem_dealloc(*tslot, kNTmem);
    }
}

// exact HLLD for the faces of direction d that the network sent back
__global__ void __launch_bounds__(kThreads) k_nn_fallback(Geo G, const float *__restrict__ core,
                                                          float *__restrict__ flux, const int *__restrict__ list,
                                                          const unsigned long long *__restrict__ cnt, int d,
                                                          const Scalars *S) {
    const unsigned long long n = cnt[3 + d];
    const CoreView<float> cv{core, G.ndim == 3 ? kCore3 : kCore2};
    const double dt = S->dt;
    for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < n;
         q += (unsigned long long)gridDim.x * blockDim.x) {
        const long long t = list[q];
        int i, j, k;
        split3((unsigned)t, G.dFX, G.dFY, i, j, k);
        i++; j++; k++;
        long long cl, cr;
        face_cells(G, d, i, j, k, cl, cr);
        face_flux(G, cv, cl, cr, d, i, dt, flux, t);
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
    // the primitive variables of godunov come out of the same pass (Q without the half-kick)
    const long long ng = (long long)(G.nx + 5) * ((G.ndim > 1) ? G.ny + 5 : 1) * ((G.ndim == 3) ? G.nz + 5 : 1);
    TIMED(KS_DT, s, (k_prim_dt_hl<<<nblocks(ng, kThreads), kThreads, 0, s>>>(G, st(B, cur), (float *)B.Q, B.S)));
    TIMED(KS_DT, s, (k_dt_final<<<1, 1, 0, s>>>(G, B.S)));
    return 3;
}

// 3D trace as two kernels: cell fields, then face fields
#ifndef DG_TRACE_SPLIT32
#define DG_TRACE_SPLIT32 0
#endif
constexpr bool kTraceSplit32 = DG_TRACE_SPLIT32 != 0;
// 3D trace with its stencil staged in shared memory (k_trace3d_tile)
#ifndef DG_TRACE_TILE32
#define DG_TRACE_TILE32 1
#endif
constexpr bool kTraceTile32 = DG_TRACE_TILE32 != 0;

// 3D Riemann work as two kernels (faces, then edges) instead of one
#ifndef DG_RIEMANN_SPLIT32
#define DG_RIEMANN_SPLIT32 0
#endif
constexpr bool kRiemannSplit32 = DG_RIEMANN_SPLIT32 != 0;

int launch_godunov(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreHL U = st(B, cur), Un = st(B, cur ^ 1);
    float *Q = (float *)B.Q, *core = (float *)B.core;
    float *E0 = (float *)B.E[0], *E1 = (float *)B.E[1], *E2 = (float *)B.E[2];
    float *fx = (float *)B.flx[0], *fy = (float *)B.flx[1], *fz = (float *)B.flx[2];
    float *ex = (float *)B.emf[0], *ey = (float *)B.emf[1], *ez = (float *)B.emf[2];
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    int n = (G.shearing ? 1 : 0) + 4;
    if (!B.q_fresh) {
        TIMED(KS_PRIM, s, (k_prim_hl<<<nblocks((long long)ni * nj * nk, kThreads), kThreads, 0, s>>>(G, U, Q, B.S)));
        n++;
    } else if (G.omega0 > 0.0) {  // Q of this state from launch_dt: add the rotation half-kick
        TIMED(KS_PRIM, s, (k_kick<<<nblocks(G.sv, kThreads), kThreads, 0, s>>>(G, Q, B.S)));
        n++;
    }
    if (G.shearing) TIMED(KS_SCALARS, s, (k_shear_offset<<<1, 1, 0, s>>>(G, B.S, 0.5)));
    int faces = 1;
    if (G.ndim == 3) {
        // the tiled trace computes its edge fields itself
        if (kTraceTile32) n--;
        else TIMED(KS_EFIELD, s, (k_efield3d<float><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2)));
        if (kTraceTile32 && kTraceSplit32) {
            TIMED(KS_TRACE, s, (launch_trace_tile<float, 1>(G, Q, U.hi, core, B.S, s)));
            TIMED(KS_TRACE, s, (launch_trace_tile<float, 2>(G, Q, U.hi, core, B.S, s)));
            n++;
        } else if (kTraceTile32) {
            TIMED(KS_TRACE, s, (launch_trace_tile<float>(G, Q, U.hi, core, B.S, s)));
        } else if (kTraceSplit32) {
            TIMED(KS_TRACE, s, (k_trace3d<float, 1><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2, core, B.S)));
            TIMED(KS_TRACE, s, (k_trace3d<float, 2><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2, core, B.S)));
            n++;
        } else {
            TIMED(KS_TRACE, s, (k_trace3d<float><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2, core, B.S)));
        }
    } else {
        TIMED(KS_EFIELD, s, (k_efield2d<float><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E2)));
        TIMED(KS_TRACE, s, (k_trace2d<float><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E2, core, B.S)));
    }
    float *fl[3] = {fx, fy, fz};
    if (B.net) {
        // the network's faces, with the faces it sends back to HLLD listed per direction
        cudaMemsetAsync(B.nn_count + 3, 0, 3 * sizeof(unsigned long long), s);
        const long long groups = (G.fsz + 128 * kNWG - 1) / (128 * kNWG);
        const unsigned grid = (unsigned)(groups < 148 ? groups : 148);
        for (int d = 0; d < G.ndim; d++) {
            TIMED(KS_NN_FACES, s, (k_nn_faces<<<grid, 128 * kNWG, kNSmem, s>>>(G, core, fl[d], B.fb_list[d], d, *B.net, B.S, B.nn_count, B.nn_err)));
            n++;
        }
        faces = 0;
    }
    if (G.ndim == 3) {
        // HLLD/HLLD (the reference's default and every benchmark) runs kernels without the other solvers
        const bool hlld = G.iriemann == DG_RIEMANN_HLLD && G.iriemann2d == DG_RIEMANN_HLLD;
        const unsigned nb = nblocks(G.fsz, kThreads);
        if (kRiemannSplit32) {
            if (faces) {
                if (hlld) TIMED(KS_RIEMANN, s, (k_faces3d<float, true><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
                else TIMED(KS_RIEMANN, s, (k_faces3d<float, false><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, B.S)));
                n++;
            }
            if (hlld) TIMED(KS_RIEMANN, s, (k_edges3d<float, true><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
            else TIMED(KS_RIEMANN, s, (k_edges3d<float, false><<<nb, kThreads, 0, s>>>(G, core, ex, ey, ez, B.S)));
        } else if (hlld) {
            TIMED(KS_RIEMANN, s, (k_riemann3d<float, true><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, ex, ey, ez, B.S, faces)));
        } else {
            TIMED(KS_RIEMANN, s, (k_riemann3d<float, false><<<nb, kThreads, 0, s>>>(G, core, fx, fy, fz, ex, ey, ez, B.S, faces)));
        }
    } else {
        TIMED(KS_RIEMANN, s, (k_riemann2d<float><<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, core, fx, fy, ez, B.S, faces)));
    }
    if (B.net) {
        for (int d = 0; d < G.ndim; d++) {
            // the list's length is on the device: a grid-stride grid of 16 blocks per SM, above the ~7
            // that stay resident, so that every SM has its full share of the scattered gathers in flight
            TIMED(KS_NN_FALLBACK, s, (k_nn_fallback<<<148 * 16, kThreads, 0, s>>>(G, core, fl[d], B.fb_list[d], B.nn_count, d, B.S)));
            n++;
        }
    }
    if (G.ndim == 3) {
        TIMED(KS_UPDATE, s, (k_update3d_hl<<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, U, Un, fx, fy, fz, ex, ey, ez, B.S)));
    } else {
        TIMED(KS_UPDATE, s, (k_update2d_hl<<<nblocks(G.fsz, kThreads), kThreads, 0, s>>>(G, U, Un, fx, fy, ez, B.S)));
    }
    return n;
}

int launch_trace_only(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreHL U = st(B, cur);
    float *Q = (float *)B.Q, *core = (float *)B.core;
    float *E0 = (float *)B.E[0], *E1 = (float *)B.E[1], *E2 = (float *)B.E[2];
    const int ni = G.nx + 5, nj = (G.ndim > 1) ? G.ny + 5 : 1, nk = (G.ndim == 3) ? G.nz + 5 : 1;
    TIMED(KS_PRIM, s, (k_prim_hl<<<nblocks((long long)ni * nj * nk, kThreads), kThreads, 0, s>>>(G, U, Q, B.S)));
    if (G.ndim == 3) {
        TIMED(KS_EFIELD, s, (k_efield3d<float><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2)));
        TIMED(KS_TRACE, s, (k_trace3d<float><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E0, E1, E2, core, B.S)));
    } else {
        TIMED(KS_EFIELD, s, (k_efield2d<float><<<nblocks(G.esz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E2)));
        TIMED(KS_TRACE, s, (k_trace2d<float><<<nblocks(G.csz, kThreads), kThreads, 0, s>>>(G, Q, U.hi, E2, core, B.S)));
    }
    return 3;
}

const void *nn_faces_kernel() { return (const void *)k_nn_faces; }
int nn_faces_smem() { return kNSmem; }

long long harvest_faces(const Geo &G, int d) {
    int ex, ey, ez;
    harvest_extent(G, d, ex, ey, ez);
    return (long long)ex * ey * ez;
}

int launch_harvest(const Geo &G, const Bufs &B, int d, int stride, float *xs, float *ts, long long first,
                   long long count, cudaStream_t s) {
    TIMED(KS_NN_FACES, s, (k_nn_harvest<<<nblocks(count, kThreads), kThreads, 0, s>>>(G, (const float *)B.core, d, stride, xs, ts, first, count)));
    return 1;
}

int launch_fargo(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    float *fex = (float *)B.femf[0], *fez = (float *)B.femf[1];
    TIMED(KS_FARGO_EMF, s, (k_fargo_emf_hl<<<nblocks(fargo_line_threads(G), kThreads), kThreads, 0, s>>>(G, st(B, cur), fex, fez, B.S)));
    TIMED(KS_FARGO_UPDATE, s, (k_fargo_update_hl<<<nblocks(fargo_line_threads(G), kThreads), kThreads, 0, s>>>(G, st(B, cur), st(B, cur ^ 1), fex, fez, B.S)));
    return 2;
}

int launch_boundary(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    int n = 1;
    if (G.shearing) {
        TIMED(KS_SCALARS, s, (k_shear_offset<<<1, 1, 0, s>>>(G, B.S, 1.0)));
        n++;
    }
    TIMED(KS_BOUNDARY, s, (k_boundary<StoreHL><<<nblocks(ghost_cells(G), kThreads), kThreads, 0, s>>>(G, st(B, cur), B.nv, B.S)));
    return n;
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

// dissipation (physics.f90:272-291): resistive EMFs + CT, viscous fluxes + update, in
// place on U[cur], then boundary; the step's EMF and flux arrays are free at this point
int launch_dissipation(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const StoreHL U = st(B, cur);
    float *e0 = (float *)B.emf[0], *e1 = (float *)B.emf[1], *e2 = (float *)B.emf[2];
    float *f0 = (float *)B.flx[0], *f1 = (float *)B.flx[1], *f2 = G.ndim == 3 ? (float *)B.flx[2] : f0;
    if (G.ndim == 2) e0 = e1 = e2;  // 2D: only emfz is allocated and used
    const unsigned nb = nblocks(G.fsz, kThreads);
    int n = 0;
    if (G.eta > 0.0) {
        TIMED(KS_DISSIPATION, s, (k_resist_emf<StoreHL><<<nb, kThreads, 0, s>>>(G, U, e0, e1, e2, B.S)));
        TIMED(KS_DISSIPATION, s, (k_ct<StoreHL><<<nb, kThreads, 0, s>>>(G, U, e0, e1, e2)));
        n += 2;
    }
    if (G.nu > 0.0) {
        // the velocities go to the primitive-variable buffer, which the next step recomputes
        float *vel = (float *)B.Q;
        TIMED(KS_DISSIPATION, s, (k_visc_vel<StoreHL><<<nblocks(G.sv, kThreads), kThreads, 0, s>>>(G, U, vel)));
        TIMED(KS_DISSIPATION, s, (k_visc_flux<StoreHL><<<nb, kThreads, 0, s>>>(G, U, vel, f0, f1, f2, B.S)));
        TIMED(KS_DISSIPATION, s, (k_visc_update<StoreHL><<<nb, kThreads, 0, s>>>(G, U, f0, f1, f2)));
        n += 3;
    }
    return n + launch_boundary(G, B, cur, s);
}

int launch_history(const Geo &G, const Bufs &B, int cur, cudaStream_t s, int variant) {
    const int nb = 296;
    const int iv2 = variant == DG_HISTORY_DEFAULT ? IW : IV, ib2 = variant == DG_HISTORY_DEFAULT ? IC : IB;
    TIMED(KS_HISTORY, s, (k_hist_yzmean<StoreHL><<<G.nx, 256, 0, s>>>(G, st(B, cur), B.part, 0, iv2)));
    TIMED(KS_HISTORY, s, (k_hist_sums<StoreHL><<<nb, 256, 0, s>>>(G, st(B, cur), B.part, B.part + 2 * G.nx, iv2, ib2)));
    TIMED(KS_HISTORY, s, (k_hist_final<<<1, 32, 0, s>>>(G, B.part + 2 * G.nx, nb, B.hist)));
    return 3;
}

int launch_history_columns(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    TIMED(KS_HISTORY, s, (k_hist_yzmean<StoreHL><<<G.nx, 256, 0, s>>>(G, st(B, cur), B.part, 1)));
    return 1;
}

int launch_history_share(const Geo &G, const Bufs &B, int cur, cudaStream_t s) {
    const int nb = 296;
    TIMED(KS_HISTORY, s, (k_hist_sums<StoreHL><<<nb, 256, 0, s>>>(G, st(B, cur), B.part, B.part + 2 * G.nx)));
    TIMED(KS_HISTORY, s, (k_hist_final<<<1, 32, 0, s>>>(G, B.part + 2 * G.nx, nb, B.hist)));
    return 2;
}

#include "debug_bounds.cuh"

}  // namespace f32
}  // namespace dg
