// Riemann solvers of the MHD step as device functions, templated on the
// arithmetic type T (double for the plain path, float for the mixed path).
//
// 1D interface solvers (face fluxes), src/modules/solvers/solver.f90:
//   llf :393-498, hll :504-612, hlld :618-836, upwind :842-935.
//   State order: 0 rho, 1 P, 2 u_n, 3 B_n, 4 v_t1, 5 B_t1, 6 v_t2, 7 B_t2.
//   HLLD returns the normal-momentum flux without total pressure and the star
//   total pressure p*_T separately (solver.f90:818-833); the other solvers put
//   the pressure in the flux and report p*_T = 0 (pgstar is zeroed, :94-99).
// 2D edge solvers (EMFs), src/modules/solvers/solver_magnetic.f90:
//   llf :241-356, hlld :362-548, upwind :554-600, hlla :688-727.
//   Corner order LL, LR, RL, RR as set by solver_magnetic_utils (:32-49).
#pragma once
#include "dg_common.cuh"

namespace dg {

// the square of the fast magnetosonic speed; the solvers that only need the largest of several
// speeds take one square root of the largest square: sqrt is monotone and correctly rounded, so
// sqrt(max(x)) is max(sqrt(x)) bit for bit (and the ternary max picks the same element either way)
template <typename T>
__device__ __forceinline__ T cfast2(T gamma, T ploc, T rho, T a, T b, T c) {
    const T half = T(0.5);
    T c2 = gamma * ploc / rho;
    T b2 = a * a + b * b + c * c;
    T d2 = half * (c2 + b2 / rho);
    return d2 + sqr(d2 * d2 - c2 * a * a / rho);
}
template <typename T>
__device__ __forceinline__ T cfast(T gamma, T ploc, T rho, T a, T b, T c) {
    return sqr(cfast2(gamma, ploc, rho, a, b, c));
}
// the same from b2 = a^2 + b^2 + c^2 computed by the caller: the x and y speeds of an edge
// corner sum the same three squares in two orders, (A^2 + B^2) + C^2 and (B^2 + A^2) + C^2,
// which are equal (IEEE addition commutes), so one b2 / rho serves both
template <typename T>
__device__ __forceinline__ T cfast2_b2(T gamma, T ploc, T rho, T a, T b2) {
    const T half = T(0.5);
    T c2 = gamma * ploc / rho;
    T d2 = half * (c2 + b2 / rho);
    return d2 + sqr(d2 * d2 - c2 * a * a / rho);
}

// left/right physical fluxes and conserved states shared by llf, hll, upwind
template <typename T>
__device__ __forceinline__ void lr_fluxes(const T *ql, const T *qr, T gamma, T ciso, int iso,
                                          T *fl, T *cl, T *fr, T *cr, T &ploc, T &proc, T &a) {
    const T one = T(1), half = T(0.5);
    const T rl = ql[0], ul = ql[2], vl = ql[4], bl = ql[5], wl = ql[6], clv = ql[7];
    const T rr = qr[0], ur = qr[2], vr = qr[4], br = qr[5], wr = qr[6], crv = qr[7];
    const T entho = one / (gamma - one);
    a = half * (ql[3] + qr[3]);
    const T al = a, ar = a;
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); }
    else { ploc = ql[1]; proc = qr[1]; }
    T ecin = half * (ul * ul + vl * vl + wl * wl) * rl;
    T emag = half * (a * a + bl * bl + clv * clv);
    T etot = ploc * entho + ecin + emag;
    T ptot = ploc + emag;
    fl[0] = rl * ul;
    fl[1] = (etot + ptot) * ul - al * (ul * al + vl * bl + wl * clv);
    fl[2] = rl * ul * ul + ptot - al * al;
    fl[3] = T(0);
    fl[4] = rl * ul * vl - al * bl;
    fl[5] = bl * ul - al * vl;
    fl[6] = rl * ul * wl - al * clv;
    fl[7] = clv * ul - al * wl;
    cl[0] = rl; cl[1] = etot; cl[2] = rl * ul; cl[3] = al; cl[4] = rl * vl; cl[5] = bl; cl[6] = rl * wl; cl[7] = clv;
    ecin = half * (ur * ur + vr * vr + wr * wr) * rr;
    emag = half * (a * a + br * br + crv * crv);
    etot = proc * entho + ecin + emag;
    ptot = proc + emag;
    fr[0] = rr * ur;
    fr[1] = (etot + ptot) * ur - ar * (ur * ar + vr * br + wr * crv);
    fr[2] = rr * ur * ur + ptot - ar * ar;
    fr[3] = T(0);
    fr[4] = rr * ur * vr - ar * br;
    fr[5] = br * ur - ar * vr;
    fr[6] = rr * ur * wr - ar * crv;
    fr[7] = crv * ur - ar * wr;
    cr[0] = rr; cr[1] = etot; cr[2] = rr * ur; cr[3] = ar; cr[4] = rr * vr; cr[5] = br; cr[6] = rr * wr; cr[7] = crv;
}

template <typename T>
__device__ void llf1d(const T *ql, const T *qr, T *f, T gamma, T ciso, int iso) {
    const T half = T(0.5);
    T fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, ploc, proc, a);
    T vleft = cfast(gamma, ploc, ql[0], a, ql[5], ql[7]) + fab(ql[2]);
    T vright = cfast(gamma, proc, qr[0], a, qr[5], qr[7]) + fab(qr[2]);
    T vel_info = mx(vleft, vright);
#pragma unroll
    for (int n = 0; n < 8; n++) f[n] = half * (fl[n] + fr[n]) - vel_info * half * (cr[n] - cl[n]);
}

template <typename T>
__device__ void hll1d(const T *ql, const T *qr, T *f, T gamma, T ciso, int iso) {
    T fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, ploc, proc, a);
    const T cfmax = sqr(mx(cfast2(gamma, ploc, ql[0], a, ql[5], ql[7]), cfast2(gamma, proc, qr[0], a, qr[5], qr[7])));
    T ul = ql[2], ur = qr[2];
    T sl = mn(mn(ul, ur) - cfmax, T(0));
    T sr = mx(mx(ul, ur) + cfmax, T(0));
    if constexpr (sizeof(T) == 4) {
        const T is = T(1) / (sr - sl);
#pragma unroll
        for (int n = 0; n < 8; n++) f[n] = (sr * fl[n] - sl * fr[n] + sr * sl * (cr[n] - cl[n])) * is;
        return;
    }
#pragma unroll
    for (int n = 0; n < 8; n++) f[n] = (sr * fl[n] - sl * fr[n] + sr * sl * (cr[n] - cl[n])) / (sr - sl);
}

template <typename T>
__device__ void upwind1d(const T *ql, const T *qr, T *f, T gamma, T ciso, int iso) {
    const T half = T(0.5);
    T fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, ploc, proc, a);
    T vleft = half * (ql[2] + qr[2]);
#pragma unroll
    for (int n = 0; n < 8; n++) f[n] = half * (fl[n] + fr[n]) - fab(vleft) * half * (cr[n] - cl[n]);
}

// ---------------------------------------------------------------------------
// FP32 forms of the same solvers for the mixed path: identical formulas, with each
// repeated divisor turned into one reciprocal (or reciprocal square root) and the
// fast-speed discriminant clamped at zero against FP32 rounding.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float cfast2_r(float gamma, float p, float irho, float a, float b, float c) {
    const float c2 = gamma * p * irho;
    const float d2 = 0.5f * (c2 + (a * a + b * b + c * c) * irho);
    return d2 + sqrtf(fmaxf(d2 * d2 - c2 * a * a * irho, 0.0f));
}
__device__ __forceinline__ float cfast_r(float gamma, float p, float irho, float a, float b, float c) {
    return sqrtf(cfast2_r(gamma, p, irho, a, b, c));
}

// packed FP32 (sm_100 FADD2 / FMUL2 / FFMA2: two lanes per instruction) for the mirrored
// left / right arithmetic of the solvers: x = left, y = right
__device__ __forceinline__ float2 p2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 s2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

__device__ __forceinline__ void hlld1d_f(const float *ql, const float *qr, float *f, float &pg, float gamma,
                                         float ciso, int iso) {
    const float half = 0.5f, zero = 0.0f;
    const float2 r = p2(ql[0], qr[0]), u = p2(ql[2], qr[2]), v = p2(ql[4], qr[4]), b = p2(ql[5], qr[5]);
    const float2 w = p2(ql[6], qr[6]), c = p2(ql[7], qr[7]);
    const float entho = 1.0f / (gamma - 1.0f);
    const float a = half * (ql[3] + qr[3]);
    const float aa = a * a;
    const float sgnm = copysignf(1.0f, a);
    const float2 p = iso ? mul2(r, s2(ciso * ciso)) : p2(ql[1], qr[1]);
    const float2 bsum = fma2(b, b, fma2(c, c, s2(aa)));  // a^2 + b^2 + c^2
    const float2 emag = mul2(s2(half), bsum);
    const float2 ke = fma2(u, u, fma2(v, v, mul2(w, w)));
    const float2 etot = fma2(p, s2(entho), fma2(mul2(s2(half), ke), r, emag));
    const float2 ptot = add2(p, emag);
    const float2 vdotb = fma2(u, s2(a), fma2(v, b, mul2(w, c)));
    // fast speeds (cfast2_r of each side), one square root of the larger
    const float2 irho = p2(1.0f / r.x, 1.0f / r.y);
    const float2 c2 = mul2(mul2(s2(gamma), p), irho);
    const float2 d2 = mul2(s2(half), fma2(bsum, irho, c2));
    const float2 disc = fma2(neg2(mul2(c2, s2(aa))), irho, mul2(d2, d2));
    const float cf = sqrtf(fmaxf(d2.x + sqrtf(fmaxf(disc.x, 0.0f)), d2.y + sqrtf(fmaxf(disc.y, 0.0f))));
    const float sl = fminf(u.x, u.y) - cf;
    const float sr = fmaxf(u.x, u.y) + cf;
    const float2 S = p2(sl, sr);
    const float2 Su = sub2(S, u);                     // (sl - ul, sr - ur)
    const float2 rSu = mul2(r, Su);
    const float2 rc = mul2(rSu, p2(-1.0f, 1.0f));     // (rl (ul - sl), rr (sr - ur))
    const float irc = 1.0f / (rc.y + rc.x);
    const float ustar = (rc.y * u.y + rc.x * u.x + (ptot.x - ptot.y)) * irc;
    const float ptotstar = (rc.y * ptot.x + rc.x * ptot.y + rc.x * rc.y * (u.x - u.y)) * irc;
    // single-star regions, left (x) and right (y)
    const float2 Sus = sub2(S, s2(ustar));
    const float2 is = p2(1.0f / Sus.x, 1.0f / Sus.y);
    const float2 rstar = mul2(rSu, is);
    const float2 estar = fma2(rSu, Sus, s2(-aa));
    const float2 e = fma2(rSu, Su, s2(-aa));
    const float2 ie = p2(estar.x != zero ? 1.0f / estar.x : zero, estar.y != zero ? 1.0f / estar.y : zero);
    const float2 adu_ie = mul2(mul2(s2(a), sub2(s2(ustar), u)), ie);
    const float2 eie = mul2(e, ie);
    float2 vstar = sub2(v, mul2(b, adu_ie)), wstar = sub2(w, mul2(c, adu_ie));
    float2 bstar = mul2(b, eie), cstar = mul2(c, eie);
    if (estar.x == zero) { vstar.x = v.x; bstar.x = b.x; wstar.x = w.x; cstar.x = c.x; }
    if (estar.y == zero) { vstar.y = v.y; bstar.y = b.y; wstar.y = w.y; cstar.y = c.y; }
    const float2 vdotbstar = fma2(s2(ustar), s2(a), fma2(vstar, bstar, mul2(wstar, cstar)));
    const float2 etotstar = mul2(fma2(Su, etot, fma2(neg2(ptot), u, fma2(s2(ptotstar), s2(ustar),
                                                                            mul2(s2(a), sub2(vdotb, vdotbstar))))), is);
    const float2 rs = p2(rsqrtf(rstar.x), rsqrtf(rstar.y));
    const float2 sqrr = mul2(rstar, rs);
    const float sal = ustar - fabsf(a) * rs.x;
    const float sar = ustar + fabsf(a) * rs.y;
    // double star region
    const float isum = 1.0f / (sqrr.x + sqrr.y);
    const float vstarstar = (sqrr.x * vstar.x + sqrr.y * vstar.y + sgnm * (bstar.y - bstar.x)) * isum;
    const float wstarstar = (sqrr.x * wstar.x + sqrr.y * wstar.y + sgnm * (cstar.y - cstar.x)) * isum;
    const float bstarstar = (sqrr.x * bstar.y + sqrr.y * bstar.x + sgnm * sqrr.x * sqrr.y * (vstar.y - vstar.x)) * isum;
    const float cstarstar = (sqrr.x * cstar.y + sqrr.y * cstar.x + sgnm * sqrr.x * sqrr.y * (wstar.y - wstar.x)) * isum;
    const float vdotbstarstar = ustar * a + vstarstar * bstarstar + wstarstar * cstarstar;
    // sample at x/t = 0
    float ro, uo, vo, wo, bo, co, ptoto, etoto, vdotbo;
    if (sl > zero) {
        ro = r.x; uo = u.x; vo = v.x; wo = w.x; bo = b.x; co = c.x; ptoto = ptot.x; etoto = etot.x; vdotbo = vdotb.x;
    } else if (sal > zero) {
        ro = rstar.x; uo = ustar; vo = vstar.x; wo = wstar.x; bo = bstar.x; co = cstar.x;
        ptoto = ptotstar; etoto = etotstar.x; vdotbo = vdotbstar.x;
    } else if (ustar > zero) {
        ro = rstar.x; uo = ustar; vo = vstarstar; wo = wstarstar; bo = bstarstar; co = cstarstar;
        ptoto = ptotstar; etoto = etotstar.x - sgnm * sqrr.x * (vdotbstar.x - vdotbstarstar); vdotbo = vdotbstarstar;
    } else if (sar > zero) {
        ro = rstar.y; uo = ustar; vo = vstarstar; wo = wstarstar; bo = bstarstar; co = cstarstar;
        ptoto = ptotstar; etoto = etotstar.y + sgnm * sqrr.y * (vdotbstar.y - vdotbstarstar); vdotbo = vdotbstarstar;
    } else if (sr > zero) {
        ro = rstar.y; uo = ustar; vo = vstar.y; wo = wstar.y; bo = bstar.y; co = cstar.y;
        ptoto = ptotstar; etoto = etotstar.y; vdotbo = vdotbstar.y;
    } else {
        ro = r.y; uo = u.y; vo = v.y; wo = w.y; bo = b.y; co = c.y; ptoto = ptot.y; etoto = etot.y; vdotbo = vdotb.y;
    }
    f[0] = ro * uo;
    f[1] = (etoto + ptoto) * uo - a * vdotbo;
    f[2] = ro * uo * uo - a * a;
    f[3] = zero;
    f[4] = ro * uo * vo - a * bo;
    f[5] = bo * uo - a * vo;
    f[6] = ro * uo * wo - a * co;
    f[7] = co * uo - a * wo;
    pg = ptoto;
}

// HLLD; returns p*_T in pg.  entho = 1 / (gamma - 1), the same for every interface of a run
// (formed once per context by the caller; the FP32 form takes its own reciprocal)
template <typename T>
__device__ void hlld1d(const T *ql, const T *qr, T *f, T &pg, T gamma, T ciso, int iso, T entho) {
    if constexpr (sizeof(T) == 4) {
        hlld1d_f(ql, qr, f, pg, gamma, ciso, iso);
        return;
    }
    const T half = T(0.5), zero = T(0);
    const T rl = ql[0], ul = ql[2], vl = ql[4], bl = ql[5], wl = ql[6], cl = ql[7];
    const T rr = qr[0], ur = qr[2], vr = qr[4], br = qr[5], wr = qr[6], cr = qr[7];
    const T a = half * (ql[3] + qr[3]);
    const T sgnm = sgn1(a);
    T ploc, proc;
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); }
    else { ploc = ql[1]; proc = qr[1]; }
    const T ecinl = half * (ul * ul + vl * vl + wl * wl) * rl;
    const T emagl = half * (a * a + bl * bl + cl * cl);
    const T etotl = ploc * entho + ecinl + emagl;
    const T ptotl = ploc + emagl;
    const T vdotbl = ul * a + vl * bl + wl * cl;
    const T ecinr = half * (ur * ur + vr * vr + wr * wr) * rr;
    const T emagr = half * (a * a + br * br + cr * cr);
    const T etotr = proc * entho + ecinr + emagr;
    const T ptotr = proc + emagr;
    const T vdotbr = ur * a + vr * br + wr * cr;
    const T cfmax = sqr(mx(cfast2(gamma, ploc, rl, a, bl, cl), cfast2(gamma, proc, rr, a, br, cr)));
    const T sl = mn(ul, ur) - cfmax;
    const T sr = mx(ul, ur) + cfmax;
    const T rcl = rl * (ul - sl);
    const T rcr = rr * (sr - ur);
    const T ustar = (rcr * ur + rcl * ul + (ptotl - ptotr)) / (rcr + rcl);
    const T ptotstar = (rcr * ptotl + rcl * ptotr + rcl * rcr * (ul - ur)) / (rcr + rcl);
    // left star region
    const T rstarl = rl * (sl - ul) / (sl - ustar);
    T estar = rl * (sl - ul) * (sl - ustar) - a * a;
    const T el = rl * (sl - ul) * (sl - ul) - a * a;
    T vstarl, bstarl, wstarl, cstarl;
    if (estar == zero) { vstarl = vl; bstarl = bl; wstarl = wl; cstarl = cl; }
    else {
        vstarl = vl - a * bl * (ustar - ul) / estar;
        bstarl = bl * el / estar;
        wstarl = wl - a * cl * (ustar - ul) / estar;
        cstarl = cl * el / estar;
    }
    const T vdotbstarl = ustar * a + vstarl * bstarl + wstarl * cstarl;
    const T etotstarl = ((sl - ul) * etotl - ptotl * ul + ptotstar * ustar + a * (vdotbl - vdotbstarl)) / (sl - ustar);
    const T sqrrstarl = sqr(rstarl);
    const T calfvenl = fab(a) / sqrrstarl;
    const T sal = ustar - calfvenl;
    // right star region
    const T rstarr = rr * (sr - ur) / (sr - ustar);
    estar = rr * (sr - ur) * (sr - ustar) - a * a;
    const T er = rr * (sr - ur) * (sr - ur) - a * a;
    T vstarr, bstarr, wstarr, cstarr;
    if (estar == zero) { vstarr = vr; bstarr = br; wstarr = wr; cstarr = cr; }
    else {
        vstarr = vr - a * br * (ustar - ur) / estar;
        bstarr = br * er / estar;
        wstarr = wr - a * cr * (ustar - ur) / estar;
        cstarr = cr * er / estar;
    }
    const T vdotbstarr = ustar * a + vstarr * bstarr + wstarr * cstarr;
    const T etotstarr = ((sr - ur) * etotr - ptotr * ur + ptotstar * ustar + a * (vdotbr - vdotbstarr)) / (sr - ustar);
    const T sqrrstarr = sqr(rstarr);
    const T calfvenr = fab(a) / sqrrstarr;
    const T sar = ustar + calfvenr;
    // double star region
    const T vstarstar = (sqrrstarl * vstarl + sqrrstarr * vstarr + sgnm * (bstarr - bstarl)) / (sqrrstarl + sqrrstarr);
    const T wstarstar = (sqrrstarl * wstarl + sqrrstarr * wstarr + sgnm * (cstarr - cstarl)) / (sqrrstarl + sqrrstarr);
    const T bstarstar = (sqrrstarl * bstarr + sqrrstarr * bstarl + sgnm * sqrrstarl * sqrrstarr * (vstarr - vstarl))
                      / (sqrrstarl + sqrrstarr);
    const T cstarstar = (sqrrstarl * cstarr + sqrrstarr * cstarl + sgnm * sqrrstarl * sqrrstarr * (wstarr - wstarl))
                      / (sqrrstarl + sqrrstarr);
    const T vdotbstarstar = ustar * a + vstarstar * bstarstar + wstarstar * cstarstar;
    const T etotstarstarl = etotstarl - sgnm * sqrrstarl * (vdotbstarl - vdotbstarstar);
    const T etotstarstarr = etotstarr + sgnm * sqrrstarr * (vdotbstarr - vdotbstarstar);
    // sample at x/t = 0
    T ro, uo, vo, wo, bo, co, ptoto, etoto, vdotbo;
    if (sl > zero) {
        ro = rl; uo = ul; vo = vl; wo = wl; bo = bl; co = cl; ptoto = ptotl; etoto = etotl; vdotbo = vdotbl;
    } else if (sal > zero) {
        ro = rstarl; uo = ustar; vo = vstarl; wo = wstarl; bo = bstarl; co = cstarl;
        ptoto = ptotstar; etoto = etotstarl; vdotbo = vdotbstarl;
    } else if (ustar > zero) {
        ro = rstarl; uo = ustar; vo = vstarstar; wo = wstarstar; bo = bstarstar; co = cstarstar;
        ptoto = ptotstar; etoto = etotstarstarl; vdotbo = vdotbstarstar;
    } else if (sar > zero) {
        ro = rstarr; uo = ustar; vo = vstarstar; wo = wstarstar; bo = bstarstar; co = cstarstar;
        ptoto = ptotstar; etoto = etotstarstarr; vdotbo = vdotbstarstar;
    } else if (sr > zero) {
        ro = rstarr; uo = ustar; vo = vstarr; wo = wstarr; bo = bstarr; co = cstarr;
        ptoto = ptotstar; etoto = etotstarr; vdotbo = vdotbstarr;
    } else {
        ro = rr; uo = ur; vo = vr; wo = wr; bo = br; co = cr; ptoto = ptotr; etoto = etotr; vdotbo = vdotbr;
    }
    f[0] = ro * uo;
    f[1] = (etoto + ptoto) * uo - a * vdotbo;
    f[2] = ro * uo * uo - a * a;
    f[3] = zero;
    f[4] = ro * uo * vo - a * bo;
    f[5] = bo * uo - a * vo;
    f[6] = ro * uo * wo - a * co;
    f[7] = co * uo - a * wo;
    pg = ptoto;
}

// the four corner states of an edge after solver_magnetic_utils
template <typename T>
struct Corners {
    T rLL, rLR, rRL, rRR, pLL, pLR, pRL, pRR, uLL, uLR, uRL, uRR;
    T vLL, vLR, vRL, vRR, ALL, ALR, ARL, ARR, BLL, BLR, BRL, BRR;
    T CLL, CLR, CRL, CRR, ELL, ELR, ERL, ERR;
};

template <typename T> __device__ __forceinline__ T mn4(T a, T b, T c, T d) { return mn(mn(mn(a, b), c), d); }
template <typename T> __device__ __forceinline__ T mx4(T a, T b, T c, T d) { return mx(mx(mx(a, b), c), d); }

template <typename T>
__device__ T llf2d(const Corners<T> &c, T dt, T gamma, T ciso, int iso) {
    const T half = T(0.5), forth = T(0.25);
    T E = forth * (c.ELL + c.ERL + c.ELR + c.ERR);
    T rl = half * (c.rLL + c.rLR), pl = half * (c.pLL + c.pLR), ul = half * (c.uLL + c.uLR);
    T al = half * (c.ALL + c.ALR), bl = half * (c.BLL + c.BLR), cl = half * (c.CLL + c.CLR);
    T rr = half * (c.rRR + c.rRL), pr = half * (c.pRR + c.pRL), ur = half * (c.uRR + c.uRL);
    T ar = half * (c.ARR + c.ARL), br = half * (c.BRR + c.BRL), cr = half * (c.CRR + c.CRL);
    T ploc, proc;
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); } else { ploc = pl; proc = pr; }
    al = half * (al + ar); ar = al;
    T vleft = cfast(gamma, ploc, rl, al, bl, cl) + fab(ul);
    T vright = cfast(gamma, proc, rr, ar, br, cr) + fab(ur);
    T vel_info = mx(vleft, vright);
    T flux_x = -vel_info * half * (br - bl);
    rl = half * (c.rLL + c.rRL); pl = half * (c.pLL + c.pRL); ul = half * (c.vLL + c.vRL);
    al = half * (c.BLL + c.BRL); bl = half * (c.ALL + c.ARL); cl = half * (c.CLL + c.CRL);
    rr = half * (c.rRR + c.rLR); pr = half * (c.pRR + c.pLR); ur = half * (c.vRR + c.vLR);
    ar = half * (c.BRR + c.BLR); br = half * (c.ARR + c.ALR); cr = half * (c.CRR + c.CLR);
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); } else { ploc = pl; proc = pr; }
    al = half * (al + ar); ar = al;
    vleft = cfast(gamma, ploc, rl, al, bl, cl) + fab(ul);
    vright = cfast(gamma, proc, rr, ar, br, cr) + fab(ur);
    vel_info = mx(vleft, vright);
    T flux_y = -vel_info * half * (br - bl);
    T emf = E + (flux_x - flux_y);
    return emf * dt;
}

// FP32 form of hlld2d: per corner one reciprocal density shared by the x and y fast
// speeds, reciprocal square roots of the star densities
__device__ __forceinline__ float hlld2d_f(const Corners<float> &c, float dt, float gamma) {
    const float half = 0.5f, zero = 0.0f, smallc = (float)kSmallc;
    const float iLL = 1.0f / c.rLL, iLR = 1.0f / c.rLR, iRL = 1.0f / c.rRL, iRR = 1.0f / c.rRR;
    const float cfx = sqrtf(mx4(cfast2_r(gamma, c.pLL, iLL, c.ALL, c.BLL, c.CLL), cfast2_r(gamma, c.pLR, iLR, c.ALR, c.BLR, c.CLR),
                                cfast2_r(gamma, c.pRL, iRL, c.ARL, c.BRL, c.CRL), cfast2_r(gamma, c.pRR, iRR, c.ARR, c.BRR, c.CRR)));
    const float cfy = sqrtf(mx4(cfast2_r(gamma, c.pLL, iLL, c.BLL, c.ALL, c.CLL), cfast2_r(gamma, c.pLR, iLR, c.BLR, c.ALR, c.CLR),
                                cfast2_r(gamma, c.pRL, iRL, c.BRL, c.ARL, c.CRL), cfast2_r(gamma, c.pRR, iRR, c.BRR, c.ARR, c.CRR)));
    const float SL = mn4(c.uLL, c.uLR, c.uRL, c.uRR) - cfx;
    const float SR = mx4(c.uLL, c.uLR, c.uRL, c.uRR) + cfx;
    const float SB = mn4(c.vLL, c.vLR, c.vRL, c.vRR) - cfy;
    const float ST = mx4(c.vLL, c.vLR, c.vRL, c.vRR) + cfy;
    const float PtotLL = c.pLL + half * (c.ALL * c.ALL + c.BLL * c.BLL + c.CLL * c.CLL);
    const float PtotLR = c.pLR + half * (c.ALR * c.ALR + c.BLR * c.BLR + c.CLR * c.CLR);
    const float PtotRL = c.pRL + half * (c.ARL * c.ARL + c.BRL * c.BRL + c.CRL * c.CRL);
    const float PtotRR = c.pRR + half * (c.ARR * c.ARR + c.BRR * c.BRR + c.CRR * c.CRR);
    const float rcLLx = c.rLL * (c.uLL - SL), rcRLx = c.rRL * (SR - c.uRL);
    const float rcLRx = c.rLR * (c.uLR - SL), rcRRx = c.rRR * (SR - c.uRR);
    const float rcLLy = c.rLL * (c.vLL - SB), rcLRy = c.rLR * (ST - c.vLR);
    const float rcRLy = c.rRL * (c.vRL - SB), rcRRy = c.rRR * (ST - c.vRR);
    const float ustar = (rcLLx * c.uLL + rcLRx * c.uLR + rcRLx * c.uRL + rcRRx * c.uRR + (PtotLL - PtotRL + PtotLR - PtotRR))
                      / (rcLLx + rcLRx + rcRLx + rcRRx);
    const float vstar = (rcLLy * c.vLL + rcLRy * c.vLR + rcRLy * c.vRL + rcRRy * c.vRR + (PtotLL - PtotLR + PtotRL - PtotRR))
                      / (rcLLy + rcLRy + rcRLy + rcRRy);
    const float SLustar = 1.0f / (SL - ustar), SRustar = 1.0f / (SR - ustar);
    const float SBvstar = 1.0f / (SB - vstar), STvstar = 1.0f / (ST - vstar);
    const float fLLx = (SL - c.uLL) * SLustar, fLLy = (SB - c.vLL) * SBvstar;
    const float fLRx = (SL - c.uLR) * SLustar, fLRy = (ST - c.vLR) * STvstar;
    const float fRLx = (SR - c.uRL) * SRustar, fRLy = (SB - c.vRL) * SBvstar;
    const float fRRx = (SR - c.uRR) * SRustar, fRRy = (ST - c.vRR) * STvstar;
    const float BstarLL = c.BLL * fLLx, AstarLL = c.ALL * fLLy;
    const float BstarLR = c.BLR * fLRx, AstarLR = c.ALR * fLRy;
    const float BstarRL = c.BRL * fRLx, AstarRL = c.ARL * fRLy;
    const float BstarRR = c.BRR * fRRx, AstarRR = c.ARR * fRRy;
    const float EstarLLx = ustar * BstarLL - c.vLL * c.ALL, EstarLLy = c.uLL * c.BLL - vstar * AstarLL;
    const float EstarLRx = ustar * BstarLR - c.vLR * c.ALR, EstarLRy = c.uLR * c.BLR - vstar * AstarLR;
    const float EstarRLx = ustar * BstarRL - c.vRL * c.ARL, EstarRLy = c.uRL * c.BRL - vstar * AstarRL;
    const float EstarRRx = ustar * BstarRR - c.vRR * c.ARR, EstarRRy = c.uRR * c.BRR - vstar * AstarRR;
    const float EstarLL = ustar * BstarLL - vstar * AstarLL, EstarLR = ustar * BstarLR - vstar * AstarLR;
    const float EstarRL = ustar * BstarRL - vstar * AstarRL, EstarRR = ustar * BstarRR - vstar * AstarRR;
    // 1/sqrt of rstar, rstarx, rstary per corner (rstar = rho fx fy)
    const float qLL = rsqrtf(c.rLL * fLLx * fLLy), qLR = rsqrtf(c.rLR * fLRx * fLRy);
    const float qRL = rsqrtf(c.rRL * fRLx * fRLy), qRR = rsqrtf(c.rRR * fRRx * fRRy);
    const float calfvenL = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(c.ALR) * rsqrtf(c.rLR * fLRx), fabsf(AstarLR) * qLR),
                                             fabsf(c.ALL) * rsqrtf(c.rLL * fLLx)), fabsf(AstarLL) * qLL), smallc);
    const float calfvenR = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(c.ARR) * rsqrtf(c.rRR * fRRx), fabsf(AstarRR) * qRR),
                                             fabsf(c.ARL) * rsqrtf(c.rRL * fRLx)), fabsf(AstarRL) * qRL), smallc);
    const float calfvenB = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(c.BLL) * rsqrtf(c.rLL * fLLy), fabsf(BstarLL) * qLL),
                                             fabsf(c.BRL) * rsqrtf(c.rRL * fRLy)), fabsf(BstarRL) * qRL), smallc);
    const float calfvenT = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(c.BLR) * rsqrtf(c.rLR * fLRy), fabsf(BstarLR) * qLR),
                                             fabsf(c.BRR) * rsqrtf(c.rRR * fRRy)), fabsf(BstarRR) * qRR), smallc);
    const float SAL = fminf(ustar - calfvenL, zero), SAR = fmaxf(ustar + calfvenR, zero);
    const float SAB = fminf(vstar - calfvenB, zero), SAT = fmaxf(vstar + calfvenT, zero);
    const float SARSAL = 1.0f / (SAR - SAL);
    const float SATSAB = 1.0f / (SAT - SAB);
    float E;
    if (SB > zero) {
        if (SL > zero) E = c.ELL;
        else if (SR < zero) E = c.ERL;
        else E = (SAR * EstarLLx - SAL * EstarRLx + SAR * SAL * (c.BRL - c.BLL)) * SARSAL;
    } else if (ST < zero) {
        if (SL > zero) E = c.ELR;
        else if (SR < zero) E = c.ERR;
        else E = (SAR * EstarLRx - SAL * EstarRRx + SAR * SAL * (c.BRR - c.BLR)) * SARSAL;
    } else if (SL > zero) {
        E = (SAT * EstarLLy - SAB * EstarLRy - SAT * SAB * (c.ALR - c.ALL)) * SATSAB;
    } else if (SR < zero) {
        E = (SAT * EstarRLy - SAB * EstarRRy - SAT * SAB * (c.ARR - c.ARL)) * SATSAB;
    } else {
        const float AstarT = (SAR * AstarRR - SAL * AstarLR) * SARSAL;
        const float AstarB = (SAR * AstarRL - SAL * AstarLL) * SARSAL;
        const float BstarR = (SAT * BstarRR - SAB * BstarRL) * SATSAB;
        const float BstarL = (SAT * BstarLR - SAB * BstarLL) * SATSAB;
        E = (SAL * SAB * EstarRR - SAL * SAT * EstarRL - SAR * SAB * EstarLR + SAR * SAT * EstarLL) * SARSAL * SATSAB
          - SAT * SAB * SATSAB * (AstarT - AstarB) + SAR * SAL * SARSAL * (BstarR - BstarL);
    }
    return E * dt;
}

template <typename T>
__device__ T hlld2d(const Corners<T> &c, T dt, T gamma) {
    if constexpr (sizeof(T) == 4) return hlld2d_f(c, dt, gamma);
    const T one = T(1), half = T(0.5), zero = T(0), smallc = T(kSmallc);
    const T b2LL = c.ALL * c.ALL + c.BLL * c.BLL + c.CLL * c.CLL, b2LR = c.ALR * c.ALR + c.BLR * c.BLR + c.CLR * c.CLR;
    const T b2RL = c.ARL * c.ARL + c.BRL * c.BRL + c.CRL * c.CRL, b2RR = c.ARR * c.ARR + c.BRR * c.BRR + c.CRR * c.CRR;
    const T cfx = sqr(mx4(cfast2_b2(gamma, c.pLL, c.rLL, c.ALL, b2LL), cfast2_b2(gamma, c.pLR, c.rLR, c.ALR, b2LR),
                          cfast2_b2(gamma, c.pRL, c.rRL, c.ARL, b2RL), cfast2_b2(gamma, c.pRR, c.rRR, c.ARR, b2RR)));
    const T cfy = sqr(mx4(cfast2_b2(gamma, c.pLL, c.rLL, c.BLL, b2LL), cfast2_b2(gamma, c.pLR, c.rLR, c.BLR, b2LR),
                          cfast2_b2(gamma, c.pRL, c.rRL, c.BRL, b2RL), cfast2_b2(gamma, c.pRR, c.rRR, c.BRR, b2RR)));
    const T SL = mn4(c.uLL, c.uLR, c.uRL, c.uRR) - cfx;
    const T SR = mx4(c.uLL, c.uLR, c.uRL, c.uRR) + cfx;
    const T SB = mn4(c.vLL, c.vLR, c.vRL, c.vRR) - cfy;
    const T ST = mx4(c.vLL, c.vLR, c.vRL, c.vRR) + cfy;
    const T PtotLL = c.pLL + half * (c.ALL * c.ALL + c.BLL * c.BLL + c.CLL * c.CLL);
    const T PtotLR = c.pLR + half * (c.ALR * c.ALR + c.BLR * c.BLR + c.CLR * c.CLR);
    const T PtotRL = c.pRL + half * (c.ARL * c.ARL + c.BRL * c.BRL + c.CRL * c.CRL);
    const T PtotRR = c.pRR + half * (c.ARR * c.ARR + c.BRR * c.BRR + c.CRR * c.CRR);
    const T rcLLx = c.rLL * (c.uLL - SL), rcRLx = c.rRL * (SR - c.uRL);
    const T rcLRx = c.rLR * (c.uLR - SL), rcRRx = c.rRR * (SR - c.uRR);
    const T rcLLy = c.rLL * (c.vLL - SB), rcLRy = c.rLR * (ST - c.vLR);
    const T rcRLy = c.rRL * (c.vRL - SB), rcRRy = c.rRR * (ST - c.vRR);
    const T ustar = (rcLLx * c.uLL + rcLRx * c.uLR + rcRLx * c.uRL + rcRRx * c.uRR + (PtotLL - PtotRL + PtotLR - PtotRR))
                  / (rcLLx + rcLRx + rcRLx + rcRRx);
    const T vstar = (rcLLy * c.vLL + rcLRy * c.vLR + rcRLy * c.vRL + rcRRy * c.vRR + (PtotLL - PtotLR + PtotRL - PtotRR))
                  / (rcLLy + rcLRy + rcRLy + rcRRy);
    const T SLustar = one / (SL - ustar), SRustar = one / (SR - ustar);
    const T SBvstar = one / (SB - vstar), STvstar = one / (ST - vstar);
    const T rstarLLx = c.rLL * (SL - c.uLL) * SLustar;
    const T BstarLL = c.BLL * (SL - c.uLL) * SLustar;
    const T rstarLLy = c.rLL * (SB - c.vLL) * SBvstar;
    const T AstarLL = c.ALL * (SB - c.vLL) * SBvstar;
    const T rstarLL = c.rLL * (SL - c.uLL) * SLustar * (SB - c.vLL) * SBvstar;
    const T EstarLLx = ustar * BstarLL - c.vLL * c.ALL;
    const T EstarLLy = c.uLL * c.BLL - vstar * AstarLL;
    const T EstarLL = ustar * BstarLL - vstar * AstarLL;
    const T rstarLRx = c.rLR * (SL - c.uLR) * SLustar;
    const T BstarLR = c.BLR * (SL - c.uLR) * SLustar;
    const T rstarLRy = c.rLR * (ST - c.vLR) * STvstar;
    const T AstarLR = c.ALR * (ST - c.vLR) * STvstar;
    const T rstarLR = c.rLR * (SL - c.uLR) * SLustar * (ST - c.vLR) * STvstar;
    const T EstarLRx = ustar * BstarLR - c.vLR * c.ALR;
    const T EstarLRy = c.uLR * c.BLR - vstar * AstarLR;
    const T EstarLR = ustar * BstarLR - vstar * AstarLR;
    const T rstarRLx = c.rRL * (SR - c.uRL) * SRustar;
    const T BstarRL = c.BRL * (SR - c.uRL) * SRustar;
    const T rstarRLy = c.rRL * (SB - c.vRL) * SBvstar;
    const T AstarRL = c.ARL * (SB - c.vRL) * SBvstar;
    const T rstarRL = c.rRL * (SR - c.uRL) * SRustar * (SB - c.vRL) * SBvstar;
    const T EstarRLx = ustar * BstarRL - c.vRL * c.ARL;
    const T EstarRLy = c.uRL * c.BRL - vstar * AstarRL;
    const T EstarRL = ustar * BstarRL - vstar * AstarRL;
    const T rstarRRx = c.rRR * (SR - c.uRR) * SRustar;
    const T BstarRR = c.BRR * (SR - c.uRR) * SRustar;
    const T rstarRRy = c.rRR * (ST - c.vRR) * STvstar;
    const T AstarRR = c.ARR * (ST - c.vRR) * STvstar;
    const T rstarRR = c.rRR * (SR - c.uRR) * SRustar * (ST - c.vRR) * STvstar;
    const T EstarRRx = ustar * BstarRR - c.vRR * c.ARR;
    const T EstarRRy = c.uRR * c.BRR - vstar * AstarRR;
    const T EstarRR = ustar * BstarRR - vstar * AstarRR;
    const T sqrtrstarLR = one / sqr(rstarLR);
    const T sqrtrstarRL = one / sqr(rstarRL);
    const T sqrtrstarRR = one / sqr(rstarRR);
    const T sqrtrstarLL = one / sqr(rstarLL);
    const T calfvenL = mx(mx(mx(mx(fab(c.ALR) / sqr(rstarLRx), fab(AstarLR) * sqrtrstarLR),
                                fab(c.ALL) / sqr(rstarLLx)), fab(AstarLL) * sqrtrstarLL), smallc);
    const T calfvenR = mx(mx(mx(mx(fab(c.ARR) / sqr(rstarRRx), fab(AstarRR) * sqrtrstarRR),
                                fab(c.ARL) / sqr(rstarRLx)), fab(AstarRL) * sqrtrstarRL), smallc);
    const T calfvenB = mx(mx(mx(mx(fab(c.BLL) / sqr(rstarLLy), fab(BstarLL) * sqrtrstarLL),
                                fab(c.BRL) / sqr(rstarRLy)), fab(BstarRL) * sqrtrstarRL), smallc);
    const T calfvenT = mx(mx(mx(mx(fab(c.BLR) / sqr(rstarLRy), fab(BstarLR) * sqrtrstarLR),
                                fab(c.BRR) / sqr(rstarRRy)), fab(BstarRR) * sqrtrstarRR), smallc);
    const T SAL = mn(ustar - calfvenL, zero), SAR = mx(ustar + calfvenR, zero);
    const T SAB = mn(vstar - calfvenB, zero), SAT = mx(vstar + calfvenT, zero);
    const T SARSAL = one / (SAR - SAL);
    const T SATSAB = one / (SAT - SAB);
    const T AstarT = (SAR * AstarRR - SAL * AstarLR) * SARSAL;
    const T AstarB = (SAR * AstarRL - SAL * AstarLL) * SARSAL;
    const T BstarR = (SAT * BstarRR - SAB * BstarRL) * SATSAB;
    const T BstarL = (SAT * BstarLR - SAB * BstarLL) * SATSAB;
    T E;
    if (SB > zero) {
        if (SL > zero) E = c.ELL;
        else if (SR < zero) E = c.ERL;
        else E = (SAR * EstarLLx - SAL * EstarRLx + SAR * SAL * (c.BRL - c.BLL)) * SARSAL;
    } else if (ST < zero) {
        if (SL > zero) E = c.ELR;
        else if (SR < zero) E = c.ERR;
        else E = (SAR * EstarLRx - SAL * EstarRRx + SAR * SAL * (c.BRR - c.BLR)) * SARSAL;
    } else if (SL > zero) {
        E = (SAT * EstarLLy - SAB * EstarLRy - SAT * SAB * (c.ALR - c.ALL)) * SATSAB;
    } else if (SR < zero) {
        E = (SAT * EstarRLy - SAB * EstarRRy - SAT * SAB * (c.ARR - c.ARL)) * SATSAB;
    } else {
        E = (SAL * SAB * EstarRR - SAL * SAT * EstarRL - SAR * SAB * EstarLR + SAR * SAT * EstarLL) * SARSAL * SATSAB
          - SAT * SAB * SATSAB * (AstarT - AstarB) + SAR * SAL * SARSAL * (BstarR - BstarL);
    }
    return E * dt;
}

template <typename T>
__device__ T upwind2d(const Corners<T> &c, T dt) {
    const T half = T(0.5), forth = T(0.25);
    T E = forth * (c.ELL + c.ERL + c.ELR + c.ERR);
    T ul = half * (c.uLL + c.uLR), bl = half * (c.BLL + c.BLR);
    T ur = half * (c.uRR + c.uRL), br = half * (c.BRR + c.BRL);
    T vel_info = half * (ul + ur);
    T flux_x = -fab(vel_info) * half * (br - bl);
    ul = half * (c.vLL + c.vRL); bl = half * (c.ALL + c.ARL);
    ur = half * (c.vRR + c.vLR); br = half * (c.ARR + c.ALR);
    vel_info = half * (ul + ur);
    T flux_y = -fab(vel_info) * half * (br - bl);
    T emf = E + (flux_x - flux_y);
    return emf * dt;
}

template <typename T>
__device__ T hlla2d(const Corners<T> &c, T dt) {
    const T zero = T(0), smallc = T(kSmallc);
    const T cLLx = sqr(c.ALL * c.ALL / c.rLL), cLRx = sqr(c.ALR * c.ALR / c.rLR);
    const T cRLx = sqr(c.ARL * c.ARL / c.rRL), cRRx = sqr(c.ARR * c.ARR / c.rRR);
    const T cLLy = sqr(c.BLL * c.BLL / c.rLL), cLRy = sqr(c.BLR * c.BLR / c.rLR);
    const T cRLy = sqr(c.BRL * c.BRL / c.rRL), cRRy = sqr(c.BRR * c.BRR / c.rRR);
    const T SL = mn(mn4(c.uLL, c.uLR, c.uRL, c.uRR) - mx(mx4(cLLx, cLRx, cRLx, cRRx), smallc), zero);
    const T SR = mx(mx4(c.uLL, c.uLR, c.uRL, c.uRR) + mx(mx4(cLLx, cLRx, cRLx, cRRx), smallc), zero);
    const T SB = mn(mn4(c.vLL, c.vLR, c.vRL, c.vRR) - mx(mx4(cLLy, cLRy, cRLy, cRRy), smallc), zero);
    const T ST = mx(mx4(c.vLL, c.vLR, c.vRL, c.vRR) + mx(mx4(cLLy, cLRy, cRLy, cRRy), smallc), zero);
    T emf = (SL * SB * c.ERR - SL * ST * c.ERL - SR * SB * c.ELR + SR * ST * c.ELL) / (SR - SL) / (ST - SB)
          - ST * SB / (ST - SB) * (c.ARR - c.ALL) + SR * SL / (SR - SL) * (c.BRR - c.BLL);
    return emf * dt;
}

}  // namespace dg
