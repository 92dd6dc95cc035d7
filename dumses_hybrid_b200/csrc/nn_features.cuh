// Inputs, targets and gates of the learned face-flux surrogate.
//
// The network stands in for the HLLD face solver (src/modules/solvers/solver.f90:618-836)
// on smooth interfaces.  It does not predict the flux itself but the difference between
// the HLLD flux and the local Lax-Friedrichs flux of the same interface states
// (solver.f90:393-498).  States are first put in units of the interface: density
// rho0 = (rhoL + rhoR) / 2, a speed a0 >= both fast magnetosonic speeds, and the field
// unit sqrt(rho0) a0.  On a smooth interface the HLLD-LLF difference is a dissipation
// correction proportional to the jump between the two states, so the inputs are the
// mean state, the direction of the jump and its size J, and the target is the
// correction divided by J: both stay of order one however small the jump, and the
// network's error enters the flux multiplied by J.  (BF16 inputs could not resolve a
// small jump given as two nearly equal states.)
//
// Interface state order (as passed to the 1D solvers): 0 rho, 1 P, 2 u_n, 3 B_n (the face
// mean), 4 v_t1, 5 B_t1, 6 v_t2, 7 B_t2.
// 17 inputs, from the left/right rho, u_n, v_t1, v_t2, P, B_t1, B_t2 and the face B_n:
//   0..6   mean of u_n, v_t1, v_t2, P, B_n, B_t1, B_t2 (the mean density is 1 by construction)
//   7..13  (right - left) / J of rho, u_n, v_t1, v_t2, P, B_t1, B_t2, J = the norm of that jump
//   14     J,  15  ln(J) / 10,  16  gamma - 1
// 8 outputs, each divided by J and by its unit: corrections of the mass, energy, full
// normal-momentum (HLLD's flux plus its p*_T), t1-momentum, B_t1, t2-momentum and B_t2
// fluxes, and of p*_T against the mean total pressure.
#pragma once
#include <cuda_bf16.h>

#include "solvers.cuh"

namespace dg {
namespace nn {

// Network shape: kNHid hidden layers of kHid units (a build option, DG_NN_WIDTH and
// DG_NN_DEPTH; 64 and 2 by default: of the shapes measured, the fastest that learns every
// output's correction on small harvests as well as on large ones).  kHid is 32, 64 or 128: one M = 128 tile of faces
// holds its accumulator in kHid tensor-memory columns, and the transposed hidden operands
// of the weight-gradient products keep kHidT = 128 rows (rows kHid.. stay zero), so those
// products stay M = 128 MMAs at every width.
#ifndef DG_NN_WIDTH
#define DG_NN_WIDTH 64
#endif
#ifndef DG_NN_DEPTH
#define DG_NN_DEPTH 2
#endif
constexpr int kIn = 17, kInPad = 32, kHid = DG_NN_WIDTH, kOut = 8, kOutPad = 16;
constexpr int kNHid = DG_NN_DEPTH;  // hidden layers
constexpr int kNL = kNHid + 1;      // weight layers; layer kNHid is the output layer
constexpr int kHidT = 128;
static_assert(kHid == 32 || kHid == 64 || kHid == 128, "hidden width must be 32, 64 or 128");
static_assert(kNHid >= 1 && kNHid <= 3, "one to three hidden layers");

struct FaceUnits {
    float rho0, a0, b0, jump;  // interface units and the jump size J
};

constexpr float kTinyJump = 1e-20f;

// per-output scale factor in units of the interface (without J)
__device__ __forceinline__ float out_scale(const FaceUnits &u, int c) {
    const float m = u.rho0 * u.a0;
    switch (c) {
        case 0: return m;                         // mass
        case 1: return m * u.a0 * u.a0;           // energy
        case 4: case 6: return u.b0 * u.a0;       // induction
        default: return m * u.a0;                 // momenta and p*_T
    }
}

// network inputs of one interface; iso states use P = rho ciso^2 as the solvers do
__device__ __forceinline__ FaceUnits face_inputs(const float *ql, const float *qr, float gamma, float ciso, int iso,
                                                 float x[kIn]) {
    const float pl = iso ? ql[0] * (ciso * ciso) : ql[1];
    const float pr = iso ? qr[0] * (ciso * ciso) : qr[1];
    const float bn = ql[3];
    const float b2l = bn * bn + ql[5] * ql[5] + ql[7] * ql[7];
    const float b2r = bn * bn + qr[5] * qr[5] + qr[7] * qr[7];
    FaceUnits u;
    u.rho0 = 0.5f * (ql[0] + qr[0]);
    u.a0 = sqrtf(fmaxf((gamma * pl + b2l) / ql[0], (gamma * pr + b2r) / qr[0]));
    u.b0 = sqrtf(u.rho0) * u.a0;
    const float ir = 1.0f / u.rho0, ia = 1.0f / u.a0, ip = ir * ia * ia, ib = 1.0f / u.b0;
    // scaled left and right: rho, u_n, v_t1, v_t2, P, B_t1, B_t2
    const float L[7] = {ql[0] * ir, ql[2] * ia, ql[4] * ia, ql[6] * ia, pl * ip, ql[5] * ib, ql[7] * ib};
    const float R[7] = {qr[0] * ir, qr[2] * ia, qr[4] * ia, qr[6] * ia, pr * ip, qr[5] * ib, qr[7] * ib};
    float j2 = 0.0f;
#pragma unroll
    for (int n = 0; n < 7; n++) j2 += (R[n] - L[n]) * (R[n] - L[n]);
    u.jump = sqrtf(j2);
    const float ij = (u.jump > kTinyJump) ? 1.0f / u.jump : 0.0f;
    x[0] = 0.5f * (L[1] + R[1]); x[1] = 0.5f * (L[2] + R[2]); x[2] = 0.5f * (L[3] + R[3]);
    x[3] = 0.5f * (L[4] + R[4]); x[4] = bn * ib;             x[5] = 0.5f * (L[5] + R[5]);
    x[6] = 0.5f * (L[6] + R[6]);
#pragma unroll
    for (int n = 0; n < 7; n++) x[7 + n] = (R[n] - L[n]) * ij;
    x[14] = u.jump;
    x[15] = 0.1f * logf(fmaxf(u.jump, kTinyJump));
    x[16] = gamma - 1.0f;
    return u;
}

// the base of the correction: LLF fluxes in output order and the mean total pressure, and
// the LLF dissipation term dis (central flux minus LLF flux; zero for p*_T)
template <typename T>
__device__ __forceinline__ void base_fluxes(const T *ql, const T *qr, T gamma, T ciso, int iso, T b[kOut],
                                            T dis[kOut]) {
    T fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, ploc, proc, a);
    const T half = T(0.5);
    const T vel = mx(cfast(gamma, ploc, ql[0], a, ql[5], ql[7]) + fab(ql[2]),
                     cfast(gamma, proc, qr[0], a, qr[5], qr[7]) + fab(qr[2]));
    const int src[7] = {0, 1, 2, 4, 5, 6, 7};
#pragma unroll
    for (int c = 0; c < 7; c++) {
        const int n = src[c];
        dis[c] = vel * half * (cr[n] - cl[n]);
        b[c] = half * (fl[n] + fr[n]) - dis[c];
    }
    const T bn = ql[3];
    const T ptl = ploc + half * (bn * bn + ql[5] * ql[5] + ql[7] * ql[7]);
    const T ptr = proc + half * (bn * bn + qr[5] * qr[5] + qr[7] * qr[7]);
    b[7] = half * (ptl + ptr);
    dis[7] = T(0);
}

// dissipation gate: per flux component, the learned correction k (in units of scale x J)
// must move the flux from LLF towards the central flux, no further than the whole LLF
// dissipation dn (same units), up to eps = 5% of the largest |dn|.  A flux outside that
// band would be anti-diffusive or more diffusive than LLF: HLLD is used instead.
__device__ __forceinline__ bool gate_dissipation(const float y[kOut], const float dn[kOut]) {
    float dmax = 0.0f;
#pragma unroll
    for (int c = 0; c < 7; c++) dmax = fmaxf(dmax, fabsf(dn[c]));
    const float eps = 0.05f * dmax;
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 7; c++) {
        const float k = (dn[c] >= 0.0f) ? y[c] : -y[c];
        ok = ok && k >= -eps && k <= fabsf(dn[c]) + eps;
    }
    return ok;
}

// HLLD fluxes in output order (normal momentum including p*_T), FP64 labels
__device__ __forceinline__ void hlld_targets(const double *ql, const double *qr, double gamma, double ciso, int iso,
                                             double t[kOut]) {
    double f[8], pg;
    hlld1d<double>(ql, qr, f, pg, gamma, ciso, iso, 1.0 / (gamma - 1.0));
    t[0] = f[0]; t[1] = f[1]; t[2] = f[2] + pg; t[3] = f[4]; t[4] = f[5]; t[5] = f[6]; t[6] = f[7]; t[7] = pg;
}

// gates and the envelope of the training inputs/outputs, set when training ends
struct Gates {
    float xmin[kIn], xmax[kIn];  // input envelope seen in training
    float ymax;                  // largest |output| seen in training (scaled)
    float jump;                  // relative pressure / density jump above which HLLD is used
    float compress;              // u_nR - u_nL below -compress * a0 marks a shock: HLLD
    float margin;                // envelope margin (fraction of its width)
};

// true when the interface is smooth and inside the network's training envelope
__device__ __forceinline__ bool gate_inputs(const Gates &g, const float *ql, const float *qr, float ciso, int iso,
                                            const FaceUnits &u, const float x[kIn]) {
    const float rl = ql[0], rr = qr[0];
    const float pl = iso ? rl * (ciso * ciso) : ql[1], pr = iso ? rr * (ciso * ciso) : qr[1];
    if (!(rl > 0.0f && rr > 0.0f && pl > 0.0f && pr > 0.0f)) return false;           // positivity
    if (fabsf(pl - pr) > g.jump * fminf(pl, pr)) return false;                         // pressure jump
    if (fabsf(rl - rr) > g.jump * fminf(rl, rr)) return false;                         // density jump
    if (qr[2] - ql[2] < -g.compress * u.a0) return false;                              // compression
#pragma unroll
    for (int n = 0; n < kIn; n++) {
        const float w = g.margin * (g.xmax[n] - g.xmin[n]);
        if (!(x[n] >= g.xmin[n] - w && x[n] <= g.xmax[n] + w)) return false;          // confidence: envelope
    }
    return true;
}

// SmeLU, the smooth ReLU of Shamir, Lin, Coviello and Chen ("Smooth activations and
// reproducibility in deep networks", 2020) with half-width 1:
//   f(z) = 0 (z <= -1),  (z + 1)^2 / 4 (|z| < 1),  z (z >= 1);   f'(z) = clamp((z + 1) / 2, 0, 1).
// With h = (clamp(z, -1, 1) + 1) / 2, f = max(z, h^2) ((z + 1)^2 / 4 - z = (z - 1)^2 / 4 >= 0) and f' = h:
// min/max and multiply-adds only, no transcendental (the tanh of a GELU runs on the XU pipe, at 1/8 of
// the FMA pipe's rate on this chip, and bound the face kernel with it).
__device__ __forceinline__ float smelu_h(float z) { return 0.5f * fminf(fmaxf(z, -1.0f), 1.0f) + 0.5f; }
__device__ __forceinline__ float smelu(float z) {
    const float h = smelu_h(z);
    return fmaxf(z, h * h);
}
__device__ __forceinline__ float smelu_d(float z) { return smelu_h(z); }
// two SmeLUs of pre-activations (accumulators that already hold the bias) packed as BF16x2
// (low half = a): one conversion, then BF16x2 arithmetic (h = min(relu(z/2 + 1/2), 1) in two
// instructions); the results are BF16 activations, so BF16 accuracy suffices
__device__ __forceinline__ uint32_t smelu2_bf16(float a, float b) {
    const __nv_bfloat162 z = __floats2bfloat162_rn(a, b);
    const __nv_bfloat162 one = __float2bfloat162_rn(1.0f), half = __float2bfloat162_rn(0.5f);
    const __nv_bfloat162 h = __hmin2(__hfma2_relu(z, half, half), one);
    const __nv_bfloat162 f = __hmax2(z, __hmul2(h, h));
    return *reinterpret_cast<const uint32_t *>(&f);
}

// standardisation of the network's inputs and outputs, fitted on the training samples:
// the network sees (x - xmu) * xisd (xisd = 1 / xsd) and its output is multiplied by ysd
struct Scaling {
    float xmu[kIn], xsd[kIn], ysd[kOut], xisd[kIn];
};

// The hidden layers' biases as one extra K = 16 step of their MMAs in the face kernel: a B
// operand [kHid][kBiasK] (blocked K-major) holding each bias split in two BF16 parts,
// column 0 = bf16(b), column 1 = bf16(b - column 0), the other columns zero, multiplied by
// an A operand whose columns 0 and 1 are 1.  The sum of the parts is b to within 2^-17 |b|, and
// the accumulator gets it with no per-activation add in the epilogue.
constexpr int kBiasK = 16;
__host__ __device__ __forceinline__ void bias_split(float b, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(b);
    lo = __float2bfloat16_rn(b - __bfloat162float(hi));
}

// device view of the trained network for inference inside the step
struct NetView {
    const __nv_bfloat16 *wt[kNL];   // forward B operands, blocked K-major [N_l][K_l]
    const __nv_bfloat16 *bt[kNHid]; // hidden-layer bias operands, blocked K-major [kHid][kBiasK]
    const float *b[kNL];            // biases
    Gates gates;
    Scaling sc;
};

}  // namespace nn
}  // namespace dg
