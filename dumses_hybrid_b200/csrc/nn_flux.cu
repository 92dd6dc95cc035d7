// Learned face-flux surrogate: a 17 -> kHid x kNHid -> 8 SmeLU MLP (17-64-64-8 by default)
// trained and run on sm_100a.  Every matrix product is a BF16 tcgen05 MMA with an FP32 accumulator in
// tensor memory; operands are staged into shared memory by bulk copies from the blocked
// K-major layout of nn_umma.cuh.  The forward products write the next layer's operands
// (normal and transposed) and the activation derivative from their epilogues; the backward
// products fold that derivative and the bias-gradient sums into theirs; weight gradients
// are batch-split products reduced by the Adam kernel.  No counterpart exists in the
// reference, whose face solver is always exact (src/modules/solvers/solver.f90:163-187).
#include <chrono>
#include <cstdlib>
#include <thread>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dumses_gpu.h"
#include "mhd_kernels.cuh"
#include "nn_features.cuh"
#include "nn_host.h"
#include "nn_umma.cuh"

namespace dg {
namespace nn {

using bf16 = __nv_bfloat16;

__host__ __device__ constexpr int layer_k(int l) { return l == 0 ? kInPad : kHid; }
__host__ __device__ constexpr int layer_n(int l) { return l == kNHid ? kOutPad : kHid; }
__host__ __device__ constexpr int real_k(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int real_n(int l) { return l == kNHid ? kOut : kHid; }
// row length of the weight-gradient partials of hidden layer l: its B operand is the
// transposed input (kInPad rows) or the transposed, zero-padded activations (kHidT rows)
__host__ __device__ constexpr int dw_cols(int l) { return l == 0 ? kInPad : kHidT; }

enum { M_FWD_HID = 0, M_FWD_OUT = 1, M_BWD_HID = 2, M_DW = 3 };

constexpr int kGemmSmem = 65536 + 1024;  // A tile, B tile, barriers, bias sums (caps residency at 3 CTAs/SM)

struct GemmArgs {
    const bf16 *A, *B;
    int C;             // reduction columns per CTA
    const float *bias; // forward
    bf16 *Hn, *Ht;     // outputs: blocked normal [rows][kHid] and transposed [kHidT][rows]
    float *G;          // activation derivative [rows][kHid]: written forward, read backward
    float *Y;          // network output [rows][8]
    float *part;       // weight-gradient partials [split][128][N] or bias partials [tile][128]
    long long rows;    // batch rows (row tiles x 128)
    int *err;
};

__device__ __forceinline__ void store_bf16x8(bf16 *dst, const float *v) {
    __align__(16) bf16 h[8];
#pragma unroll
    for (int q = 0; q < 8; q++) h[q] = __float2bfloat16_rn(v[q]);
    *(uint4 *)dst = *(const uint4 *)h;
}

template <int MODE, int N>
__device__ __forceinline__ void epilogue(const GemmArgs &g, uint32_t tmem, long long tile, int warp, int lane,
                                         float *sred) {
    const int rl = warp * 32 + lane;
    const long long row = tile * kTileRows + rl;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    if constexpr (MODE == M_DW) {
#pragma unroll
        for (int cc = 0; cc < N / 16; cc++) {
            float v[16];
            tmem_ld16(taddr + cc * 16, v);
            float4 *o = (float4 *)(g.part + ((long long)tile * kTileRows + rl) * N + cc * 16);
#pragma unroll
            for (int q = 0; q < 4; q++) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
    } else if constexpr (MODE == M_FWD_OUT) {
        float v[16];
        tmem_ld16(taddr, v);
        float4 *o = (float4 *)(g.Y + row * kOut);
        o[0] = make_float4(v[0] + g.bias[0], v[1] + g.bias[1], v[2] + g.bias[2], v[3] + g.bias[3]);
        o[1] = make_float4(v[4] + g.bias[4], v[5] + g.bias[5], v[6] + g.bias[6], v[7] + g.bias[7]);
    } else {
        for (int cc = 0; cc < kHid / 16; cc++) {
            float v[16];
            tmem_ld16(taddr + cc * 16, v);
            float *gp = g.G + row * kHid + cc * 16;
            if constexpr (MODE == M_FWD_HID) {
                float gd[16];
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const float z = v[q] + g.bias[cc * 16 + q];
                    v[q] = smelu(z);
                    gd[q] = smelu_d(z);
                }
#pragma unroll
                for (int q = 0; q < 4; q++) ((float4 *)gp)[q] = make_float4(gd[4 * q], gd[4 * q + 1], gd[4 * q + 2], gd[4 * q + 3]);
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float4 d = ((const float4 *)gp)[q];
                    v[4 * q] *= d.x; v[4 * q + 1] *= d.y; v[4 * q + 2] *= d.z; v[4 * q + 3] *= d.w;
                }
#pragma unroll
                for (int q = 0; q < 16; q++) {  // bias gradient: column sums over the tile
                    float s = v[q];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (lane == 0) atomicAdd(&sred[cc * 16 + q], s);
                }
            }
            // normal blocked layout [rows/128][kHid/8][128][8]
            store_bf16x8(g.Hn + ((tile * (kHid / 8) + cc * 2) * kTileRows + rl) * 8, v);
            store_bf16x8(g.Hn + ((tile * (kHid / 8) + cc * 2 + 1) * kTileRows + rl) * 8, v + 8);
            // transposed blocked layout [rows/8][kHidT][8] (rows kHid.. are never written: zero)
            bf16 *t = g.Ht + (row >> 3) * (kHidT * 8) + (row & 7);
#pragma unroll
            for (int q = 0; q < 16; q++) t[(cc * 16 + q) * 8] = __float2bfloat16_rn(v[q]);
        }
    }
}

// one 128-row tile (forward / backward modes) or one batch split (weight-gradient mode)
template <int MODE, int N>
__global__ void __launch_bounds__(128) k_gemm(GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char sm[];
    bf16 *As = (bf16 *)sm;
    bf16 *Bs = (bf16 *)(sm + 32768);
    uint64_t *bar = (uint64_t *)(sm + 65536);
    uint32_t *tslot = (uint32_t *)(sm + 65536 + 16);
    int *sflag = (int *)(sm + 65536 + 32);
    float *sred = (float *)(sm + 65536 + 64);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
        *sflag = 1;
    }
    sred[tid] = 0.0f;
    if (warp == 0) tmem_alloc(tslot, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const long long tile = blockIdx.x;
    if (tid == 0) {
        bool ok = true;
        if constexpr (MODE != M_DW) {
            const unsigned abytes = kTileRows * g.C * 2, bbytes = N * g.C * 2;
            mbar_expect_tx(&bar[0], abytes + bbytes);
            bulk_g2s(As, g.A + tile * (long long)g.C * kTileRows, abytes, &bar[0]);
            bulk_g2s(Bs, g.B, bbytes, &bar[0]);
            ok = mbar_wait(&bar[0], 0);
            if (ok) {
                tc_fence_after();
                mma_tiles(tmem, As, Bs, N, g.C / 16, 0);
                mma_commit(&bar[1]);
                ok = mbar_wait(&bar[1], 0);
                if (!ok) mbar_wait(&bar[1], 0);
            } else {
                mbar_wait(&bar[0], 0);  // let the copies land before the block leaves
            }
        } else {
            const int nch = g.C / 128;
            for (int c = 0; c < nch; c++) {
                const long long k0 = tile * (long long)g.C + c * 128;
                const unsigned abytes = kTileRows * 128 * 2, bbytes = N * 128 * 2;
                mbar_expect_tx(&bar[0], abytes + bbytes);
                bulk_g2s(As, g.A + (k0 / 8) * kTileRows * 8, abytes, &bar[0]);
                bulk_g2s(Bs, g.B + (k0 / 8) * N * 8, bbytes, &bar[0]);
                ok = mbar_wait(&bar[0], c & 1);
                if (!ok) { mbar_wait(&bar[0], c & 1); break; }
                tc_fence_after();
                mma_tiles(tmem, As, Bs, N, 8, c > 0);
                mma_commit(&bar[1]);
                ok = mbar_wait(&bar[1], c & 1);
                if (!ok) { mbar_wait(&bar[1], c & 1); break; }
            }
        }
        if (!ok) {
            *sflag = 0;
            atomicOr(g.err, NN_ERR_WAIT);
        }
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const bool ok = *sflag != 0;
    if (ok) epilogue<MODE, N>(g, tmem, tile, warp, lane, sred);
    tc_fence_before();
    __syncthreads();
    if (MODE == M_BWD_HID && ok) g.part[tile * kTileRows + tid] = sred[tid];
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 128);
    }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {  // splitmix64 finaliser
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// batch assembly: rows drawn at random (with replacement) or in order from `first`;
// rows past the end of the sample set are zero
__global__ void k_gather(const float *__restrict__ xs, const float *__restrict__ ts, long long ns, long long rows,
                         int random, unsigned long long seed, long long first, const Scaling *__restrict__ sc,
                         bf16 *__restrict__ Xn, bf16 *__restrict__ Xt, float *__restrict__ Tb) {
    const long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (b >= rows) return;
    long long idx = random ? (long long)(mix64(seed ^ (unsigned long long)b * 0xD1B54A32D192ED03ull) % (unsigned long long)ns)
                           : first + b;
    float x[kInPad], t[kOut];
#pragma unroll
    for (int n = 0; n < kInPad; n++) x[n] = 0.0f;
#pragma unroll
    for (int n = 0; n < kOut; n++) t[n] = 0.0f;
    if (idx < ns) {
#pragma unroll
        for (int n = 0; n < kIn; n++) x[n] = (xs[idx * kIn + n] - sc->xmu[n]) * sc->xisd[n];
        if (ts) {
#pragma unroll
            for (int n = 0; n < kOut; n++) t[n] = ts[idx * kOut + n] / sc->ysd[n];
        }
    }
    const long long tile = b / kTileRows, rl = b % kTileRows;
#pragma unroll
    for (int cg = 0; cg < kInPad / 8; cg++) store_bf16x8(Xn + ((tile * (kInPad / 8) + cg) * kTileRows + rl) * 8, x + cg * 8);
    bf16 *xt = Xt + (b >> 3) * (kInPad * 8) + (b & 7);
#pragma unroll
    for (int n = 0; n < kInPad; n++) xt[n * 8] = __float2bfloat16_rn(x[n]);
    float4 *tb = (float4 *)(Tb + b * kOut);
    tb[0] = make_float4(t[0], t[1], t[2], t[3]);
    tb[1] = make_float4(t[4], t[5], t[6], t[7]);
}

// mean-squared-error gradient of the outputs, its transposed copy, and per-tile sums of
// the loss and of the output-bias gradient
__global__ void __launch_bounds__(128) k_loss(const float *__restrict__ Y, const float *__restrict__ Tb, long long rows,
                                              long long valid, bf16 *__restrict__ Dn, bf16 *__restrict__ Dt,
                                              float *__restrict__ lpart, float *__restrict__ bpart) {
    const long long b = blockIdx.x * (long long)kTileRows + threadIdx.x;
    const int rl = threadIdx.x;
    const float sc = 2.0f / (float)(valid * kOut);
    float d[16], l = 0.0f;
#pragma unroll
    for (int n = 0; n < 16; n++) d[n] = 0.0f;
    if (b < valid) {
#pragma unroll
        for (int n = 0; n < kOut; n++) {
            const float e = Y[b * kOut + n] - Tb[b * kOut + n];
            d[n] = sc * e;
            l += e * e;
        }
    }
    store_bf16x8(Dn + ((blockIdx.x * 2LL + 0) * kTileRows + rl) * 8, d);
    store_bf16x8(Dn + ((blockIdx.x * 2LL + 1) * kTileRows + rl) * 8, d + 8);
    bf16 *t = Dt + (b >> 3) * (kOutPad * 8) + (b & 7);
#pragma unroll
    for (int n = 0; n < kOutPad; n++) t[n * 8] = __float2bfloat16_rn(d[n]);
    __shared__ float s[kOut + 1][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int n = 0; n <= kOut; n++) {
        float v = (n < kOut) ? d[n] : l;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s[n][w] = v;
    }
    __syncthreads();
    if (threadIdx.x <= kOut) {
        const float v = s[threadIdx.x][0] + s[threadIdx.x][1] + s[threadIdx.x][2] + s[threadIdx.x][3];
        if (threadIdx.x < kOut) bpart[blockIdx.x * (long long)kOut + threadIdx.x] = v;
        else lpart[blockIdx.x] = v;
    }
}

struct AdamArgs {
    float *W[kNL], *b[kNL], *mW[kNL], *vW[kNL], *mb[kNL], *vb[kNL];
    const float *dw[kNL];  // weight-gradient partials
    const float *db[kNL];  // bias-gradient partials
    bf16 *Wt[kNL], *Wn[kNL], *Bt[kNHid];
    int splits, tiles;
    float lr, beta1, beta2, eps, c1, c2;  // c1 = 1 - beta1^t, c2 = 1 - beta2^t
    int apply;                             // 1: Adam step; 0: only reduce the gradient; 2: only pack BF16 copies
    float *gout;                           // reduced gradients in parameter order (or null)
};

__host__ __device__ constexpr long long layer_params(int l) { return (long long)real_k(l) * real_n(l) + real_n(l); }

// one thread per real parameter: reduce its gradient partials, Adam step on the FP32
// master, BF16 copies in both operand layouts
__global__ void k_adam(AdamArgs a) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int l = 0;
    while (l < kNL && t >= layer_params(l)) { t -= layer_params(l); l++; }
    if (l >= kNL) return;
    long long off = 0;
    for (int q = 0; q < l; q++) off += layer_params(q);
    const int K = layer_k(l), N = layer_n(l), kr = real_k(l), nr = real_n(l);
    const bool is_w = t < (long long)kr * nr;
    float g = 0.0f;
    int k = 0, n = 0;
    // the face kernel's bias operand of hidden layer l < kNHid (its columns 2.. stay zero)
    auto pack_bias = [&](int nb, float b) {
        if (l < kNHid) {
            bf16 hi, lo;
            bias_split(b, hi, lo);
            a.Bt[l][blk_off(nb, 0, kBiasK, kHid)] = hi;
            a.Bt[l][blk_off(nb, 1, kBiasK, kHid)] = lo;
        }
    };
    if (a.apply == 2) {  // pack only: BF16 copies of the current masters
        if (is_w) {
            k = (int)(t / nr);
            n = (int)(t % nr);
            const float w = a.W[l][k * N + n];
            a.Wt[l][blk_off(n, k, K, N < kTileRows ? N : kTileRows)] = __float2bfloat16_rn(w);
            if (l > 0) a.Wn[l][blk_off(k, n, N, K < kTileRows ? K : kTileRows)] = __float2bfloat16_rn(w);
        } else {
            n = (int)(t - (long long)kr * nr);
            pack_bias(n, a.b[l][n]);
        }
        return;
    }
    if (is_w) {
        k = (int)(t / nr);
        n = (int)(t % nr);
        // the weight-gradient product is [n][k] for the hidden layers and [k][n] for the output layer
        for (int s = 0; s < a.splits; s++)
            g += (l < kNHid) ? a.dw[l][((long long)s * kTileRows + n) * dw_cols(l) + k]
                             : a.dw[l][((long long)s * kTileRows + k) * N + n];
    } else {
        n = (int)(t - (long long)kr * nr);
        const int stride = (l < kNHid) ? kTileRows : kOut;
        for (int s = 0; s < a.tiles; s++) g += a.db[l][(long long)s * stride + n];
    }
    if (a.gout) a.gout[off + t] = g;
    if (!a.apply) return;
    float *p = is_w ? &a.W[l][k * N + n] : &a.b[l][n];
    float *m = is_w ? &a.mW[l][k * N + n] : &a.mb[l][n];
    float *v = is_w ? &a.vW[l][k * N + n] : &a.vb[l][n];
    const float mm = a.beta1 * *m + (1.0f - a.beta1) * g;
    const float vv = a.beta2 * *v + (1.0f - a.beta2) * g * g;
    *m = mm;
    *v = vv;
    const float w = *p - a.lr * (mm / a.c1) / (sqrtf(vv / a.c2) + a.eps);
    *p = w;
    if (is_w) {
        a.Wt[l][blk_off(n, k, K, N < kTileRows ? N : kTileRows)] = __float2bfloat16_rn(w);
        if (l > 0) a.Wn[l][blk_off(k, n, N, K < kTileRows ? K : kTileRows)] = __float2bfloat16_rn(w);
    } else {
        pack_bias(n, w);
    }
}

// input envelope and largest |target| of the sample set (ordered-integer min/max)
__device__ __forceinline__ int f2o(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7FFFFFFF; }
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }
__global__ void k_envelope(const float *__restrict__ xs, const float *__restrict__ ts, long long ns, int *mn_, int *mx_,
                           int *ymax) {
    int lo[kIn], hi[kIn], ym = 0;
#pragma unroll
    for (int n = 0; n < kIn; n++) { lo[n] = 0x7FFFFFFF; hi[n] = (int)0x80000000; }
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < ns; s += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int n = 0; n < kIn; n++) {
            const int o = f2o(xs[s * kIn + n]);
            lo[n] = min(lo[n], o);
            hi[n] = max(hi[n], o);
        }
#pragma unroll
        for (int n = 0; n < kOut; n++) ym = max(ym, f2o(fabsf(ts[s * kOut + n])));
    }
#pragma unroll
    for (int n = 0; n < kIn; n++) {
        atomicMin(&mn_[n], lo[n]);
        atomicMax(&mx_[n], hi[n]);
    }
    atomicMax(ymax, ym);
}

// sums and sums of squares of every input and output over the sample set (FP64)
__global__ void k_moments(const float *__restrict__ xs, const float *__restrict__ ts, long long ns, double *acc) {
    double a[2 * (kIn + kOut)];
#pragma unroll
    for (int n = 0; n < 2 * (kIn + kOut); n++) a[n] = 0.0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < ns; s += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int n = 0; n < kIn; n++) {
            const double v = xs[s * kIn + n];
            a[n] += v;
            a[kIn + kOut + n] += v * v;
        }
#pragma unroll
        for (int n = 0; n < kOut; n++) {
            const double v = ts[s * kOut + n];
            a[kIn + n] += v;
            a[2 * kIn + kOut + n] += v * v;
        }
    }
#pragma unroll
    for (int n = 0; n < 2 * (kIn + kOut); n++) {
        double v = a[n];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&acc[n], v);
    }
}

}  // namespace nn
}  // namespace dg

using namespace dg::nn;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct dg_nn {
    int device = 0;
    cudaStream_t stream = nullptr;
    int *d_err = nullptr;
    float *W[kNL] = {}, *b[kNL] = {}, *mW[kNL] = {}, *vW[kNL] = {}, *mb[kNL] = {}, *vb[kNL] = {};
    bf16 *Wt[kNL] = {}, *Wn[kNL] = {}, *Bt[kNHid] = {};
    float *xs = nullptr, *ts = nullptr;  // samples
    long long ns = 0, cap = 0;
    // batch scratch
    long long bcap = 0;
    bf16 *Xn = nullptr, *Xt = nullptr, *Hn[kNHid] = {}, *Ht[kNHid] = {}, *Dn[2] = {}, *Dt[2] = {}, *D3n = nullptr,
         *D3t = nullptr;
    float *Tb = nullptr, *Y = nullptr, *G[kNHid] = {}, *dw[kNL] = {}, *db[kNL] = {}, *lpart = nullptr, *gout = nullptr;
    long long step = 0;
    unsigned long long seed = 1;
    float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    Gates gates{};
    Scaling sc{};              // host copy of the standardisation
    Scaling *d_sc = nullptr;   // device copy read by the batch gather
    int trained = 0;
    std::vector<void *> allocs, scratch;
};

namespace {
int nn_fail(int code, const std::string &m) { return dg::set_error(code, m.c_str()); }
#define NN_CUDA(x)                                                                                       \
    do {                                                                                                 \
        cudaError_t e_ = (x);                                                                            \
        if (e_ != cudaSuccess) return nn_fail(DG_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

int nn_alloc(dg_nn *n, void **p, size_t bytes) {
    NN_CUDA(cudaMalloc(p, bytes));
    NN_CUDA(cudaMemsetAsync(*p, 0, bytes, n->stream));
    n->allocs.push_back(*p);
    return 0;
}
template <typename X> int nn_alloc_t(dg_nn *n, X **p, size_t count) { return nn_alloc(n, (void **)p, count * sizeof(X)); }

// wait for a stream with a wall-clock bound (DG_SYNC_TIMEOUT_S, default 300 s)
int nn_bounded_sync(cudaStream_t st) {
    const char *e = std::getenv("DG_SYNC_TIMEOUT_S");
    const double limit = (e && std::atof(e) > 0) ? std::atof(e) : 300.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaStreamQuery(st);
        if (q == cudaSuccess) return 0;
        if (q != cudaErrorNotReady) return nn_fail(DG_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(q));
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return nn_fail(DG_ERR_TIMEOUT, "device work did not finish within DG_SYNC_TIMEOUT_S");
        std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 5 : 200));
    }
}

int nn_sync(dg_nn *n) {
    if (int rc = nn_bounded_sync(n->stream)) return rc;
    int err = 0;
    NN_CUDA(cudaMemcpy(&err, n->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return nn_fail(DG_ERR_STATE, "network kernel gave up waiting on a tensor-core transfer (error bits " +
                                              std::to_string(err) + ")");
    return 0;
}

int scratch_alloc(dg_nn *n, void **p, size_t bytes) {
    NN_CUDA(cudaMalloc(p, bytes));
    NN_CUDA(cudaMemsetAsync(*p, 0, bytes, n->stream));
    n->scratch.push_back(*p);
    return 0;
}
template <typename X> int scratch_t(dg_nn *n, X **p, size_t count) { return scratch_alloc(n, (void **)p, count * sizeof(X)); }

// batch work arrays for `rows` rows (reallocated when a larger batch comes)
int ensure_batch(dg_nn *n, long long rows) {
    if (rows <= n->bcap) return 0;
    NN_CUDA(cudaStreamSynchronize(n->stream));
    for (void *p : n->scratch) cudaFree(p);
    n->scratch.clear();
    n->bcap = 0;
    int rc;
    const long long R = rows, tiles = R / kTileRows;
    const long long splits = R / ((R % 512 == 0) ? 512 : 128);
    if ((rc = scratch_t(n, &n->Xn, R * kInPad)) || (rc = scratch_t(n, &n->Xt, R * kInPad)) ||
        (rc = scratch_t(n, &n->Tb, R * kOut)) || (rc = scratch_t(n, &n->Y, R * kOut)) ||
        (rc = scratch_t(n, &n->D3n, R * kOutPad)) || (rc = scratch_t(n, &n->D3t, R * kOutPad)) ||
        (rc = scratch_t(n, &n->lpart, tiles)) || (rc = scratch_t(n, &n->gout, dg_nn_param_count())))
        return rc;
    for (int l = 0; l < kNHid; l++)
        if ((rc = scratch_t(n, &n->Hn[l], R * kHid)) || (rc = scratch_t(n, &n->Ht[l], R * kHidT)) ||
            (rc = scratch_t(n, &n->G[l], R * kHid)))
            return rc;
    for (int q = 0; q < 2; q++)
        if ((rc = scratch_t(n, &n->Dn[q], R * kHid)) || (rc = scratch_t(n, &n->Dt[q], R * kHidT))) return rc;
    for (int l = 0; l < kNL; l++)
        if ((rc = scratch_t(n, &n->dw[l], splits * kTileRows * kHidT)) || (rc = scratch_t(n, &n->db[l], tiles * kTileRows)))
            return rc;
    n->bcap = rows;
    return 0;
}

template <int MODE, int N>
int launch_gemm(dg_nn *n, const GemmArgs &g, long long grid) {
    NN_CUDA(cudaFuncSetAttribute(k_gemm<MODE, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
    k_gemm<MODE, N><<<(unsigned)grid, 128, kGemmSmem, n->stream>>>(g);
    NN_CUDA(cudaGetLastError());
    return 0;
}

// forward pass over `rows` gathered rows (a multiple of 128)
int forward(dg_nn *n, long long rows) {
    const long long tiles = rows / kTileRows;
    int rc;
    for (int l = 0; l < kNHid; l++) {
        GemmArgs g{};
        g.A = (l == 0) ? n->Xn : n->Hn[l - 1];
        g.B = n->Wt[l];
        g.C = layer_k(l);
        g.bias = n->b[l];
        g.Hn = n->Hn[l];
        g.Ht = n->Ht[l];
        g.G = n->G[l];
        g.rows = rows;
        g.err = n->d_err;
        if ((rc = launch_gemm<M_FWD_HID, kHid>(n, g, tiles))) return rc;
    }
    GemmArgs g{};
    g.A = n->Hn[kNHid - 1];
    g.B = n->Wt[kNHid];
    g.C = kHid;
    g.bias = n->b[kNHid];
    g.Y = n->Y;
    g.rows = rows;
    g.err = n->d_err;
    return launch_gemm<M_FWD_OUT, kOutPad>(n, g, tiles);
}

// loss gradient and backward pass; leaves weight/bias gradient partials in dw/db
int backward(dg_nn *n, long long rows, long long valid) {
    const long long tiles = rows / kTileRows;
    const int csplit = (rows % 512 == 0) ? 512 : 128;
    const long long splits = rows / csplit;
    k_loss<<<(unsigned)tiles, 128, 0, n->stream>>>(n->Y, n->Tb, rows, valid, n->D3n, n->D3t, n->lpart, n->db[kNHid]);
    NN_CUDA(cudaGetLastError());
    int rc;
    {   // output layer: dW[k][n] = sum_b Ht[k][b] Dt[n][b] over the last hidden layer's activations
        GemmArgs g{};
        g.A = n->Ht[kNHid - 1]; g.B = n->D3t; g.C = csplit; g.part = n->dw[kNHid]; g.rows = rows; g.err = n->d_err;
        if ((rc = launch_gemm<M_DW, kOutPad>(n, g, splits))) return rc;
    }
    const bf16 *dn = n->D3n;
    int cdn = kOutPad;
    for (int l = kNHid - 1; l >= 0; l--) {
        bf16 *on = n->Dn[l & 1], *ot = n->Dt[l & 1];
        {   // dZ_l = (dZ_{l+1} W_{l+1}^T) * f'(Z_l), bias partials of layer l
            GemmArgs g{};
            g.A = dn; g.B = n->Wn[l + 1]; g.C = cdn; g.G = n->G[l]; g.Hn = on; g.Ht = ot; g.part = n->db[l];
            g.rows = rows; g.err = n->d_err;
            if ((rc = launch_gemm<M_BWD_HID, kHid>(n, g, tiles))) return rc;
        }
        {   // dW_l[n][k] = sum_b dZt_l[n][b] Ht_{l-1}[k][b]
            GemmArgs g{};
            g.A = ot; g.B = (l == 0) ? n->Xt : n->Ht[l - 1]; g.C = csplit; g.part = n->dw[l]; g.rows = rows; g.err = n->d_err;
            if (l == 0) rc = launch_gemm<M_DW, kInPad>(n, g, splits);
            else rc = launch_gemm<M_DW, kHidT>(n, g, splits);
            if (rc) return rc;
        }
        dn = on;
        cdn = kHid;
    }
    return 0;
}

int adam(dg_nn *n, long long rows, float lr, int apply, float *gout) {
    AdamArgs a{};
    for (int l = 0; l < kNL; l++) {
        a.W[l] = n->W[l]; a.b[l] = n->b[l]; a.mW[l] = n->mW[l]; a.vW[l] = n->vW[l]; a.mb[l] = n->mb[l];
        a.vb[l] = n->vb[l]; a.dw[l] = n->dw[l]; a.db[l] = n->db[l]; a.Wt[l] = n->Wt[l]; a.Wn[l] = n->Wn[l];
        if (l < kNHid) a.Bt[l] = n->Bt[l];
    }
    a.splits = (int)(rows / ((rows % 512 == 0) ? 512 : 128));
    a.tiles = (int)(rows / kTileRows);
    a.lr = lr; a.beta1 = n->beta1; a.beta2 = n->beta2; a.eps = n->eps;
    if (apply == 1) n->step++;
    const double t = (double)(n->step > 0 ? n->step : 1);
    a.c1 = (float)(1.0 - std::pow((double)n->beta1, t));
    a.c2 = (float)(1.0 - std::pow((double)n->beta2, t));
    a.apply = apply;
    a.gout = gout;
    const long long np = dg_nn_param_count();
    k_adam<<<(unsigned)((np + 255) / 256), 256, 0, n->stream>>>(a);
    NN_CUDA(cudaGetLastError());
    return 0;
}

int gather(dg_nn *n, long long rows, int random, long long first) {
    k_gather<<<(unsigned)((rows + 127) / 128), 128, 0, n->stream>>>(n->xs, n->ts, n->ns, rows, random,
                                                                      n->seed + 0x9E37ull * (unsigned long long)n->step,
                                                                      first, n->d_sc, n->Xn, n->Xt, n->Tb);
    NN_CUDA(cudaGetLastError());
    return 0;
}

// write the BF16 operand copies of the FP32 masters
int pack_weights(dg_nn *n) {
    return adam(n, kTileRows, 0.0f, 2, nullptr);
}

int check_batch(long long batch) {
    if (batch < kTileRows || batch % kTileRows) return nn_fail(DG_ERR_ARG, "batch must be a positive multiple of 128");
    return 0;
}
}  // namespace

namespace {
// one block waiting on an mbarrier with the library's bounded wait; one thread arrives on it
// (arrive = 1) or nothing does (arrive = 0), so the wait completes or runs out its time
__global__ void k_wait_selftest(int arrive, int *err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0) mbar_arrive(&bar);
    if (!mbar_wait(&bar, 0)) atomicOr(err, NN_ERR_WAIT);
}
}  // namespace

extern "C" {

int dg_wait_selftest(int device, int arrive, double *seconds) {
    if (cudaSetDevice(device) != cudaSuccess) return nn_fail(DG_ERR_NODEVICE, "no CUDA device");
    int *d_err = nullptr;
    NN_CUDA(cudaMalloc(&d_err, sizeof(int)));
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaFree(d_err);
        return nn_fail(DG_ERR_CUDA, "cudaStreamCreate failed");
    }
    int rc = 0, err = 0;
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaMemsetAsync(d_err, 0, sizeof(int), st) != cudaSuccess) rc = nn_fail(DG_ERR_CUDA, "cudaMemsetAsync failed");
    if (!rc) {
        k_wait_selftest<<<1, 32, 0, st>>>(arrive, d_err);
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) rc = nn_fail(DG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(le));
    }
    if (!rc) rc = nn_bounded_sync(st);
    if (!rc && cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = nn_fail(DG_ERR_CUDA, "cudaMemcpy failed");
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    cudaStreamDestroy(st);
    cudaFree(d_err);
    if (rc) return rc;
    if (err) return nn_fail(DG_ERR_TIMEOUT, "an mbarrier wait ran out of its time bound");
    return DG_OK;
}

long long dg_nn_param_count(void) {
    long long n = 0;
    for (int l = 0; l < kNL; l++) n += layer_params(l);
    return n;
}

int dg_nn_shape(int *width, int *depth) {
    if (width) *width = kHid;
    if (depth) *depth = kNHid;
    return DG_OK;
}

int dg_nn_create(int device, unsigned long long seed, dg_nn **out) {
    if (!out) return nn_fail(DG_ERR_ARG, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return nn_fail(DG_ERR_NODEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return nn_fail(DG_ERR_ARG, "device index out of range");
    NN_CUDA(cudaSetDevice(device));
    dg_nn *n = new dg_nn();
    n->device = device;
    n->seed = seed;
    int rc = 0;
    auto bail = [&](int code) { dg_nn_destroy(n); return code; };
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(nn_fail(DG_ERR_CUDA, "stream creation failed"));
    if ((rc = nn_alloc_t(n, &n->d_err, 1))) return bail(rc);
    // He-normal initial weights on the host from the seed (Box-Muller over splitmix64)
    unsigned long long st = seed * 0x9E3779B97F4A7C15ull + 12345u;
    auto next = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        unsigned long long z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < kNL; l++) {
        const int K = layer_k(l), N = layer_n(l);
        if ((rc = nn_alloc_t(n, &n->W[l], (size_t)K * N)) || (rc = nn_alloc_t(n, &n->b[l], N)) ||
            (rc = nn_alloc_t(n, &n->mW[l], (size_t)K * N)) || (rc = nn_alloc_t(n, &n->vW[l], (size_t)K * N)) ||
            (rc = nn_alloc_t(n, &n->mb[l], N)) || (rc = nn_alloc_t(n, &n->vb[l], N)) ||
            (rc = nn_alloc_t(n, &n->Wt[l], (size_t)K * N)) || (rc = nn_alloc_t(n, &n->Wn[l], (size_t)K * N)) ||
            (l < kNHid && (rc = nn_alloc_t(n, &n->Bt[l], (size_t)kBiasK * kHid))))
            return bail(rc);
        std::vector<float> w((size_t)K * N, 0.0f);
        const double sd = std::sqrt(2.0 / real_k(l)) * (l == kNHid ? 0.1 : 1.0);
        for (int k = 0; k < real_k(l); k++)
            for (int j = 0; j < real_n(l); j++) {
                const double u1 = next(), u2 = next();
                w[(size_t)k * N + j] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
            }
        if (cudaMemcpyAsync(n->W[l], w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, n->stream) != cudaSuccess)
            return bail(nn_fail(DG_ERR_CUDA, "weight upload failed"));
    }
    for (int q = 0; q < kIn; q++) { n->sc.xmu[q] = 0.0f; n->sc.xsd[q] = 1.0f; n->sc.xisd[q] = 1.0f; }
    for (int q = 0; q < kOut; q++) n->sc.ysd[q] = 1.0f;
    if ((rc = nn_alloc_t(n, &n->d_sc, 1))) return bail(rc);
    if (cudaMemcpyAsync(n->d_sc, &n->sc, sizeof(Scaling), cudaMemcpyHostToDevice, n->stream) != cudaSuccess)
        return bail(nn_fail(DG_ERR_CUDA, "scaling upload failed"));
    for (int q = 0; q < kIn; q++) { n->gates.xmin[q] = -1e30f; n->gates.xmax[q] = 1e30f; }
    n->gates.ymax = 1e30f;
    n->gates.jump = 0.1f;
    n->gates.compress = 0.1f;
    n->gates.margin = 0.0f;
    if ((rc = pack_weights(n)) || (rc = nn_sync(n))) return bail(rc);
    *out = n;
    return DG_OK;
}

int dg_nn_destroy(dg_nn *n) {
    if (!n) return DG_OK;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    for (void *p : n->allocs) cudaFree(p);
    for (void *p : n->scratch) cudaFree(p);
    if (n->xs) cudaFree(n->xs);
    if (n->ts) cudaFree(n->ts);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return DG_OK;
}

int dg_nn_set_samples(dg_nn *n, const float *x, const float *t, long long count) {
    if (!n || !x || !t || count <= 0) return nn_fail(DG_ERR_ARG, "bad sample arguments");
    NN_CUDA(cudaSetDevice(n->device));
    int rc;
    if ((rc = dg_nn_reserve_samples(n, count))) return rc;
    NN_CUDA(cudaMemcpyAsync(n->xs, x, (size_t)count * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    NN_CUDA(cudaMemcpyAsync(n->ts, t, (size_t)count * kOut * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    n->ns = count;
    return nn_sync(n);
}

int dg_nn_reserve_samples(dg_nn *n, long long count) {
    if (!n || count <= 0) return nn_fail(DG_ERR_ARG, "bad sample count");
    if (count <= n->cap) return DG_OK;
    NN_CUDA(cudaSetDevice(n->device));
    NN_CUDA(cudaStreamSynchronize(n->stream));
    float *xs = nullptr, *ts = nullptr;
    NN_CUDA(cudaMalloc(&xs, (size_t)count * kIn * sizeof(float)));
    if (cudaMalloc(&ts, (size_t)count * kOut * sizeof(float)) != cudaSuccess) {
        cudaFree(xs);
        return nn_fail(DG_ERR_CUDA, "out of device memory for samples");
    }
    if (n->ns) {
        cudaMemcpyAsync(xs, n->xs, (size_t)n->ns * kIn * sizeof(float), cudaMemcpyDeviceToDevice, n->stream);
        cudaMemcpyAsync(ts, n->ts, (size_t)n->ns * kOut * sizeof(float), cudaMemcpyDeviceToDevice, n->stream);
        NN_CUDA(cudaStreamSynchronize(n->stream));
    }
    if (n->xs) cudaFree(n->xs);
    if (n->ts) cudaFree(n->ts);
    n->xs = xs;
    n->ts = ts;
    n->cap = count;
    return DG_OK;
}

long long dg_nn_sample_count(const dg_nn *n) { return n ? n->ns : 0; }

int dg_nn_samples_copy(dg_nn *n, long long first, long long count, float *x, float *t) {
    if (!n || first < 0 || count < 0 || first + count > n->ns || (!x && !t)) return nn_fail(DG_ERR_ARG, "bad sample range");
    NN_CUDA(cudaSetDevice(n->device));
    if (x) NN_CUDA(cudaMemcpyAsync(x, n->xs + first * kIn, (size_t)count * kIn * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    if (t) NN_CUDA(cudaMemcpyAsync(t, n->ts + first * kOut, (size_t)count * kOut * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    return nn_sync(n);
}

int dg_nn_train(dg_nn *n, int steps, int batch, float lr, float *loss_out) {
    if (!n || steps < 0) return nn_fail(DG_ERR_ARG, "bad training arguments");
    if (n->ns <= 0) return nn_fail(DG_ERR_ARG, "no samples");
    int rc;
    if ((rc = check_batch(batch))) return rc;
    NN_CUDA(cudaSetDevice(n->device));
    if ((rc = ensure_batch(n, batch))) return rc;
    for (int s = 0; s < steps; s++) {
        if ((rc = gather(n, batch, 1, 0)) || (rc = forward(n, batch)) || (rc = backward(n, batch, batch)) ||
            (rc = adam(n, batch, lr, 1, nullptr)))
            return rc;
    }
    if (loss_out) {
        std::vector<float> lp((size_t)batch / kTileRows);
        NN_CUDA(cudaMemcpyAsync(lp.data(), n->lpart, lp.size() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
        if ((rc = nn_sync(n))) return rc;
        double l = 0.0;
        for (float v : lp) l += v;
        *loss_out = (float)(l / ((double)batch * kOut));
    }
    n->trained = 1;
    return nn_sync(n);
}

int dg_nn_gradients(dg_nn *n, const float *x, const float *t, int batch, float *loss, float *grad) {
    if (!n || !x || !t || !grad) return nn_fail(DG_ERR_ARG, "bad gradient arguments");
    int rc;
    if ((rc = check_batch(batch))) return rc;
    NN_CUDA(cudaSetDevice(n->device));
    if ((rc = ensure_batch(n, batch))) return rc;
    // a private sample set holding exactly this batch, in order
    float *xs = n->xs, *ts = n->ts;
    const long long ns = n->ns, cap = n->cap;
    n->xs = nullptr; n->ts = nullptr; n->ns = 0; n->cap = 0;
    rc = dg_nn_set_samples(n, x, t, batch);
    if (!rc) rc = gather(n, batch, 0, 0);
    if (!rc) rc = forward(n, batch);
    if (!rc) rc = backward(n, batch, batch);
    if (!rc) rc = adam(n, batch, 0.0f, 0, n->gout);
    const long long np = dg_nn_param_count();
    if (!rc && cudaMemcpyAsync(grad, n->gout, (size_t)np * sizeof(float), cudaMemcpyDeviceToHost, n->stream) != cudaSuccess)
        rc = nn_fail(DG_ERR_CUDA, "gradient read-back failed");
    std::vector<float> lp((size_t)batch / kTileRows);
    if (!rc && cudaMemcpyAsync(lp.data(), n->lpart, lp.size() * sizeof(float), cudaMemcpyDeviceToHost, n->stream) != cudaSuccess)
        rc = nn_fail(DG_ERR_CUDA, "loss read-back failed");
    if (!rc) rc = nn_sync(n);
    if (n->xs) cudaFree(n->xs);
    if (n->ts) cudaFree(n->ts);
    n->xs = xs; n->ts = ts; n->ns = ns; n->cap = cap;
    if (!rc && loss) {
        double l = 0.0;
        for (float v : lp) l += v;
        *loss = (float)(l / ((double)batch * kOut));
    }
    return rc;
}

int dg_nn_forward(dg_nn *n, const float *x, long long count, float *y) {
    if (!n || !x || !y || count <= 0) return nn_fail(DG_ERR_ARG, "bad forward arguments");
    NN_CUDA(cudaSetDevice(n->device));
    const long long rows = n->bcap ? n->bcap : 16384;
    int rc;
    if ((rc = ensure_batch(n, rows))) return rc;
    float *xs = n->xs, *ts = n->ts;
    const long long ns = n->ns, cap = n->cap;
    n->xs = nullptr; n->ts = nullptr; n->ns = 0; n->cap = 0;
    std::vector<float> zeros((size_t)count * kOut, 0.0f);
    rc = dg_nn_set_samples(n, x, zeros.data(), count);
    for (long long first = 0; !rc && first < count; first += rows) {
        const long long m = std::min(rows, count - first);
        const long long r = (m + kTileRows - 1) / kTileRows * kTileRows;
        if (!rc) rc = gather(n, r, 0, first);
        if (!rc) rc = forward(n, r);
        if (!rc && cudaMemcpyAsync(y + first * kOut, n->Y, (size_t)m * kOut * sizeof(float), cudaMemcpyDeviceToHost,
                                   n->stream) != cudaSuccess)
            rc = nn_fail(DG_ERR_CUDA, "output read-back failed");
        if (!rc) rc = nn_sync(n);
        for (long long r2 = 0; !rc && r2 < m; r2++)
            for (int c = 0; c < kOut; c++) y[(first + r2) * kOut + c] *= n->sc.ysd[c];
    }
    if (n->xs) cudaFree(n->xs);
    if (n->ts) cudaFree(n->ts);
    n->xs = xs; n->ts = ts; n->ns = ns; n->cap = cap;
    return rc;
}

int dg_nn_get_params(dg_nn *n, float *host, long long count) {
    if (!n || !host || count < dg_nn_param_count()) return nn_fail(DG_ERR_ARG, "bad parameter buffer");
    NN_CUDA(cudaSetDevice(n->device));
    long long off = 0;
    for (int l = 0; l < kNL; l++) {
        const int K = layer_k(l), N = layer_n(l);
        std::vector<float> w((size_t)K * N), b(N);
        NN_CUDA(cudaMemcpyAsync(w.data(), n->W[l], w.size() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
        NN_CUDA(cudaMemcpyAsync(b.data(), n->b[l], b.size() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
        NN_CUDA(cudaStreamSynchronize(n->stream));
        for (int k = 0; k < real_k(l); k++)
            for (int j = 0; j < real_n(l); j++) host[off++] = w[(size_t)k * N + j];
        for (int j = 0; j < real_n(l); j++) host[off++] = b[j];
    }
    return DG_OK;
}

int dg_nn_set_params(dg_nn *n, const float *host, long long count) {
    if (!n || !host || count < dg_nn_param_count()) return nn_fail(DG_ERR_ARG, "bad parameter buffer");
    NN_CUDA(cudaSetDevice(n->device));
    long long off = 0;
    for (int l = 0; l < kNL; l++) {
        const int K = layer_k(l), N = layer_n(l);
        std::vector<float> w((size_t)K * N, 0.0f), b(N, 0.0f);
        for (int k = 0; k < real_k(l); k++)
            for (int j = 0; j < real_n(l); j++) w[(size_t)k * N + j] = host[off++];
        for (int j = 0; j < real_n(l); j++) b[j] = host[off++];
        NN_CUDA(cudaMemcpyAsync(n->W[l], w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, n->stream));
        NN_CUDA(cudaMemcpyAsync(n->b[l], b.data(), b.size() * sizeof(float), cudaMemcpyHostToDevice, n->stream));
        NN_CUDA(cudaStreamSynchronize(n->stream));
    }
    int rc = pack_weights(n);
    return rc ? rc : nn_sync(n);
}

// input envelope and output bound of the current samples become the confidence gate
int dg_nn_fit_envelope(dg_nn *n, float margin) {
    if (!n || n->ns <= 0) return nn_fail(DG_ERR_ARG, "no samples");
    NN_CUDA(cudaSetDevice(n->device));
    int *d = nullptr;
    NN_CUDA(cudaMalloc(&d, (2 * kIn + 1) * sizeof(int)));
    std::vector<int> init(2 * kIn + 1);
    for (int q = 0; q < kIn; q++) { init[q] = 0x7FFFFFFF; init[kIn + q] = (int)0x80000000; }
    init[2 * kIn] = 0;
    cudaMemcpyAsync(d, init.data(), init.size() * sizeof(int), cudaMemcpyHostToDevice, n->stream);
    k_envelope<<<296, 256, 0, n->stream>>>(n->xs, n->ts, n->ns, d, d + kIn, d + 2 * kIn);
    std::vector<int> h(2 * kIn + 1);
    cudaMemcpyAsync(h.data(), d, h.size() * sizeof(int), cudaMemcpyDeviceToHost, n->stream);
    const cudaError_t e = cudaStreamSynchronize(n->stream);
    cudaFree(d);
    if (e != cudaSuccess) return nn_fail(DG_ERR_CUDA, cudaGetErrorString(e));
    auto o2f_h = [](int i) { int j = i >= 0 ? i : i ^ 0x7FFFFFFF; float f; std::memcpy(&f, &j, 4); return f; };
    for (int q = 0; q < kIn; q++) { n->gates.xmin[q] = o2f_h(h[q]); n->gates.xmax[q] = o2f_h(h[kIn + q]); }
    n->gates.ymax = o2f_h(h[2 * kIn]);
    n->gates.margin = margin;
    return DG_OK;
}

int dg_nn_fit_scaling(dg_nn *n) {
    if (!n || n->ns <= 0) return nn_fail(DG_ERR_ARG, "no samples");
    NN_CUDA(cudaSetDevice(n->device));
    const int na = 2 * (kIn + kOut);
    double *d = nullptr;
    NN_CUDA(cudaMalloc(&d, na * sizeof(double)));
    cudaMemsetAsync(d, 0, na * sizeof(double), n->stream);
    k_moments<<<296, 128, 0, n->stream>>>(n->xs, n->ts, n->ns, d);
    std::vector<double> h(na);
    cudaMemcpyAsync(h.data(), d, na * sizeof(double), cudaMemcpyDeviceToHost, n->stream);
    const cudaError_t e = cudaStreamSynchronize(n->stream);
    cudaFree(d);
    if (e != cudaSuccess) return nn_fail(DG_ERR_CUDA, cudaGetErrorString(e));
    const double N = (double)n->ns;
    for (int q = 0; q < kIn; q++) {
        const double mu = h[q] / N, var = std::max(h[kIn + kOut + q] / N - mu * mu, 0.0);
        n->sc.xmu[q] = (float)mu;
        n->sc.xsd[q] = var > 1e-12 ? (float)std::sqrt(var) : 1.0f;  // a constant input stays at zero
        n->sc.xisd[q] = 1.0f / n->sc.xsd[q];
    }
    for (int q = 0; q < kOut; q++) {
        const double rms = std::sqrt(h[2 * kIn + kOut + q] / N);
        n->sc.ysd[q] = rms > 1e-30 ? (float)rms : 1.0f;
    }
    NN_CUDA(cudaMemcpyAsync(n->d_sc, &n->sc, sizeof(Scaling), cudaMemcpyHostToDevice, n->stream));
    return nn_sync(n);
}

int dg_nn_set_gates(dg_nn *n, float jump, float compress) {
    if (!n || !(jump >= 0.0f) || !(compress >= 0.0f)) return nn_fail(DG_ERR_ARG, "bad gate thresholds");
    n->gates.jump = jump;
    n->gates.compress = compress;
    return DG_OK;
}

}  // extern "C"

// ---- internal accessors for the step kernels (nn_host.h) ---------------------------
int dg_nn_view(const dg_nn *n, dg::nn::NetView *v) {
    if (!n) return DG_ERR_ARG;
    for (int l = 0; l < kNL; l++) { v->wt[l] = n->Wt[l]; v->b[l] = n->b[l]; }
    for (int l = 0; l < kNHid; l++) v->bt[l] = n->Bt[l];
    v->gates = n->gates;
    v->sc = n->sc;
    return DG_OK;
}
int dg_nn_device(const dg_nn *n) { return n ? n->device : -1; }
float *dg_nn_sample_x(dg_nn *n) { return n->xs; }
float *dg_nn_sample_t(dg_nn *n) { return n->ts; }
void dg_nn_set_count(dg_nn *n, long long c) { n->ns = c; }
