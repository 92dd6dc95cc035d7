// sm_100a building blocks of the flux-surrogate network: BF16 tcgen05 MMAs with FP32
// accumulators in tensor memory, operands staged in shared memory by bulk copies, and
// mbarrier waits that give up after a bounded time.
//
// Operand layout ("blocked K-major"): a matrix X with R rows and C reduction columns
// (C a multiple of 8) is stored as [R / RT][C / 8][RT][8] BF16, RT = min(R, 128) rows
// per tile.  One 16-byte group holds 8 consecutive reduction elements of one row, so
// 8 rows x 16 B form the 128-byte core matrix of the tcgen05 no-swizzle K-major layout:
// in shared memory a tile [C / 8][RT][8] has its 8-row groups 128 B apart (SBO) and its
// 8-column chunks RT * 16 B apart (LBO), and any run of whole chunks of one row tile is
// one contiguous block of global memory, copied with one cp.async.bulk.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace dg {
namespace nn {

constexpr int kTileRows = 128;               // rows per tcgen05 tile (cta_group::1, M = 128)
constexpr unsigned long long kWaitNs = 1000000000ull;  // an mbarrier wait gives up after 1 s (%globaltimer)

// error bits written to the network's device error word
enum { NN_ERR_WAIT = 1 };

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// poll the phase with the given parity; false when kWaitNs ran out first
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    const uint32_t a = smem_addr(bar);
    const unsigned long long t0 = global_ns();
    for (unsigned n = 1;; n++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((n & 255) == 0 && global_ns() - t0 > kWaitNs) return false;
    }
}

// ---- bulk copy global -> shared (contiguous, 16-byte aligned, size % 16 == 0) -----
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// make generic-proxy shared-memory writes visible to the tensor-core (async) proxy
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- tensor memory --------------------------------------------------------
// one warp allocates `cols` columns (power of two >= 32); the address lands in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, unsigned cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, unsigned cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor, no swizzle, K-major (version 1 for sm_100)
__device__ __forceinline__ uint64_t sdesc(const void *tile, unsigned lbo_bytes, unsigned sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr(tile) >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version
    return d;                // base offset 0, LBO mode 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4)                       // D format F32
           | (1u << 7)                     // A format BF16
           | (1u << 10)                    // B format BF16
           | ((uint32_t)(n >> 3) << 17)    // N / 8
           | ((uint32_t)(m >> 4) << 24);   // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, one K = 16 step, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
// arrive on `bar` once all previously issued MMAs of this thread have completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane (warp w of the
// warpgroup reads lanes 32w .. 32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int n = 0; n < 16; n++) v[n] = __uint_as_float(r[n]);
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int n = 0; n < 32; n++) v[n] = __uint_as_float(r[n]);
}

// K-major MMA sequence over a staged pair of tiles: A tile [k/8][128][8], B tile [k/8][nrows][8]
// (nrows = N of the MMA), `ksteps` steps of K = 16 (two 8-column chunks each)
__device__ __forceinline__ void mma_tiles(uint32_t d_tmem, const void *a_tile, const void *b_tile, int n, int ksteps,
                                          int acc_first) {
    const uint32_t id = idesc_bf16(kTileRows, n);
    const unsigned a_lbo = kTileRows * 16, b_lbo = (unsigned)n * 16;
    for (int s = 0; s < ksteps; s++) {
        const char *a = (const char *)a_tile + (size_t)s * 2 * a_lbo;
        const char *b = (const char *)b_tile + (size_t)s * 2 * b_lbo;
        mma_bf16(d_tmem, sdesc(a, a_lbo, 128), sdesc(b, b_lbo, 128), id, (s > 0) || acc_first);
    }
}

// one more K = 16 step over a second pair of tiles (A [2][128][8], B [2][n][8]), accumulating
__device__ __forceinline__ void mma_extra_step(uint32_t d_tmem, const void *a_tile, const void *b_tile, int n) {
    mma_bf16(d_tmem, sdesc(a_tile, kTileRows * 16, 128), sdesc(b_tile, (unsigned)n * 16, 128), idesc_bf16(kTileRows, n), 1);
}

// blocked K-major element offset of (row r, column c) for a matrix with C reduction columns
__host__ __device__ __forceinline__ long long blk_off(long long r, int c, int C, int RT) {
    return ((r / RT) * (C / 8) + c / 8) * (long long)RT * 8 + (r % RT) * 8 + (c % 8);
}

}  // namespace nn
}  // namespace dg
