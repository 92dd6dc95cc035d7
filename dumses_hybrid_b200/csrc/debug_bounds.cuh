// Host side of the bounds-checked build (-DDG_CHECK_BOUNDS): the table of device buffers the
// kernels of this translation unit may touch (every buffer of every live context, registered
// by dg_init and removed by dg_finalize), and the count of accesses that fell outside it.
// Included at namespace dg::<arithmetic> scope after the kernels (step_impl.cuh includes the
// standard headers it needs); a no-op in normal builds.
#pragma once

#ifdef DG_CHECK_BOUNDS
namespace {
std::vector<std::pair<const char *, const char *>> g_host_bufs;
int upload_buffer_table() {
    const char *lo[kMaxBufs] = {}, *hi[kMaxBufs] = {};
    const int n = (int)(g_host_bufs.size() < (size_t)kMaxBufs ? g_host_bufs.size() : (size_t)kMaxBufs);
    for (int b = 0; b < n; b++) {
        lo[b] = g_host_bufs[b].first;
        hi[b] = g_host_bufs[b].second;
    }
    if (cudaMemcpyToSymbol(g_buf_lo, lo, sizeof lo) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(g_buf_hi, hi, sizeof hi) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(g_nbuf, &n, sizeof n) != cudaSuccess) return -1;
    return g_host_bufs.size() > (size_t)kMaxBufs ? -1 : 0;
}
}  // namespace
int debug_register(const void *p, size_t bytes, int add) {
    if (!p) return 0;
    const char *lo = (const char *)p, *hi = lo + bytes;
    if (add) {
        g_host_bufs.emplace_back(lo, hi);
    } else {
        for (size_t b = 0; b < g_host_bufs.size(); b++)
            if (g_host_bufs[b].first == lo) {
                g_host_bufs.erase(g_host_bufs.begin() + (long)b);
                break;
            }
    }
    return upload_buffer_table();
}
long long debug_oob() {
    unsigned long long v = 0;
    if (cudaMemcpyFromSymbol(&v, g_oob, sizeof v) != cudaSuccess) return -2;
    return (long long)v;
}
#else
int debug_register(const void *, size_t, int) { return 0; }
long long debug_oob() { return -1; }
#endif
