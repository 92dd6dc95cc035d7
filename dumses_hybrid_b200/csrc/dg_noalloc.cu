// History sums of a caller-owned device state without any device allocation.
//
// Who needs it: a Fortran driver that keeps uin in its OpenACC runtime's
// present table hands the library device pointers from
// `!$acc host_data use_device(uin)`; it must not create a library context, which
// would cudaMalloc a second copy of the state plus the work arrays of a step, and
// some production jobs run under a device-memory budget that forbids allocation
// after start-up.  For them this entry point computes the MRI history sums of
// src/problem/mri/history.f90:60-125 directly from their array, with the caller's
// output buffer, and keeps its reduction scratch (per-column yz means and
// per-block partial sums) in the file-scope array below.
#include <mutex>
#include <string>

#include "dumses_gpu.h"
#include "mhd_kernels.cuh"

namespace {

// Largest nx accepted; the scratch holds 2*nx column means and the block partials.
constexpr int kNoAllocMaxNx = DG_HISTORY_NOALLOC_MAX_NX;
constexpr long long kScratchDoubles = 2LL * kNoAllocMaxNx + 8LL * 296 + 64;

// One copy per GPU that loads the library, kept until the process exits.
static __device__ __align__(256) double g_history_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// the pointer must be device (or managed) memory that the current device can use
bool on_device(const void *ptr, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();  // an unrecognised pointer leaves a non-sticky error: clear only that one
        return false;
    }
    if (a.type == cudaMemoryTypeDevice) return a.device == dev;
    return a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int dg_history_noalloc(const dg_params *p, const double *uin_dev, double *out_dev, void *stream) {
    if (!p || !uin_dev || !out_dev) return dg::set_error(DG_ERR_ARG, "null argument");
    if (p->ndim != 3) return dg::set_error(DG_ERR_UNSUPPORTED, "the MRI history is defined for ndim = 3");
    if (p->nx < 3 || p->ny < 3 || p->nz < 3) return dg::set_error(DG_ERR_ARG, "nx, ny and nz must be >= 3");
    if (!(p->xmax > p->xmin) || !(p->ymax > p->ymin) || !(p->zmax > p->zmin))
        return dg::set_error(DG_ERR_ARG, "dg_history_noalloc: empty domain");
    if (p->nx > kNoAllocMaxNx)
        return dg::set_error(DG_ERR_ARG, "dg_history_noalloc: nx exceeds DG_HISTORY_NOALLOC_MAX_NX");
    // an error the caller's own code left pending is theirs to read: report it without clearing it
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        return dg::set_error(DG_ERR_CUDA, (std::string("dg_history_noalloc: a CUDA error is already pending: ") +
                                           cudaGetErrorString(pending)).c_str());
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return dg::set_error(DG_ERR_NODEVICE, "dg_history_noalloc: no usable current CUDA device");
    if (!on_device(uin_dev, dev) || !on_device(out_dev, dev))
        return dg::set_error(DG_ERR_ARG, "dg_history_noalloc: uin_dev and out_dev must be device or managed memory "
                                         "of the current device (a host array needs `host_data use_device`)");
    double *scratch = nullptr;
    {
        // set-up, once per device, on the caller's current device
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            cudaError_t e = cudaGetSymbolAddress((void **)&g_scratch_ptr[dev], g_history_scratch);
            if (e != cudaSuccess) {
                g_scratch_ptr[dev] = nullptr;
                return dg::set_error(DG_ERR_CUDA, cudaGetErrorString(e));
            }
        }
        scratch = g_scratch_ptr[dev];
    }
    const dg::Geo G = dg::make_geo(*p);
    if (dg::f64::history_scratch_doubles(G) > kScratchDoubles)
        return dg::set_error(DG_ERR_ARG, "dg_history_noalloc: scratch too small for this grid");
    const cudaStream_t st = (cudaStream_t)stream;
    // The bounds-checked build (debug_oob() >= 0) checks every access against a table of known
    // buffers: the caller's arrays and the scratch join it for this call, which then waits for
    // its kernels before they leave it again.
    const bool checked = dg::f64::debug_oob() >= 0;
    const size_t uin_bytes = (size_t)G.sv * 11 * sizeof(double);
    if (checked) {
        dg::f64::debug_register(uin_dev, uin_bytes, 1);
        dg::f64::debug_register(out_dev, 9 * sizeof(double), 1);
        dg::f64::debug_register(scratch, kScratchDoubles * sizeof(double), 1);
    }
    dg::f64::launch_history_ptrs(G, uin_dev, scratch, out_dev, st);
    cudaError_t e = cudaPeekAtLastError();
    if (checked) {
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        dg::f64::debug_register(scratch, 0, 0);
        dg::f64::debug_register(out_dev, 0, 0);
        dg::f64::debug_register(uin_dev, 0, 0);
    }
    if (e != cudaSuccess) return dg::set_error(DG_ERR_CUDA, cudaGetErrorString(e));
    return DG_OK;
}
