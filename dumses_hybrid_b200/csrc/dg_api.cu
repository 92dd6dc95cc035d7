// C-ABI of libdumses_gpu (declarations and reference mapping in include/dumses_gpu.h).
//
// One context owns the device state of one grid: two state buffers used in
// ping-pong (each step reads one and writes the other), the work arrays of the
// step, and a CUDA stream.  Device scalars (dt, time, CFL minimum, error word)
// stay on the device so that whole steps can be enqueued back to back.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>

#include <vector>

#include "dumses_gpu.h"
#include "dump_io.h"
#include "mhd_kernels.cuh"
#include "nn_host.h"

namespace {
// CUDA-event timing of every kernel the context enqueues, on the context's stream
struct EventTimer : dg::KernelTimer {
    struct Rec { int slot; cudaEvent_t a, b; };
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> recs;
    cudaEvent_t pending = nullptr;
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int, cudaStream_t st) override { pending = get(); cudaEventRecord(pending, st); }
    void end(int slot, cudaStream_t st) override {
        cudaEvent_t b = get();
        cudaEventRecord(b, st);
        recs.push_back({slot, pending, b});
        pending = nullptr;
    }
    ~EventTimer() override {
        for (auto &r : recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        for (auto e : pool) cudaEventDestroy(e);
    }
};
const char *kSlotNames[dg::KS_COUNT] = {"scalars", "cfl_dt", "primitive", "trace", "riemann_flux_emf", "update_ct",
                                       "fargo_emf", "fargo_update", "boundary", "history", "right_faces", "edge_efield",
                                       "nn_faces", "nn_fallback", "dissipation"};
}  // namespace

namespace {
// the launch set of one arithmetic
struct Launches {
    int (*set_scalars)(const dg::Bufs &, double, double, int, int, cudaStream_t);
    int (*advance_time)(const dg::Bufs &, cudaStream_t);
    int (*dt)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*godunov)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*fargo)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*boundary)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*history)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t, int);
    int (*history_columns)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*history_share)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*dissipation)(const dg::Geo &, const dg::Bufs &, int, cudaStream_t);
    int (*right_faces)(const dg::Geo &, const dg::Bufs &, int, double *, cudaStream_t);
    int (*to_f64)(const dg::Geo &, const dg::Bufs &, int, double *, cudaStream_t);
    int (*from_f64)(const dg::Geo &, const dg::Bufs &, int, const double *, int, cudaStream_t);
};
#define DG_LAUNCH_TABLE(ns)                                                                                  \
    Launches{ns::launch_set_scalars, ns::launch_advance_time, ns::launch_dt, ns::launch_godunov, ns::launch_fargo, \
             ns::launch_boundary, ns::launch_history, ns::launch_history_columns, ns::launch_history_share,   \
             ns::launch_dissipation, ns::launch_right_faces,                                                 \
             ns::launch_state_to_f64, ns::launch_f64_to_state}
const Launches kLaunchF64 = DG_LAUNCH_TABLE(dg::f64);
const Launches kLaunchF32 = DG_LAUNCH_TABLE(dg::f32);
}  // namespace

namespace dg {
thread_local KernelTimer *g_timer = nullptr;
// stored state planes: the 8 variables, plus the right-face B copies the reference never
// refreshes (z in 2D; y and z in 1D), frozen at their initial values
int nstate_vars(const Geo &G) { return G.ndim == 3 ? 8 : G.ndim == 2 ? 9 : 10; }
}  // namespace dg

struct dg_ctx {
    dg_params p;
    dg::Geo G;
    dg::Bufs B;
    const Launches *L = &kLaunchF64;
    size_t es = 8;  // bytes per element of the work arrays
    int cur = 0;
    int nv = 8;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    dg::Scalars *h_scal = nullptr;  // pinned read-back of the device scalars
    double *h_hist = nullptr;       // pinned read-back of history sums
    size_t bytes = 0;
    std::vector<std::pair<void *, size_t>> allocations;  // every device buffer, for the checked build
    EventTimer *timer = nullptr;    // non-null while per-kernel profiling is on
    long long version = 0;          // bumped by every call that changes the device state
    long long q_version = -1;       // state version whose primitive variables the CFL pass left in Q
    dg_nn *nn = nullptr;            // attached flux network (surrogate = 1)
    dg::nn::NetView view{};         // its device view, as of dg_attach_surrogate
};

namespace {
// attach the context's timer (if any) to the launches of the current call
struct TimerScope {
    explicit TimerScope(dg_ctx *c) { dg::g_timer = c ? c->timer : nullptr; }
    ~TimerScope() { dg::g_timer = nullptr; }
};
}  // namespace

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

#define DG_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

double sync_timeout_s() {
    const char *e = std::getenv("DG_SYNC_TIMEOUT_S");
    if (e) {
        double v = std::atof(e);
        if (v > 0) return v;
    }
    return 300.0;
}

// wait for the stream with a wall-clock bound instead of blocking forever
int bounded_sync(cudaStream_t s) {
    const double limit = sync_timeout_s();
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return DG_OK;
        if (e != cudaErrorNotReady) return fail(DG_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return fail(DG_ERR_TIMEOUT, "device work did not finish within DG_SYNC_TIMEOUT_S");
        std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 5 : 200));
    }
}

// wait for an event with the same wall-clock bound
int bounded_event(cudaEvent_t ev) {
    const double limit = sync_timeout_s();
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return DG_OK;
        if (e != cudaErrorNotReady) return fail(DG_ERR_CUDA, std::string("event: ") + cudaGetErrorString(e));
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return fail(DG_ERR_TIMEOUT, "device work did not finish within DG_SYNC_TIMEOUT_S");
        std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 5 : 200));
    }
}

int check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(DG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return DG_OK;
}

int validate(const dg_params *p) {
    if (!p) return fail(DG_ERR_ARG, "null parameters");
    if (p->ndim < 1 || p->ndim > 3) return fail(DG_ERR_UNSUPPORTED, "ndim must be 1, 2 or 3");
    if (p->ndim == 1) {
        if (p->ny != 1 || p->nz != 1) return fail(DG_ERR_ARG, "ny and nz must be 1 when ndim = 1");
        if (p->precision != DG_PREC_FP64) return fail(DG_ERR_UNSUPPORTED, "ndim = 1 runs the FP64 path only");
        if (p->slope_type > 2) return fail(DG_ERR_UNSUPPORTED, "ndim = 1 takes slope_type 0, 1 or 2 (scheme.f90:313-315)");
        if (p->nu > 0.0 || p->eta > 0.0) return fail(DG_ERR_UNSUPPORTED, "dissipation with ndim = 1 is not built");
    }
    if (p->nx < 3 || (p->ndim > 1 && p->ny < 3))
        return fail(DG_ERR_ARG, "nx (and ny with ndim > 1) must be >= 3 (three ghost layers are copied)");
    if (p->ndim == 3 && p->nz < 3) return fail(DG_ERR_ARG, "nz must be >= 3 when ndim = 3");
    if (p->ndim == 2 && p->nz != 1) return fail(DG_ERR_ARG, "nz must be 1 when ndim = 2");
    if (!(p->xmax > p->xmin) || !(p->ymax > p->ymin) || !(p->zmax > p->zmin)) return fail(DG_ERR_ARG, "empty domain");
    if (!(p->courant > 0)) return fail(DG_ERR_ARG, "courant must be > 0");
    if (p->iso && !(p->ciso > 0)) return fail(DG_ERR_ARG, "isothermal EOS needs ciso > 0");
    if (!p->iso && !(p->gamma > 1)) return fail(DG_ERR_ARG, "adiabatic EOS needs gamma > 1");
    if (p->slope_type < 0 || p->slope_type > 3) return fail(DG_ERR_ARG, "slope_type must be 0..3");
    if (p->iriemann != DG_RIEMANN_LLF && p->iriemann != DG_RIEMANN_HLL && p->iriemann != DG_RIEMANN_HLLD &&
        p->iriemann != DG_RIEMANN_UPWIND)
        return fail(DG_ERR_UNSUPPORTED, "iriemann must be llf, hll, hlld or upwind");
    if (p->iriemann2d != DG_RIEMANN_LLF && p->iriemann2d != DG_RIEMANN_HLLD && p->iriemann2d != DG_RIEMANN_UPWIND &&
        p->iriemann2d != DG_RIEMANN_HLLA)
        return fail(DG_ERR_UNSUPPORTED, "iriemann2d must be llf, hlld, upwind or hlla");
    for (int d = 0; d < 3; d++)
        if (p->bc[d] < DG_BC_PERIODIC || p->bc[d] > DG_BC_SHEARINGBOX) return fail(DG_ERR_ARG, "unknown boundary type");
    if (p->bc[1] == DG_BC_SHEARINGBOX || p->bc[2] == DG_BC_SHEARINGBOX)
        return fail(DG_ERR_UNSUPPORTED, "the shearing box is an x boundary");
    if (p->bc[0] == DG_BC_SHEARINGBOX && p->ndim != 3)
        return fail(DG_ERR_UNSUPPORTED, "the shearing-box boundary exists for ndim = 3 only (boundary.f90:40)");
    if (p->bc[0] == DG_BC_SHEARINGBOX && p->bc[1] != DG_BC_PERIODIC)
        return fail(DG_ERR_UNSUPPORTED, "the shearing box needs a periodic y direction");
    if (p->fargo && (p->ndim != 3 || p->bc[1] != DG_BC_PERIODIC))
        return fail(DG_ERR_UNSUPPORTED, "FARGO needs ndim = 3 and a periodic y direction");
    if (p->precision != DG_PREC_FP64 && p->precision != DG_PREC_FP32) return fail(DG_ERR_ARG, "unknown precision");
    if (p->surrogate && p->precision != DG_PREC_FP32) return fail(DG_ERR_UNSUPPORTED, "the flux surrogate needs the FP32 path");
    if (!(p->nu >= 0.0) || !(p->eta >= 0.0)) return fail(DG_ERR_ARG, "nu and eta must be >= 0");
    if (p->surrogate && p->iriemann != DG_RIEMANN_HLLD)
        return fail(DG_ERR_UNSUPPORTED, "the flux surrogate stands in for HLLD (iriemann = hlld)");
    // the kernels index cells, faces and edges with 32-bit linear indices
    if ((double)(p->nx + 6) * (p->ndim > 1 ? p->ny + 6 : 1) * (p->ndim == 3 ? p->nz + 6 : 1) >= 2147483647.0)
        return fail(DG_ERR_UNSUPPORTED, "grid too large: (nx+6)(ny+6)(nz+6) must stay below 2^31 cells");
    if (p->nzslice < 0) return fail(DG_ERR_ARG, "nzslice must be >= 0");
    if (p->nzslice > 1) {
        if (p->ndim != 3) return fail(DG_ERR_UNSUPPORTED, "a z-slab decomposition needs ndim = 3");
        if (p->zposition < 0 || p->zposition >= p->nzslice) return fail(DG_ERR_ARG, "zposition must be in [0, nzslice)");
        if (p->bc[2] != DG_BC_PERIODIC && p->bc[2] != DG_BC_ZERO_GRADIENT)
            return fail(DG_ERR_UNSUPPORTED, "z slabs need a periodic or zero-gradient z boundary");
    } else if (p->zposition != 0) {
        return fail(DG_ERR_ARG, "zposition must be 0 without a z-slab decomposition");
    }
    return DG_OK;
}

}  // namespace

dg::Geo dg::make_geo(const dg_params &p) {
    dg::Geo G{};
    G.ndim = p.ndim; G.nx = p.nx; G.ny = p.ny; G.nz = p.nz;
    G.NX = p.nx + 6;
    G.NY = p.ndim > 1 ? p.ny + 6 : 1;
    G.NZ = p.ndim == 3 ? p.nz + 6 : 1;
    G.gy = p.ndim > 1 ? 3 : 0;
    G.gz = p.ndim == 3 ? 3 : 0;
    G.sy = G.NX;
    G.sz = (long long)G.NX * G.NY;
    G.sv = G.sz * G.NZ;
    G.CX = p.nx + 2; G.CY = p.ndim > 1 ? p.ny + 2 : 1;
    G.CZ = p.ndim == 3 ? p.nz + 2 : 1;
    G.kc0 = p.ndim == 3 ? 0 : 1;
    G.csz = (long long)G.CX * G.CY * G.CZ;
    G.FX = p.nx + 1; G.FY = p.ndim > 1 ? p.ny + 1 : 1;
    G.FZ = p.ndim == 3 ? p.nz + 1 : 1;
    G.fsz = (long long)G.FX * G.FY * G.FZ;
    G.EX = p.nx + 3; G.EY = p.ndim > 1 ? p.ny + 3 : 1;
    G.EZ = p.ndim == 3 ? p.nz + 3 : 1;
    G.ke0 = p.ndim == 3 ? 0 : 1;
    G.esz = (long long)G.EX * G.EY * G.EZ;
    // init_grid (init.f90:447-449), single rank
    G.dx = (p.xmax - p.xmin) / p.nx;
    G.dy = (p.ymax - p.ymin) / p.ny;
    // a z slab's dz is that of the whole box, (zmax - zmin) / nzglob (init.f90:447-449)
    G.nzslice = p.nzslice > 1 ? p.nzslice : 1;
    G.zposition = p.nzslice > 1 ? p.zposition : 0;
    G.dz = (p.zmax - p.zmin) / (p.nz * G.nzslice);
    G.xmin = p.xmin; G.xmax = p.xmax; G.ymin = p.ymin; G.ymax = p.ymax; G.zmin = p.zmin; G.zmax = p.zmax;
    G.gamma = p.gamma; G.ciso = p.ciso; G.omega0 = p.omega0; G.courant = p.courant;
    G.nu = p.nu; G.eta = p.eta;
    G.iso = p.iso; G.slope_type = p.slope_type; G.iriemann = p.iriemann; G.iriemann2d = p.iriemann2d;
    G.fargo = p.fargo;
    G.shearing = (p.bc[0] == DG_BC_SHEARINGBOX);
    for (int d = 0; d < 3; d++) G.bc[d] = p.bc[d];
    // slab sides: a neighbour's halo, except a zero-gradient box edge, which the slab fills itself
    G.bcz_lo = G.bcz_hi = p.bc[2];
    if (G.nzslice > 1) {
        G.bcz_lo = (p.bc[2] == DG_BC_ZERO_GRADIENT && G.zposition == 0) ? DG_BC_ZERO_GRADIENT : dg::kBcHalo;
        G.bcz_hi = (p.bc[2] == DG_BC_ZERO_GRADIENT && G.zposition == G.nzslice - 1) ? DG_BC_ZERO_GRADIENT : dg::kBcHalo;
    }
    // dividers of the linear index spaces (every space has fewer than 2^31 points: validate)
    G.dFX = dg::make_fastdiv((unsigned)G.FX); G.dFY = dg::make_fastdiv((unsigned)G.FY);
    G.dFZ = dg::make_fastdiv((unsigned)G.FZ);
    G.dCX = dg::make_fastdiv((unsigned)G.CX); G.dCY = dg::make_fastdiv((unsigned)G.CY);
    G.dEX = dg::make_fastdiv((unsigned)G.EX); G.dEY = dg::make_fastdiv((unsigned)G.EY);
    G.dPX = dg::make_fastdiv((unsigned)(p.nx + 5)); G.dPY = dg::make_fastdiv((unsigned)(p.ndim > 1 ? p.ny + 5 : 1));
    // smallp = smallr smallc^2 / gamma, as the trace and the solvers form it (trace3d, solver.f90)
    G.smallp = dg::kSmallr * (dg::kSmallc * dg::kSmallc) / p.gamma;
    G.dvloc = 1.0 / (G.dx * G.dy * G.dz);
    G.entho = 1.0 / (p.gamma - 1.0);
    G.rdx = 1.0 / G.dx; G.rdy = 1.0 / G.dy; G.rdz = 1.0 / G.dz;
    auto pow2 = [](double d) { int e; return d > 0.0 && std::frexp(d, &e) == 0.5 && e > -1000 && e < 1000; };
    G.p2x = pow2(G.dx); G.p2y = pow2(G.dy); G.p2z = pow2(G.dz);
    // ndim_act, init.f90:203-213
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    if ((nx == 1 && ny == 1) || (nx == 1 && nz == 1) || (ny == 1 && nz == 1)) G.ndim_act = 1;
    else if ((nx == 1 && ny > 1 && nz > 1) || (nx > 1 && ny == 1 && nz > 1) || (nx > 1 && ny > 1 && nz == 1)) G.ndim_act = 2;
    else G.ndim_act = 3;
    return G;
}

int dg::set_error(int code, const char *msg) { return fail(code, msg); }

namespace {

int alloc_bytes(dg_ctx *c, void **p, size_t b) {
    cudaError_t e = cudaMalloc(p, b);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(DG_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(b) + " bytes: " + cudaGetErrorString(e));
    }
    c->bytes += b;
    c->allocations.emplace_back(*p, b);
    DG_CUDA(cudaMemsetAsync(*p, 0, b, c->stream));
    return DG_OK;
}
int alloc(dg_ctx *c, double **p, size_t n) { return alloc_bytes(c, (void **)p, n * sizeof(double)); }
int alloc_w(dg_ctx *c, void **p, size_t n) { return alloc_bytes(c, p, n * c->es); }

int read_scalars(dg_ctx *c) {
    DG_CUDA(cudaMemcpyAsync(c->h_scal, c->B.S, sizeof(dg::Scalars), cudaMemcpyDeviceToHost, c->stream));
    int rc = bounded_sync(c->stream);
    if (rc) return rc;
    if (c->h_scal->err) {
        int e = c->h_scal->err;
        c->h_scal->err = 0;
        DG_CUDA(cudaMemsetAsync(&c->B.S->err, 0, sizeof(int), c->stream));
        if (e == DG_ERR_DT) return fail(e, "CFL reduction produced dt <= 0 or a non-finite dt");
        return fail(e, "non-finite or non-physical state met in the CFL reduction");
    }
    return DG_OK;
}

}  // namespace

extern "C" {

void dg_default_params(dg_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // default_parameters, init.f90:244-302
    p->ndim = 3; p->iso = 0;
    p->nx = 256; p->ny = 256; p->nz = 256;
    p->xmin = 0.0; p->xmax = 1.0; p->ymin = -0.5; p->ymax = 0.5; p->zmin = 0.0; p->zmax = 1.0;
    p->gamma = 5.0 / 3.0; p->ciso = 0.0; p->omega0 = 0.0; p->courant = 0.7;
    p->slope_type = 2; p->iriemann = DG_RIEMANN_HLLD; p->iriemann2d = DG_RIEMANN_HLLD;
    p->bc[0] = p->bc[1] = p->bc[2] = DG_BC_PERIODIC;
    p->fargo = 0; p->precision = DG_PREC_FP64; p->surrogate = 0; p->device = 0;
}

long long dg_uin_size(const dg_params *p) {
    if (!p) return 0;
    long long nx = p->nx + 6, ny = p->ndim > 1 ? p->ny + 6 : 1, nz = p->ndim == 3 ? p->nz + 6 : 1;
    return nx * ny * nz * 11;
}

const char *dg_last_error(void) { return g_last_error.c_str(); }

int dg_init(const dg_params *p, dg_ctx **out) {
    if (!out) return fail(DG_ERR_ARG, "null context pointer");
    *out = nullptr;
    int rc = validate(p);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(DG_ERR_NODEVICE, "no CUDA device visible");
    if (p->device < 0 || p->device >= ndev) return fail(DG_ERR_ARG, "device ordinal out of range");
    DG_CUDA(cudaSetDevice(p->device));
    dg_ctx *c = new dg_ctx();
    c->p = *p;
    c->G = dg::make_geo(*p);
    c->nv = dg::nstate_vars(c->G);
    std::memset(&c->B, 0, sizeof(c->B));
    c->B.nv = c->nv;
    c->B.sv = c->G.sv;
    if (p->precision == DG_PREC_FP32) { c->L = &kLaunchF32; c->es = 4; }
    auto bail = [&](int code) { dg_finalize(c); return code; };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(DG_ERR_CUDA, "cudaStreamCreate failed"));
    const dg::Geo &G = c->G;
    const size_t nt = (size_t)G.sv;
    // the state takes 8 bytes per variable and cell in both paths (FP64, or an FP32 hi/lo pair)
    if ((rc = alloc(c, (double **)&c->B.U[0], nt * c->nv))) return bail(rc);
    if ((rc = alloc(c, (double **)&c->B.U[1], nt * c->nv))) return bail(rc);
    if (p->precision == DG_PREC_FP32 && (rc = alloc(c, &c->B.stage, nt * c->nv))) return bail(rc);
    if ((rc = alloc_w(c, &c->B.Q, nt * 8))) return bail(rc);
    const int ncore = p->ndim == 3 ? dg::kCore3 : dg::kCore2;
    if ((rc = alloc_w(c, &c->B.core, (size_t)dg::core_elems(G.csz, ncore)))) return bail(rc);
    for (int d = 0; d < p->ndim; d++)
        if ((rc = alloc_w(c, &c->B.flx[d], (size_t)G.fsz * (p->ndim == 1 ? dg::kFluxRec1 : dg::kFluxComp))))
            return bail(rc);
    for (int d = 0; d < 3; d++) {
        if (p->ndim == 1 || (p->ndim == 2 && d < 2)) continue;
        if ((rc = alloc_w(c, &c->B.emf[d], (size_t)G.fsz))) return bail(rc);
    }
    for (int d = 0; d < 3; d++) {
        if (p->ndim == 1 || (p->ndim == 2 && d < 2)) continue;
        if ((rc = alloc_w(c, &c->B.E[d], (size_t)G.esz))) return bail(rc);
    }
    if (p->fargo)
        for (int d = 0; d < 2; d++)
            if ((rc = alloc(c, &c->B.femf[d], (size_t)G.fsz))) return bail(rc);
    if (p->surrogate) {
        for (int d = 0; d < p->ndim; d++)
            if ((rc = alloc_bytes(c, (void **)&c->B.fb_list[d], (size_t)G.fsz * sizeof(int)))) return bail(rc);
        if ((rc = alloc_bytes(c, (void **)&c->B.nn_count, 8 * sizeof(unsigned long long)))) return bail(rc);
        c->B.nn_err = (int *)(c->B.nn_count + 2);
    }
    if ((rc = alloc(c, &c->B.part, (size_t)(2 * p->nx + 8 * 296 + 64)))) return bail(rc);
    if ((rc = alloc(c, &c->B.hist, 16))) return bail(rc);
    {
        cudaError_t e = cudaMalloc((void **)&c->B.S, sizeof(dg::Scalars));
        if (e != cudaSuccess) return bail(fail(DG_ERR_NOMEM, "cudaMalloc of the device scalars failed"));
        cudaMemsetAsync(c->B.S, 0, sizeof(dg::Scalars), c->stream);
    }
    if (cudaMallocHost((void **)&c->h_scal, sizeof(dg::Scalars)) != cudaSuccess ||
        cudaMallocHost((void **)&c->h_hist, 16 * sizeof(double)) != cudaSuccess)
        return bail(fail(DG_ERR_NOMEM, "cudaMallocHost failed"));
    if ((rc = bounded_sync(c->stream))) return bail(rc);
    for (auto &a : c->allocations) {  // no-ops unless the library is the bounds-checked build
        dg::f64::debug_register(a.first, a.second, 1);
        dg::f32::debug_register(a.first, a.second, 1);
    }
    *out = c;
    return DG_OK;
}

int dg_finalize(dg_ctx *c) {
    if (!c) return DG_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &a : c->allocations) {
        dg::f64::debug_register(a.first, a.second, 0);
        dg::f32::debug_register(a.first, a.second, 0);
    }
    void *bufs[] = {c->B.U[0], c->B.U[1], c->B.Q, c->B.core, c->B.flx[0], c->B.flx[1], c->B.flx[2], c->B.emf[0],
                    c->B.emf[1], c->B.emf[2], c->B.femf[0], c->B.femf[1], c->B.part, c->B.hist,
                    c->B.E[0], c->B.E[1], c->B.E[2], c->B.stage, c->B.fb_list[0], c->B.fb_list[1], c->B.fb_list[2],
                    c->B.nn_count};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (c->B.S) cudaFree(c->B.S);
    if (c->h_scal) cudaFreeHost(c->h_scal);
    if (c->h_hist) cudaFreeHost(c->h_hist);
    delete c->timer;
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return DG_OK;
}

int dg_upload(dg_ctx *c, const double *uin) {
    if (!c || !uin) return fail(DG_ERR_ARG, "null argument");
    TimerScope ts_(c);
    DG_CUDA(cudaSetDevice(c->p.device));
    const size_t nt = (size_t)c->G.sv;
    if (c->p.precision == DG_PREC_FP64) {
        // uin(:,:,:,1:8) is contiguous in the reference layout
        DG_CUDA(cudaMemcpyAsync(c->B.U[c->cur], uin, nt * 8 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        // the right-face B that the reference never refreshes (uin var 11 in 2D, vars 10-11 in
        // 1D) stays at its initial value; both state buffers carry it (planes 8..nv-1)
        const size_t nf = (size_t)c->nv - 8;
        for (int b = 0; b < 2 && nf > 0; b++)
            DG_CUDA(cudaMemcpyAsync((double *)c->B.U[b] + nt * 8, uin + nt * (11 - nf), nf * nt * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
    } else {
        const size_t nf = (size_t)c->nv - 8;
        DG_CUDA(cudaMemcpyAsync(c->B.stage, uin, nt * 8 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (nf > 0)
            DG_CUDA(cudaMemcpyAsync(c->B.stage + nt * 8, uin + nt * (11 - nf), nf * nt * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
        c->launches += c->L->from_f64(c->G, c->B, c->cur, c->B.stage, c->nv, c->stream);
        if (nf > 0) c->launches += c->L->from_f64(c->G, c->B, c->cur ^ 1, c->B.stage, c->nv, c->stream);
        int rc = check_launch();
        if (rc) return rc;
    }
    c->version++;
    return bounded_sync(c->stream);
}

int dg_download(dg_ctx *c, double *uin) {
    if (!c || !uin) return fail(DG_ERR_ARG, "null argument");
    TimerScope ts_(c);
    DG_CUDA(cudaSetDevice(c->p.device));
    const size_t nt = (size_t)c->G.sv;
    double *scratch;
    if (c->p.precision == DG_PREC_FP64) {
        DG_CUDA(cudaMemcpyAsync(uin, c->B.U[c->cur], nt * 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        scratch = (double *)c->B.Q;  // 8 planes of doubles, recomputed by every step
        c->q_version = -1;           // no longer the primitive variables of the CFL pass
    } else {
        c->launches += c->L->to_f64(c->G, c->B, c->cur, c->B.stage, c->stream);
        DG_CUDA(cudaMemcpyAsync(uin, c->B.stage, nt * 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (int rc = bounded_sync(c->stream)) return rc;
        scratch = c->B.stage;
    }
    c->launches += c->L->right_faces(c->G, c->B, c->cur, scratch, c->stream);
    int rc = check_launch();
    if (rc) return rc;
    DG_CUDA(cudaMemcpyAsync(uin + nt * 8, scratch, nt * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return bounded_sync(c->stream);
}

// ---------------------------------------------------------------------------
// Fortran 'binary' dumps (output.f90:224-235, restart.f90:212-221), record layout in dump_io.h
// ---------------------------------------------------------------------------
namespace {
dg::dump::Header make_header(const dg_params &p, double time, double dt) {
    const dg::Geo G = dg::make_geo(p);
    dg::dump::Header h{};
    h.nx = p.nx; h.ny = p.ny; h.nz = p.nz;
    h.nxslice = h.nyslice = 1;
    h.nzslice = G.nzslice;  // a z slab writes its own rank's file, as each MPI rank does
    h.time = time; h.dt = dt; h.dx = G.dx; h.dy = G.dy; h.dz = G.dz;
    h.xmin = p.xmin; h.xmax = p.xmax; h.ymin = p.ymin; h.ymax = p.ymax; h.zmin = p.zmin; h.zmax = p.zmax;
    h.gamma = p.gamma; h.ciso = p.ciso;
    return h;
}

// a dump read into a context (or a host array of its grid) must hold the same grid and constants
int check_header(const dg::dump::Header &h, const dg_params &p, const char *path) {
    const int nzslice = p.nzslice > 1 ? p.nzslice : 1;
    if (h.nxslice != 1 || h.nyslice != 1 || h.nzslice != nzslice)
        return fail(DG_ERR_UNSUPPORTED, std::string(path) + ": a dump of another decomposition (slices " +
                                            std::to_string(h.nxslice) + "x" + std::to_string(h.nyslice) + "x" +
                                            std::to_string(h.nzslice) + ")");
    if (h.nx != p.nx || h.ny != p.ny || h.nz != p.nz)
        return fail(DG_ERR_ARG, std::string(path) + ": grid " + std::to_string(h.nx) + "x" + std::to_string(h.ny) +
                                    "x" + std::to_string(h.nz) + " differs from the context's");
    const dg::dump::Header e = make_header(p, 0.0, 0.0);
    const double got[] = {h.dx, h.dy, h.dz, h.xmin, h.xmax, h.ymin, h.ymax, h.zmin, h.zmax, h.gamma, h.ciso};
    const double want[] = {e.dx, e.dy, e.dz, e.xmin, e.xmax, e.ymin, e.ymax, e.zmin, e.zmax, e.gamma, e.ciso};
    for (int q = 0; q < 11; q++)
        if (!(got[q] == want[q]))
            return fail(DG_ERR_ARG, std::string(path) + ": domain, gamma or ciso differ from the context's");
    return DG_OK;
}

struct FileCloser {
    FILE *f = nullptr;
    ~FileCloser() { if (f) std::fclose(f); }
    int close_checked(const char *path) {
        const int e = std::fclose(f);
        f = nullptr;
        return e == 0 ? DG_OK : fail(DG_ERR_ARG, std::string(path) + ": write failed");
    }
};

// two pinned host planes and their copy events, for streaming the uin record
struct PlaneBuffers {
    double *b[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int init(size_t n) {
        for (int q = 0; q < 2; q++) {
            if (cudaMallocHost(&b[q], n * sizeof(double)) != cudaSuccess)
                return fail(DG_ERR_NOMEM, "cudaMallocHost of a dump plane failed");
            if (cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming) != cudaSuccess)
                return fail(DG_ERR_CUDA, "cudaEventCreate failed");
        }
        return DG_OK;
    }
    ~PlaneBuffers() {
        for (int q = 0; q < 2; q++) {
            if (ev[q]) cudaEventDestroy(ev[q]);
            if (b[q]) cudaFreeHost(b[q]);
        }
    }
};
}  // namespace

int dg_dump_header(const char *path, dg_dump_info *out) {
    if (!path || !out) return fail(DG_ERR_ARG, "null argument");
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return fail(DG_ERR_ARG, std::string("cannot open ") + path);
    dg::dump::Header h;
    if (!dg::dump::read_header(fc.f, h)) return fail(DG_ERR_ARG, std::string(path) + ": not a dump header");
    // length of the uin record: walk its subrecord markers
    long long bytes = 0;
    for (;;) {
        int32_t lead, trail;
        if (std::fread(&lead, 4, 1, fc.f) != 1) return fail(DG_ERR_ARG, std::string(path) + ": no uin record");
        const long long len = lead < 0 ? -(long long)lead : (long long)lead;
        if (std::fseek(fc.f, (long)len, SEEK_CUR) != 0 || std::fread(&trail, 4, 1, fc.f) != 1)
            return fail(DG_ERR_ARG, std::string(path) + ": truncated uin record");
        bytes += len;
        if (lead >= 0) break;
    }
    out->nx = h.nx; out->ny = h.ny; out->nz = h.nz;
    out->nxslice = h.nxslice; out->nyslice = h.nyslice; out->nzslice = h.nzslice;
    out->time = h.time; out->dt = h.dt; out->dx = h.dx; out->dy = h.dy; out->dz = h.dz;
    out->xmin = h.xmin; out->xmax = h.xmax; out->ymin = h.ymin; out->ymax = h.ymax; out->zmin = h.zmin; out->zmax = h.zmax;
    out->gamma = h.gamma; out->ciso = h.ciso;
    out->uin_bytes = bytes;
    return DG_OK;
}

int dg_dump_write_host(const char *path, const dg_params *p, double time, double dt, const double *uin) {
    if (!path || !uin) return fail(DG_ERR_ARG, "null argument");
    if (int rc = validate(p)) return rc;
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return fail(DG_ERR_ARG, std::string("cannot open ") + path + " for writing");
    const long long bytes = dg_uin_size(p) * (long long)sizeof(double);
    if (!dg::dump::write_header(fc.f, make_header(*p, time, dt))) return fail(DG_ERR_ARG, std::string(path) + ": write failed");
    dg::dump::RecordWriter w(fc.f, bytes);
    if (!w.write(uin, bytes) || !w.close()) return fail(DG_ERR_ARG, std::string(path) + ": write failed");
    return fc.close_checked(path);
}

int dg_dump_read_host(const char *path, const dg_params *p, double *time, double *dt, double *uin) {
    if (!path || !uin || !time || !dt) return fail(DG_ERR_ARG, "null argument");
    if (int rc = validate(p)) return rc;
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return fail(DG_ERR_ARG, std::string("cannot open ") + path);
    dg::dump::Header h;
    if (!dg::dump::read_header(fc.f, h)) return fail(DG_ERR_ARG, std::string(path) + ": not a dump header");
    if (int rc = check_header(h, *p, path)) return rc;
    dg::dump::RecordReader r(fc.f);
    if (!r.read(uin, dg_uin_size(p) * (long long)sizeof(double)) || !r.close())
        return fail(DG_ERR_ARG, std::string(path) + ": the uin record does not hold this grid");
    *time = h.time;
    *dt = h.dt;
    return DG_OK;
}

int dg_dump_write(dg_ctx *c, const char *path, double time, double dt) {
    if (!c || !path) return fail(DG_ERR_ARG, "null argument");
    TimerScope ts_(c);
    DG_CUDA(cudaSetDevice(c->p.device));
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return fail(DG_ERR_ARG, std::string("cannot open ") + path + " for writing");
    const size_t nt = (size_t)c->G.sv;
    PlaneBuffers pb;
    if (int rc = pb.init(nt)) return rc;
    // device planes of uin vars 1-8: the FP64 state, or its FP64 values in the staging buffer;
    // vars 9-11 from the right-face kernel into a scratch buffer that is free at this point
    const double *left;
    double *scratch;
    if (c->p.precision == DG_PREC_FP64) {
        left = (const double *)c->B.U[c->cur];
        scratch = (double *)c->B.Q;
        c->q_version = -1;  // Q is scratch here: a following godunov recomputes the primitives
    } else {
        // the staging buffer: its planes 0-2 take vars 9-11 once vars 1-8 are copied out
        c->launches += c->L->to_f64(c->G, c->B, c->cur, c->B.stage, c->stream);
        left = c->B.stage;
        scratch = c->B.stage;
    }
    if (int rc = check_launch()) return rc;
    if (!dg::dump::write_header(fc.f, make_header(c->p, time, dt)))
        return fail(DG_ERR_ARG, std::string(path) + ": write failed");
    dg::dump::RecordWriter w(fc.f, (long long)nt * 11 * (long long)sizeof(double));
    // plane v is copied while plane v-1 is written to the file
    for (int v = 0; v <= 11; v++) {
        if (v < 11) {
            if (v == 8) {
                // vars 9-11, after the copies of vars 1-8 in stream order
                c->launches += c->L->right_faces(c->G, c->B, c->cur, scratch, c->stream);
                if (int rc = check_launch()) return rc;
            }
            const double *src = v < 8 ? left + (size_t)v * nt : scratch + (size_t)(v - 8) * nt;
            DG_CUDA(cudaMemcpyAsync(pb.b[v & 1], src, nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            DG_CUDA(cudaEventRecord(pb.ev[v & 1], c->stream));
        }
        if (v > 0) {
            if (int rc = bounded_event(pb.ev[(v - 1) & 1])) return rc;
            if (!w.write(pb.b[(v - 1) & 1], (long long)(nt * sizeof(double))))
                return fail(DG_ERR_ARG, std::string(path) + ": write failed");
        }
    }
    if (!w.close()) return fail(DG_ERR_ARG, std::string(path) + ": write failed");
    if (int rc = bounded_sync(c->stream)) return rc;
    return fc.close_checked(path);
}

int dg_dump_read(dg_ctx *c, const char *path, double *time, double *dt) {
    if (!c || !path || !time || !dt) return fail(DG_ERR_ARG, "null argument");
    TimerScope ts_(c);
    DG_CUDA(cudaSetDevice(c->p.device));
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return fail(DG_ERR_ARG, std::string("cannot open ") + path);
    dg::dump::Header h;
    if (!dg::dump::read_header(fc.f, h)) return fail(DG_ERR_ARG, std::string(path) + ": not a dump header");
    if (int rc = check_header(h, c->p, path)) return rc;
    const size_t nt = (size_t)c->G.sv;
    PlaneBuffers pb;
    if (int rc = pb.init(nt)) return rc;
    if (int rc = bounded_sync(c->stream)) return rc;  // no step may still read the state
    const bool f64 = c->p.precision == DG_PREC_FP64;
    dg::dump::RecordReader r(fc.f);
    // plane v is read from the file while plane v-1 is copied; the right faces are derived from
    // the left faces and skipped, except the frozen copies: var 11 in 2D, vars 10-11 in 1D
    // (stored planes 8..nv-1, both buffers)
    for (int v = 0; v < 11; v++) {
        if (v >= 2)
            if (int rc = bounded_event(pb.ev[v & 1])) return rc;  // the copy of plane v-2 is done
        if (!r.read(pb.b[v & 1], (long long)(nt * sizeof(double))))
            return fail(DG_ERR_ARG, std::string(path) + ": the uin record does not hold this grid");
        double *dst[2] = {nullptr, nullptr};
        if (v < 8) {
            dst[0] = f64 ? (double *)c->B.U[c->cur] + (size_t)v * nt : c->B.stage + (size_t)v * nt;
        } else if (v >= 11 - (c->nv - 8)) {
            const size_t pl = (size_t)(v - (11 - (c->nv - 8)) + 8);
            if (f64) {
                dst[0] = (double *)c->B.U[0] + nt * pl;
                dst[1] = (double *)c->B.U[1] + nt * pl;
            } else {
                dst[0] = c->B.stage + nt * pl;
            }
        }
        for (double *d : dst)
            if (d) DG_CUDA(cudaMemcpyAsync(d, pb.b[v & 1], nt * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        DG_CUDA(cudaEventRecord(pb.ev[v & 1], c->stream));
    }
    if (!r.close()) return fail(DG_ERR_ARG, std::string(path) + ": the uin record does not hold this grid");
    if (!f64) {
        c->launches += c->L->from_f64(c->G, c->B, c->cur, c->B.stage, c->nv, c->stream);
        if (c->nv > 8) c->launches += c->L->from_f64(c->G, c->B, c->cur ^ 1, c->B.stage, c->nv, c->stream);
        if (int rc = check_launch()) return rc;
    }
    c->version++;
    if (int rc = bounded_sync(c->stream)) return rc;
    *time = h.time;
    *dt = h.dt;
    return DG_OK;
}

int dg_compute_dt(dg_ctx *c, double *dt) {
    TimerScope ts_(c);
    if (!c || !dt) return fail(DG_ERR_ARG, "null argument");
    c->launches += c->L->dt(c->G, c->B, c->cur, c->stream);
    c->q_version = c->version;  // the CFL pass also left primitive(0) of this state in Q
    int rc = check_launch();
    if (rc) return rc;
    if ((rc = read_scalars(c))) return rc;
    *dt = c->h_scal->dt;
    return DG_OK;
}

int dg_godunov(dg_ctx *c, double dt, double time) {
    TimerScope ts_(c);
    if (!c) return fail(DG_ERR_ARG, "null context");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(DG_ERR_DT, "dt must be positive and finite");
    c->launches += c->L->set_scalars(c->B, dt, time, 1, 1, c->stream);
    c->B.q_fresh = (c->q_version == c->version);
    c->launches += c->L->godunov(c->G, c->B, c->cur, c->stream);
    c->cur ^= 1;
    c->version++;
    return check_launch();
}

int dg_fargo_update(dg_ctx *c, double dt) {
    TimerScope ts_(c);
    if (!c) return fail(DG_ERR_ARG, "null context");
    if (!c->p.fargo) return fail(DG_ERR_ARG, "context was created with fargo = 0");
    c->launches += c->L->set_scalars(c->B, dt, 0.0, 1, 0, c->stream);
    c->launches += c->L->fargo(c->G, c->B, c->cur, c->stream);
    c->cur ^= 1;
    c->version++;
    return check_launch();
}

int dg_boundary(dg_ctx *c, double time, double dt) {
    TimerScope ts_(c);
    if (!c) return fail(DG_ERR_ARG, "null context");
    c->launches += c->L->set_scalars(c->B, dt, time, 1, 1, c->stream);
    c->launches += c->L->boundary(c->G, c->B, c->cur, c->stream);
    c->version++;
    return check_launch();
}

int dg_dissipation(dg_ctx *c, double time, double dt) {
    TimerScope ts_(c);
    if (!c) return fail(DG_ERR_ARG, "null context");
    if (!(c->G.nu > 0.0) && !(c->G.eta > 0.0)) return DG_OK;  // dumses.f90:104 calls it only then
    c->launches += c->L->set_scalars(c->B, dt, time, 1, 1, c->stream);
    c->launches += c->L->dissipation(c->G, c->B, c->cur, c->stream);
    c->version++;
    return check_launch();
}

int dg_run(dg_ctx *c, int nsteps, double *time, double *dt) {
    TimerScope ts_(c);
    if (!c || !time) return fail(DG_ERR_ARG, "null argument");
    if (nsteps < 0) return fail(DG_ERR_ARG, "nsteps < 0");
    if (c->G.nzslice > 1)
        return fail(DG_ERR_UNSUPPORTED, "a z slab needs its halos exchanged every step: drive it with dg_compute_dt, "
                                        "dg_godunov, dg_fargo_update, dg_boundary and dg_halo_pack/unpack");
    c->launches += c->L->set_scalars(c->B, 0.0, *time, 0, 1, c->stream);
    for (int n = 0; n < nsteps; n++) {
        c->launches += c->L->dt(c->G, c->B, c->cur, c->stream);
        c->B.q_fresh = 1;  // Q holds primitive(0) of this state from the CFL pass
        c->launches += c->L->godunov(c->G, c->B, c->cur, c->stream);
        c->cur ^= 1;
        if (c->p.fargo) {
            c->launches += c->L->fargo(c->G, c->B, c->cur, c->stream);
            c->cur ^= 1;
        }
        c->launches += c->L->boundary(c->G, c->B, c->cur, c->stream);
        if (c->G.nu > 0.0 || c->G.eta > 0.0) c->launches += c->L->dissipation(c->G, c->B, c->cur, c->stream);
        c->version++;
        c->launches += c->L->advance_time(c->B, c->stream);
    }
    int rc = check_launch();
    if (rc) return rc;
    if ((rc = read_scalars(c))) return rc;
    *time = c->h_scal->time;
    if (dt) *dt = c->h_scal->dt;
    return DG_OK;
}

int dg_step(dg_ctx *c, double *time, double *dt) { return dg_run(c, 1, time, dt); }

int dg_history_variant(dg_ctx *c, int variant, double out[9]) {
    TimerScope ts_(c);
    if (!c || !out) return fail(DG_ERR_ARG, "null argument");
    if (variant != DG_HISTORY_MRI && variant != DG_HISTORY_DEFAULT) return fail(DG_ERR_ARG, "unknown history variant");
    if (c->p.ndim == 1 && variant == DG_HISTORY_DEFAULT) {
        // the one-dimensional line (history.f90:37-59): rho, rho u_x and E at x = 1/2
        c->launches += dg::f64::launch_history_1d(c->G, (const double *)c->B.U[c->cur], c->B.hist, c->stream);
    } else if (c->p.ndim != 3) {
        return fail(DG_ERR_UNSUPPORTED, "the history sums are defined for ndim = 3 (and the line of ndim = 1)");
    } else {
        c->launches += c->L->history(c->G, c->B, c->cur, c->stream, variant);
    }
    int rc = check_launch();
    if (rc) return rc;
    DG_CUDA(cudaMemcpyAsync(c->h_hist, c->B.hist, 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((rc = bounded_sync(c->stream))) return rc;
    std::memcpy(out, c->h_hist, 9 * sizeof(double));
    return DG_OK;
}

int dg_history(dg_ctx *c, double out[9]) { return dg_history_variant(c, DG_HISTORY_MRI, out); }

// ---- z-slab halos: 3 planes of every stored state plane (FP64: nv double planes;
// FP32: 2 nv float planes, hi then lo), one strided copy per side
namespace {
struct HaloGeom {
    size_t width;   // bytes of 3 planes of one stored plane
    size_t pitch;   // bytes between stored planes
    size_t planes;  // stored planes
    size_t es;      // bytes per element of the state
};
HaloGeom halo_geom(const dg_ctx *c) {
    const bool f64 = c->p.precision == DG_PREC_FP64;
    HaloGeom h;
    h.es = f64 ? 8 : 4;
    h.planes = f64 ? (size_t)c->nv : 2 * (size_t)c->nv;
    h.width = 3 * (size_t)c->G.sz * h.es;
    h.pitch = (size_t)c->G.sv * h.es;
    return h;
}
int halo_check(const dg_ctx *c, int side, const void *buf) {
    if (!c || !buf) return fail(DG_ERR_ARG, "null argument");
    if (side != 0 && side != 1) return fail(DG_ERR_ARG, "side must be 0 (lower) or 1 (upper)");
    if (c->p.ndim != 3) return fail(DG_ERR_UNSUPPORTED, "z halos exist for ndim = 3");
    return DG_OK;
}
}  // namespace

long long dg_halo_count(const dg_ctx *c) {
    if (!c || c->p.ndim != 3) return 0;
    return 3LL * c->G.sz * c->nv;
}

int dg_halo_pack(dg_ctx *c, int side, double *buf) {
    if (int rc = halo_check(c, side, buf)) return rc;
    DG_CUDA(cudaSetDevice(c->p.device));
    const HaloGeom h = halo_geom(c);
    // active planes k = 1..3 (side 0) or nz-2..nz (side 1): plane k starts at (k + 2) * sz
    const size_t k0 = side == 0 ? 3 : (size_t)c->G.nz;
    const char *src = (const char *)c->B.U[c->cur] + k0 * (size_t)c->G.sz * h.es;
    DG_CUDA(cudaMemcpy2DAsync(buf, h.width, src, h.pitch, h.width, h.planes, cudaMemcpyDefault, c->stream));
    return DG_OK;
}

int dg_halo_unpack(dg_ctx *c, int side, const double *buf) {
    if (int rc = halo_check(c, side, buf)) return rc;
    DG_CUDA(cudaSetDevice(c->p.device));
    const HaloGeom h = halo_geom(c);
    // ghost planes k = -2..0 (side 0, from 0) or nz+1..nz+3 (side 1, from (nz + 3) * sz)
    const size_t k0 = side == 0 ? 0 : (size_t)c->G.nz + 3;
    char *dst = (char *)c->B.U[c->cur] + k0 * (size_t)c->G.sz * h.es;
    DG_CUDA(cudaMemcpy2DAsync(dst, h.pitch, buf, h.width, h.width, h.planes, cudaMemcpyDefault, c->stream));
    c->version++;
    return DG_OK;
}

int dg_history_columns(dg_ctx *c, double *col) {
    TimerScope ts_(c);
    if (!c || !col) return fail(DG_ERR_ARG, "null argument");
    if (c->p.ndim != 3) return fail(DG_ERR_UNSUPPORTED, "the MRI history is defined for ndim = 3");
    DG_CUDA(cudaSetDevice(c->p.device));
    c->launches += c->L->history_columns(c->G, c->B, c->cur, c->stream);
    if (int rc = check_launch()) return rc;
    DG_CUDA(cudaMemcpyAsync(col, c->B.part, 2 * (size_t)c->G.nx * sizeof(double), cudaMemcpyDefault, c->stream));
    return bounded_sync(c->stream);
}

int dg_history_share(dg_ctx *c, const double *colmean, double out[9]) {
    TimerScope ts_(c);
    if (!c || !colmean || !out) return fail(DG_ERR_ARG, "null argument");
    if (c->p.ndim != 3) return fail(DG_ERR_UNSUPPORTED, "the MRI history is defined for ndim = 3");
    DG_CUDA(cudaSetDevice(c->p.device));
    DG_CUDA(cudaMemcpyAsync(c->B.part, colmean, 2 * (size_t)c->G.nx * sizeof(double), cudaMemcpyDefault, c->stream));
    c->launches += c->L->history_share(c->G, c->B, c->cur, c->stream);
    if (int rc = check_launch()) return rc;
    DG_CUDA(cudaMemcpyAsync(c->h_hist, c->B.hist, 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (int rc = bounded_sync(c->stream)) return rc;
    std::memcpy(out, c->h_hist, 9 * sizeof(double));
    return DG_OK;
}

long long dg_debug_oob_count(void) {
    const long long a = dg::f64::debug_oob(), b = dg::f32::debug_oob();
    return (a < 0 || b < 0) ? -1 : a + b;
}

int dg_sync(dg_ctx *c) {
    if (!c) return fail(DG_ERR_ARG, "null context");
    return bounded_sync(c->stream);
}

int dg_attach_surrogate(dg_ctx *c, dg_nn *nn) {
    if (!c) return fail(DG_ERR_ARG, "null context");
    if (!c->p.surrogate) return fail(DG_ERR_ARG, "the context was made with surrogate = 0");
    if (nn && dg_nn_device(nn) != c->p.device) return fail(DG_ERR_ARG, "network and context are on different devices");
    DG_CUDA(cudaSetDevice(c->p.device));
    DG_CUDA(cudaStreamSynchronize(c->stream));
    c->nn = nn;
    if (nn) {
        dg_nn_view(nn, &c->view);
        c->B.net = &c->view;
        DG_CUDA(cudaFuncSetAttribute(dg::f32::nn_faces_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     dg::f32::nn_faces_smem()));
    } else {
        c->B.net = nullptr;
    }
    return DG_OK;
}

int dg_surrogate_stats(dg_ctx *c, long long *faces, long long *fallback) {
    if (!c || !faces || !fallback) return fail(DG_ERR_ARG, "null argument");
    *faces = 0;
    *fallback = 0;
    if (!c->p.surrogate) return DG_OK;
    DG_CUDA(cudaSetDevice(c->p.device));
    unsigned long long h[4] = {0, 0, 0, 0};
    DG_CUDA(cudaMemcpyAsync(h, c->B.nn_count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    int rc = bounded_sync(c->stream);
    if (rc) return rc;
    DG_CUDA(cudaMemsetAsync(c->B.nn_count, 0, 2 * sizeof(unsigned long long), c->stream));
    *faces = (long long)h[0];
    *fallback = (long long)h[1];
    if ((int)h[2]) return fail(DG_ERR_TIMEOUT, "a face-network kernel gave up waiting on a tensor-core transfer");
    return DG_OK;
}

int dg_nn_harvest(dg_ctx *c, dg_nn *nn, int stride, long long *added) {
    if (!c || !nn || stride < 1) return fail(DG_ERR_ARG, "bad harvest arguments");
    if (c->p.precision != DG_PREC_FP32) return fail(DG_ERR_UNSUPPORTED, "harvesting reads the FP32 trace");
    if (dg_nn_device(nn) != c->p.device) return fail(DG_ERR_ARG, "network and context are on different devices");
    DG_CUDA(cudaSetDevice(c->p.device));
    TimerScope ts(c);
    const dg::Geo &G = c->G;
    long long cnt[3] = {0, 0, 0}, total = 0;
    for (int d = 0; d < G.ndim; d++) {
        cnt[d] = (dg::f32::harvest_faces(G, d) + stride - 1) / stride;
        total += cnt[d];
    }
    const long long first = dg_nn_sample_count(nn);
    int rc = dg_nn_reserve_samples(nn, first + total);
    if (rc) return rc;
    c->launches += dg::f32::launch_trace_only(G, c->B, c->cur, c->stream);
    c->q_version = -1;  // Q now holds the kicked primitive variables
    long long at = first;
    for (int d = 0; d < G.ndim; d++) {
        c->launches += dg::f32::launch_harvest(G, c->B, d, stride, dg_nn_sample_x(nn), dg_nn_sample_t(nn), at, cnt[d],
                                               c->stream);
        at += cnt[d];
    }
    DG_CUDA(cudaGetLastError());
    if ((rc = bounded_sync(c->stream))) return rc;
    dg_nn_set_count(nn, first + total);
    if (added) *added = total;
    return DG_OK;
}

int dg_debug_copy(dg_ctx *c, int which, double *host, long long count, long long *copied) {
    if (!c || !host) return fail(DG_ERR_ARG, "null argument");
    const void *src = nullptr;
    long long n = 0;
    if (which >= 0 && which <= 2) { src = c->B.flx[which]; n = c->G.fsz * dg::flux_rec(c->G.ndim); }
    else if (which >= 3 && which <= 5) { src = c->B.emf[which - 3]; n = c->G.fsz; }
    else if (which == 6) { src = c->B.Q; n = c->G.sv * 8; }
    if (!src) return fail(DG_ERR_ARG, "no such array for this context");
    if (count < n) return fail(DG_ERR_ARG, "host buffer too small");
    if (c->es == sizeof(double)) {
        DG_CUDA(cudaMemcpyAsync(host, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        int rc = bounded_sync(c->stream);
        if (rc) return rc;
    } else {
        std::vector<float> tmp((size_t)n);
        DG_CUDA(cudaMemcpyAsync(tmp.data(), src, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        int rc = bounded_sync(c->stream);
        if (rc) return rc;
        for (long long k = 0; k < n; k++) host[k] = tmp[(size_t)k];
    }
    if (copied) *copied = n;
    return DG_OK;
}

long long dg_kernel_launches(const dg_ctx *c) { return c ? c->launches : 0; }

int dg_profile(dg_ctx *c, int on) {
    if (!c) return fail(DG_ERR_ARG, "null context");
    if (on && !c->timer) c->timer = new EventTimer();
    if (!on && c->timer) {
        cudaStreamSynchronize(c->stream);
        delete c->timer;
        c->timer = nullptr;
    }
    return DG_OK;
}

int dg_profile_read(dg_ctx *c, double *ms, long long *count, int nslots) {
    if (!c || !ms || !count) return fail(DG_ERR_ARG, "null argument");
    for (int k = 0; k < nslots; k++) { ms[k] = 0.0; count[k] = 0; }
    if (!c->timer) return DG_OK;
    int rc = bounded_sync(c->stream);
    if (rc) return rc;
    for (auto &r : c->timer->recs) {
        float t = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        if (r.slot < nslots) { ms[r.slot] += t; count[r.slot] += 1; }
        c->timer->pool.push_back(r.a);
        c->timer->pool.push_back(r.b);
    }
    c->timer->recs.clear();
    return DG_OK;
}

const char *dg_profile_slot_name(int slot) {
    return (slot >= 0 && slot < dg::KS_COUNT) ? kSlotNames[slot] : "";
}

void *dg_stream(dg_ctx *c) { return c ? (void *)c->stream : nullptr; }

}  // extern "C"
