// Launch interface of the MHD step kernels (definitions in step_fp64.cu and
// step_fp32.cu, both instantiating step_impl.cuh).
#pragma once
#include "dg_common.cuh"

namespace dg {

namespace nn {
struct NetView;
}

// device buffers of one context; element type of the work arrays is the compute
// type of the path (double for FP64, float for FP32)
struct Bufs {
    void *U[2];        // state: FP64 path nv double planes; FP32 path 2*nv float planes (hi planes, then lo planes)
    void *Q;           // primitive variables (8 planes) on the ghosted grid
    void *core;        // trace core over the core index space
    void *flx[3];      // face fluxes per direction, face-major records (flux_rec(ndim) values per face)
    void *emf[3];      // edge EMFs (x, y, z) over the face index space, already multiplied by dt
    void *E[3];        // edge electric fields of the trace over the edge index space
    double *femf[2];   // FARGO EMFs (x, z), FP64
    double *stage;     // FP64 staging planes for upload/download of the compensated state
    double *part;      // reduction partials
    double *hist;      // history results
    Scalars *S;        // device scalars
    int nv;            // state variables: 8, or 9 with ndim = 2 (frozen right z-face)
    long long sv;      // cells per plane
    int q_fresh;       // FP32 path: Q holds the primitive variables (without the rotation half-kick)
                       // of U[cur], written by the last launch_dt with no state change since
    // learned face flux (FP32 path with surrogate = 1)
    const nn::NetView *net;         // attached network (host copy of its device view), null: HLLD everywhere
    int *fb_list[3];                // per direction: faces sent back to HLLD in the current step
    unsigned long long *nn_count;   // device counters: [0] faces seen, [1] faces sent back to HLLD
                                    // (both since the last read), [3 + d] length of fb_list[d]
    int *nn_err;                    // device error word of the network kernels
};

int nstate_vars(const Geo &G);

// per-kernel timing slots (CUDA events around each launch when a timer is attached)
enum KernelSlot { KS_SCALARS = 0, KS_DT, KS_PRIM, KS_TRACE, KS_RIEMANN, KS_UPDATE, KS_FARGO_EMF, KS_FARGO_UPDATE,
                  KS_BOUNDARY, KS_HISTORY, KS_RIGHT_FACES, KS_EFIELD, KS_NN_FACES, KS_NN_FALLBACK, KS_DISSIPATION,
                  KS_COUNT };
struct KernelTimer {
    virtual void begin(int slot, cudaStream_t st) = 0;
    virtual void end(int slot, cudaStream_t st) = 0;
    virtual ~KernelTimer() {}
};
extern thread_local KernelTimer *g_timer;  // set by the context that enqueues (one host thread per context)

// The launch set of one arithmetic; every function returns the number of kernels enqueued.
#define DG_DECLARE_LAUNCHES                                                                          \
    int launch_set_scalars(const Bufs &B, double dt, double time, int set_dt, int set_time, cudaStream_t st); \
    int launch_advance_time(const Bufs &B, cudaStream_t st);                                         \
    int launch_dt(const Geo &G, const Bufs &B, int cur, cudaStream_t st);                            \
    int launch_godunov(const Geo &G, const Bufs &B, int cur, cudaStream_t st);   /* U[cur] -> U[cur^1] */ \
    int launch_fargo(const Geo &G, const Bufs &B, int cur, cudaStream_t st);     /* U[cur] -> U[cur^1] */ \
    int launch_boundary(const Geo &G, const Bufs &B, int cur, cudaStream_t st);  /* in place on U[cur] */ \
    int launch_history(const Geo &G, const Bufs &B, int cur, cudaStream_t st, int variant);          \
    /* z slabs: per-column sums of v_x, v_y into B.part (2 nx doubles); then this slab's share of */ \
    /* the history with the box's column means read from B.part, into B.hist */                      \
    int launch_history_columns(const Geo &G, const Bufs &B, int cur, cudaStream_t st);               \
    int launch_history_share(const Geo &G, const Bufs &B, int cur, cudaStream_t st);                 \
    int launch_dissipation(const Geo &G, const Bufs &B, int cur, cudaStream_t st); /* in place, then boundary */ \
    int launch_right_faces(const Geo &G, const Bufs &B, int cur, double *out, cudaStream_t st);      \
    int launch_state_to_f64(const Geo &G, const Bufs &B, int cur, double *out, cudaStream_t st);     \
    int launch_f64_to_state(const Geo &G, const Bufs &B, int b, const double *in, int nv, cudaStream_t st); \
    /* bounds-checked build: add (add = 1) or remove a device buffer; accesses outside all of them */ \
    int debug_register(const void *p, size_t bytes, int add);                                        \
    long long debug_oob(); /* -1 in a normal build */

namespace f64 {
DG_DECLARE_LAUNCHES
// history of any FP64 state array U with explicit scratch (>= history_scratch_doubles(G)
// doubles) and a 9-double output, all device pointers
int launch_history_ptrs(const Geo &G, const double *U, double *scratch, double *out, cudaStream_t st,
                        int variant = DG_HISTORY_MRI);
long long history_scratch_doubles(const Geo &G);
// the ndim = 1 history line: out[0..2] = rho, rho u_x, E of the first cell at x >= 1/2, out[3..8] = 0
int launch_history_1d(const Geo &G, const double *U, double *out, cudaStream_t st);
}  // namespace f64

namespace f32 {
DG_DECLARE_LAUNCHES
// primitive variables, edge fields and trace of U[cur] (the first half of godunov)
int launch_trace_only(const Geo &G, const Bufs &B, int cur, cudaStream_t st);
// every stride-th interface of direction d from the trace core: scaled inputs into xs and
// scaled HLLD-minus-LLF targets into ts, samples [first, first + count)
int launch_harvest(const Geo &G, const Bufs &B, int d, int stride, float *xs, float *ts, long long first,
                   long long count, cudaStream_t st);
// faces of direction d (0..ndim-1) enumerated as harvested: (nx+1) ny nz for x, ...
long long harvest_faces(const Geo &G, int d);
// the face-network kernel and its dynamic shared memory (for the attribute call)
const void *nn_faces_kernel();
int nn_faces_smem();
}  // namespace f32

// shared host helpers (dg_api.cu)
Geo make_geo(const dg_params &p);
int set_error(int code, const char *msg);

}  // namespace dg
