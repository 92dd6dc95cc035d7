// Kernel declarations of the MHD step (definitions in mhd_kernels.cu).
#pragma once
#include "dg_common.cuh"

namespace dg {

// device buffers of one context
struct Bufs {
    double *U[2];      // state, 8 (ndim = 3) or 9 (ndim = 2: + frozen right z-face) variables
    double *Q;         // primitive variables (8) on the ghosted grid
    double *core;      // trace core, kCore3/kCore2 fields over the core index space
    double *flx[3];    // face fluxes per direction, kFluxComp components over the face index space
    double *emf[3];    // edge EMFs (x, y, z) over the face index space, already multiplied by dt
    double *femf[2];   // FARGO EMFs (x, z) over the face index space
    double *part;      // reduction partials
    double *hist;      // history results
    Scalars *S;        // device scalars
};

int nstate_vars(const Geo &G);

// per-kernel timing slots (CUDA events around each launch when a timer is attached)
enum KernelSlot { KS_SCALARS = 0, KS_DT, KS_PRIM, KS_TRACE, KS_RIEMANN, KS_UPDATE, KS_FARGO_EMF, KS_FARGO_UPDATE,
                  KS_BOUNDARY, KS_HISTORY, KS_RIGHT_FACES, KS_COUNT };
struct KernelTimer {
    virtual void begin(int slot, cudaStream_t st) = 0;
    virtual void end(int slot, cudaStream_t st) = 0;
    virtual ~KernelTimer() {}
};
extern thread_local KernelTimer *g_timer;  // set by the context that enqueues (one host thread per context)

// launches (return the number of kernels enqueued)
int launch_dt(const Geo &G, const Bufs &B, int cur, cudaStream_t st);
int launch_godunov(const Geo &G, const Bufs &B, int cur, cudaStream_t st);   // U[cur] -> U[cur^1]
int launch_fargo(const Geo &G, const Bufs &B, int cur, cudaStream_t st);     // U[cur] -> U[cur^1]
int launch_boundary(const Geo &G, const Bufs &B, int cur, cudaStream_t st);  // in place on U[cur]
int launch_set_scalars(const Bufs &B, double dt, double time, int set_dt, int set_time, cudaStream_t st);
int launch_advance_time(const Bufs &B, cudaStream_t st);
int launch_history(const Geo &G, const Bufs &B, int cur, cudaStream_t st);
// history of any state array U (8 leading variables in the reference layout) with explicit
// scratch (>= history_scratch_doubles(G) doubles) and a 9-double output, all device pointers
int launch_history_ptrs(const Geo &G, const double *U, double *scratch, double *out, cudaStream_t st);
long long history_scratch_doubles(const Geo &G);

// shared host helpers (dg_api.cu)
Geo make_geo(const dg_params &p);
int set_error(int code, const char *msg);
int launch_right_faces(const Geo &G, const double *U, double *out, cudaStream_t st);  // vars 9-11 for download

}  // namespace dg
