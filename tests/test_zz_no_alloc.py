"""dg_history_noalloc: the history sums of a caller-owned device state, for
callers that cannot let the library allocate device memory (a Fortran driver
whose uin lives in its OpenACC runtime, or a job under a fixed device-memory
budget).  Its output must match the context-based dg_history and the oracle's
history routine on the same state, on two calls in a row (the calls share the
library's static scratch array), and the calls after the first must leave the
device's free memory unchanged.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import dumses_hybrid_b200 as dg
from _oracle import Oracle

pytestmark = pytest.mark.gpu

P = dg.Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
              zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
DG_ERR_ARG = -1


def close_sums(got, ref):
    """FP64 sums of the same state in another order: relative 1e-12; div B at round-off."""
    scale = np.maximum(np.abs(ref), 1e-300)
    for q in range(8):
        assert abs(got[q] - ref[q]) <= 1e-12 * scale[q] + 1e-18, (q, got[q], ref[q])
    assert abs(got[8] - ref[8]) <= 1e-12 * max(abs(ref[8]), 1.0), (got[8], ref[8])


def test_history_noalloc_matches_context_history_and_oracle():
    import torch

    lib = dg.load_library()
    u0 = dg.condinit(P, "mri", beta=1000.0, amp=0.1, seed=5)
    with dg.Context(P) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        g.run(3, 0.0)
        ref = g.history()
        u = g.download()
    o = Oracle(P)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t = 0.0
    for _ in range(3):
        t, _ = o.step(t)
    ref_oracle = o.history()
    o.close()
    # the caller's own device copy of uin (reference layout) and output buffers, all made
    # before the calls so that nothing else allocates device memory between them
    d_u = torch.from_numpy(np.ascontiguousarray(u.T)).cuda()
    outs = [torch.full((9,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
    cp = P.to_c()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free = []
    for call, out in enumerate(outs):
        rc = lib.dg_history_noalloc(ctypes.byref(cp), ctypes.c_void_p(d_u.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.dg_last_error()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        got = out.cpu().numpy()
        close_sums(got, ref)
        close_sums(got, ref_oracle)
    # the first call may load the library's module (lazy loading); the later ones allocate nothing
    assert free[1] == free[0] and free[2] == free[0], free


def test_history_noalloc_refuses_host_memory_and_empty_domains():
    import torch

    lib = dg.load_library()
    cp = P.to_c()
    host_u = np.zeros(P.shape, order="F")
    d_out = torch.zeros(9, dtype=torch.float64, device="cuda")
    d_u = torch.zeros(int(np.prod(P.shape)), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    # a host array (a Fortran caller that forgot `host_data use_device`) is refused before any launch
    rc = lib.dg_history_noalloc(ctypes.byref(cp), ctypes.c_void_p(host_u.ctypes.data), ctypes.c_void_p(d_out.data_ptr()),
                                None)
    assert rc == DG_ERR_ARG and b"device or managed memory" in lib.dg_last_error()
    host_out = np.zeros(9)
    rc = lib.dg_history_noalloc(ctypes.byref(cp), ctypes.c_void_p(d_u.data_ptr()), ctypes.c_void_p(host_out.ctypes.data),
                                None)
    assert rc == DG_ERR_ARG
    empty = dg.Params(**{**P.__dict__, "xmax": P.xmin}).to_c()
    rc = lib.dg_history_noalloc(ctypes.byref(empty), ctypes.c_void_p(d_u.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                None)
    assert rc == DG_ERR_ARG and b"empty domain" in lib.dg_last_error()
    # and the library still works afterwards
    rc = lib.dg_history_noalloc(ctypes.byref(cp), ctypes.c_void_p(d_u.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                None)
    assert rc == 0, lib.dg_last_error()
    torch.cuda.synchronize()


def test_history_noalloc_rejects_oversized_grid():
    lib = dg.load_library()
    big = dg.Params(ndim=3, nx=dg_max_nx() + 1, ny=8, nz=8).to_c()
    rc = lib.dg_history_noalloc(ctypes.byref(big), ctypes.c_void_p(1), ctypes.c_void_p(1), None)
    assert rc == DG_ERR_ARG
    assert b"DG_HISTORY_NOALLOC_MAX_NX" in lib.dg_last_error()


def dg_max_nx() -> int:
    import pathlib
    import re
    h = (pathlib.Path(dg.__file__).resolve().parents[1] / "include" / "dumses_gpu.h").read_text()
    return int(re.search(r"#define DG_HISTORY_NOALLOC_MAX_NX (\d+)", h).group(1))
