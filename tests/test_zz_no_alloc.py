"""dg_history_noalloc: the history sums of a caller-owned device state, for
callers that cannot let the library allocate device memory (a Fortran driver
whose uin lives in its OpenACC runtime, or a job under a fixed device-memory
budget).  Its output must match the context-based dg_history on the same state,
on two calls in a row (the calls share the library's static scratch array).
This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import dumses_hybrid_b200 as dg

pytestmark = pytest.mark.gpu

P = dg.Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
              zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)


def test_history_noalloc_matches_context_history():
    import torch

    lib = dg.load_library()
    u0 = dg.condinit(P, "mri", beta=1000.0, amp=0.1, seed=5)
    with dg.Context(P) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        g.run(3, 0.0)
        ref = g.history()
        u = g.download()
    # the caller's own device copy of uin (reference layout) and output buffer
    d_u = torch.from_numpy(np.ascontiguousarray(u.T)).cuda()
    cp = P.to_c()
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((9,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.dg_history_noalloc(ctypes.byref(cp), ctypes.c_void_p(d_u.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.dg_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        scale = np.maximum(np.abs(ref), 1e-300)
        for q in range(8):
            assert abs(got[q] - ref[q]) <= 1e-12 * scale[q] + 1e-18, (call, q, got[q], ref[q])
        assert abs(got[8] - ref[8]) <= 1e-12 * max(abs(ref[8]), 1.0), (call, got[8], ref[8])


def test_history_noalloc_rejects_oversized_grid():
    lib = dg.load_library()
    big = dg.Params(ndim=3, nx=dg_max_nx() + 1, ny=8, nz=8).to_c()
    rc = lib.dg_history_noalloc(ctypes.byref(big), ctypes.c_void_p(1), ctypes.c_void_p(1), None)
    assert rc == -1
    assert b"DG_HISTORY_NOALLOC_MAX_NX" in lib.dg_last_error()


def dg_max_nx() -> int:
    import pathlib
    import re
    h = (pathlib.Path(dg.__file__).resolve().parents[1] / "include" / "dumses_gpu.h").read_text()
    return int(re.search(r"#define DG_HISTORY_NOALLOC_MAX_NX (\d+)", h).group(1))
