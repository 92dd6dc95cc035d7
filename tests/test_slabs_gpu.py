"""The z-slab decomposition on one GPU: the box cut into 2 or 4 slab contexts, stepped with the
halo exchange between them, must end bit-identical (FP64) to the oracle's undecomposed box, with
the same dt every step; the FP32 slabs must equal the FP32 box; the history reduced over the
slabs must match the oracle's at 1e-12 (sums in another order)."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Context, Params, condinit
from dumses_hybrid_b200.slabs import SlabSet, join_states, split_state
from _oracle import Oracle
from test_parity_gpu import MRI_FARGO, OT16, compare_states

pytestmark = pytest.mark.gpu


def run_slabs(box: Params, u0: np.ndarray, nzslice: int, nsteps: int):
    with Context(box) as g:  # the box's ghost fill, as init does before the loop
        g.upload(u0)
        g.boundary(0.0, 0.0)
        u0 = g.download()
    with SlabSet(box, nzslice) as S:
        S.upload(split_state(u0, box, nzslice))
        S.boundary(0.0, 0.0)
        t, dts = 0.0, []
        for _ in range(nsteps):
            t, dt = S.step(t)
            dts.append(dt)
        return join_states(S.download(), box), t, dts, S.history()


def run_oracle(box: Params, u0: np.ndarray, nsteps: int):
    o = Oracle(box)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t, dts = 0.0, []
    for _ in range(nsteps):
        t, dt = o.step(t)
        dts.append(dt)
    return o, t, dts


@pytest.mark.parametrize("nzslice", [2, 4])
def test_slabs_mri_fargo_bit_identical_to_the_box(nzslice):
    box = MRI_FARGO
    u0 = condinit(box, "mri", beta=1000.0, amp=0.1, seed=5)
    us, ts, dts, hist = run_slabs(box, u0, nzslice, 5)
    o, to, dto, = run_oracle(box, u0, 5)
    assert dts == dto and ts == to
    compare_states(us, o.uin, box)
    h = o.history()
    for q in range(8):
        assert abs(hist[q] - h[q]) <= 1e-12 * abs(h[q]) + 1e-18, (q, hist[q], h[q])
    assert abs(hist[8]) < 1e-9


def test_slabs_orszag_tang_bit_identical_to_the_box():
    box = OT16
    u0 = condinit(box, "orszag_tang")
    us, ts, dts, _ = run_slabs(box, u0, 4, 4)
    o, to, dto = run_oracle(box, u0, 4)
    assert dts == dto and ts == to
    compare_states(us, o.uin, box)


def test_slabs_zero_gradient_z_and_dissipation():
    box = Params(**{**MRI_FARGO.__dict__, "bdtypez": "zero_gradient", "nu": 1e-3, "eta": 1e-3})
    u0 = condinit(box, "mri", beta=400.0, amp=0.1, seed=13)
    us, ts, dts, _ = run_slabs(box, u0, 2, 4)
    o, to, dto = run_oracle(box, u0, 4)
    assert dts == dto and ts == to
    compare_states(us, o.uin, box)


def test_fp32_slabs_equal_the_fp32_box():
    box = Params(**{**MRI_FARGO.__dict__, "precision": "fp32"})
    u0 = condinit(box, "mri", beta=1000.0, amp=0.1, seed=5)
    us, ts, dts, _ = run_slabs(box, u0, 4, 5)
    with Context(box) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        t = 0.0
        for _ in range(5):
            dt = g.compute_dt()
            g.godunov(dt, t)
            g.fargo_update(dt)
            g.boundary(t, dt)
            t += dt
        ub = g.download()
    assert t == ts
    assert np.array_equal(us[3:-3, 3:-3, 3:-3, :8], ub[3:-3, 3:-3, 3:-3, :8])


def test_slab_contexts_refuse_the_device_loop():
    from dumses_hybrid_b200 import DumsesError
    from dumses_hybrid_b200.slabs import slab_params
    p = slab_params(MRI_FARGO, 2, 1)
    with Context(p) as g:
        with pytest.raises(DumsesError):
            g.run(1, 0.0)
