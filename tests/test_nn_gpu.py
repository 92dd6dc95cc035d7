"""The flux network on the GPU: tcgen05 forward and backward against the FP64 numpy
oracle (BF16 rounding emulated at the same points), the Adam step, training on
interfaces harvested from the FP32 path with HLLD labels, and the surrogate inside the
step with its HLLD fallback.

Tolerances: forward outputs and gradients agree with the oracle to a relative L2 error
of 2e-3 per layer (FP32 accumulation order, occasional BF16 rounding flips)."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Context, FluxNet, Params, condinit
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def random_params(net, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = []
    for k, n in net.shapes:
        p.append(rng.normal(0, scale * np.sqrt(2.0 / k), k * n))
        p.append(rng.normal(0, 0.1, n))
    p = np.concatenate(p).astype(np.float32)
    net.set_params(p)
    return p.astype(np.float64)


def layer_slices(net):
    out, off = [], 0
    for k, n in net.shapes:
        out.append(slice(off, off + k * n))
        off += k * n
        out.append(slice(off, off + n))
        off += n
    return out


def test_param_roundtrip():
    with FluxNet(seed=7) as net:
        p = net.params()
        assert p.size == sum(k * n + n for k, n in net.shapes) and np.isfinite(p).all() and np.abs(p).max() > 0
        assert net.shapes == mo.shapes(*net.shape)
        assert p.size == {(64, 1): 1672, (64, 2): 5832, (128, 3): 36360}.get(net.shape, p.size)
        net.set_params(p * 0.5)
        assert np.array_equal(net.params(), (p * 0.5).astype(np.float32))


@pytest.mark.parametrize("rows", [128, 1000])
def test_forward_matches_oracle(rows):
    rng = np.random.default_rng(rows)
    with FluxNet() as net:
        p = random_params(net, 11)
        x = rng.normal(0, 1, (rows, 17)).astype(np.float32)
        y = net.forward(x)
        yo, _ = mo.forward(p, x.astype(np.float64), shp=net.shapes)
        assert rel(y, yo) < 2e-3, rel(y, yo)


@pytest.mark.parametrize("batch", [256, 1024])
def test_gradients_match_oracle(batch):
    rng = np.random.default_rng(batch)
    with FluxNet() as net:
        p = random_params(net, 12)
        x = rng.normal(0, 1, (batch, 17)).astype(np.float32)
        t = rng.normal(0, 1, (batch, 8)).astype(np.float32)
        loss, g = net.gradients(x, t)
        lo, go = mo.loss_and_grad(p, x.astype(np.float64), t.astype(np.float64), shp=net.shapes)
        assert abs(loss - lo) <= 1e-3 * lo
        for s in layer_slices(net):
            assert rel(g[s], go[s]) < 2e-3, (s, rel(g[s], go[s]))


def test_adam_step_matches_oracle():
    rng = np.random.default_rng(5)
    with FluxNet() as net:
        p = random_params(net, 13)
        x1 = rng.normal(0, 1, (1, 17))
        t1 = rng.normal(0, 1, (1, 8))
        x = np.repeat(x1, 256, axis=0).astype(np.float32)  # every drawn batch is the same
        t = np.repeat(t1, 256, axis=0).astype(np.float32)
        _, g = net.gradients(x, t)
        net.set_samples(x, t)
        net.train(1, batch=256, lr=1e-3)
        p1 = net.params().astype(np.float64)
        po, _, _ = mo.adam_step(p, g.astype(np.float64), np.zeros_like(p), np.zeros_like(p), 1)
        moved = np.abs(g) > 1e-6 * np.abs(g).max()
        assert np.allclose(p1[moved], po[moved], rtol=0, atol=2e-6)


def test_training_fits_a_smooth_map():
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, (1 << 16, 17)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0] + x[:, 1]), x[:, 2] * x[:, 3], np.tanh(x[:, 4] - x[:, 5]), x[:, 6] ** 2,
                  np.cos(x[:, 7]), x[:, 8] - x[:, 9], 0.5 * x[:, 10] * x[:, 11], x[:, 12] + x[:, 16]], 1).astype(np.float32)
    with FluxNet(seed=3) as net:
        net.set_samples(x, t)
        l0 = net.train(1, batch=8192, lr=1e-3)
        l1 = net.train(600, batch=8192, lr=1e-3)
        print("loss", l0, "->", l1)
        assert l1 < 0.05 * l0


def ot_params(n, precision="fp32", surrogate=False):
    return Params(ndim=3, nx=n, ny=n, nz=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3,
                  courant=0.8, precision=precision, surrogate=surrogate)


def train_on_ot(net, n=32, snapshots=4, steps_between=5, train_steps=2400):
    p = ot_params(n)
    with Context(p) as g:
        g.upload(condinit(p, "orszag_tang"))
        g.boundary(0.0, 0.0)
        t = 0.0
        for _ in range(snapshots):
            t, _ = g.run(steps_between, t)
            net.harvest(g)
    x, y = net.samples()
    assert np.isfinite(x).all() and np.isfinite(y).all()
    net.fit_envelope(0.0)
    net.fit_scaling()
    for lr in (1e-3, 3e-4, 1e-4):
        loss = net.train(train_steps // 3, batch=8192, lr=lr)
    return loss


def mri_params(n, precision="fp32", surrogate=False):
    return Params(ndim=3, iso=1, nx=n, ny=n, nz=n, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5, zmin=-0.5, zmax=0.5,
                  ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True, precision=precision,
                  surrogate=surrogate)


def test_harvest_labels_and_network_learns():
    """Held-out interfaces of a shearing-box MRI run: per flux component, LLF + the learned
    correction is much closer to HLLD than LLF alone (what the network has learned; its gain
    over the method without it, FP32 with exact HLLD, is measured by the next test)."""
    p = mri_params(48)
    with FluxNet(seed=2) as net, FluxNet(seed=9) as probe, Context(p) as g:
        g.upload(condinit(p, "mri", beta=1000.0, amp=0.1, seed=2024))
        g.boundary(0.0, 0.0)
        t = 0.0
        for _ in range(4):
            t, _ = g.run(5, t)
            net.harvest(g)
        t, _ = g.run(7, t)
        probe.harvest(g, stride=3)
        xh, th = probe.samples()
        net.fit_envelope(0.0)
        net.fit_scaling()
        for lr in (1e-3, 3e-4, 1e-4):
            loss = net.train(800, batch=8192, lr=lr)
        yh = net.forward(xh)
        jump = xh[:, 14:15]  # targets are per unit jump: weigh by the jump to compare fluxes
        # per output: L1 error of LLF + network against HLLD over that of LLF alone (correction 0)
        ratio = np.sum(np.abs(yh - th) * jump, 0) / np.sum(np.abs(th) * jump, 0)
        print("samples", net.sample_count, "train loss", loss, "held-out error ratio per output",
              np.array2string(ratio, precision=3))
        assert np.mean(ratio) < 0.2 and np.max(ratio) < 0.6


def l1_rel(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


def test_network_against_fp32_hlld():
    """What the trained network gains over the method without it: the FP32 path with the learned
    face flux against the FP32 path with exact HLLD, both from the same shearing-box state, both
    measured against the FP64 path after 20 steps (relative L1 over the active cells), and the
    face work of each step timed with the library's per-kernel CUDA events.  Tolerances: the FP32
    path within 1e-4, the learned flux within 1e-1 (measured 4-5e-2 in B on this turbulent box,
    where the Orszag-Tang test above holds it to 2e-2); the measured gains are printed: on this
    problem the network loses accuracy against exact HLLD (error ratios of order 1e4) and time
    (its face kernel costs more than the HLLD face solves it replaces)."""
    n = 48
    u0 = condinit(mri_params(n), "mri", beta=1000.0, amp=0.1, seed=2024)
    with FluxNet(seed=2) as net:
        with Context(mri_params(n)) as g:
            g.upload(u0)
            g.boundary(0.0, 0.0)
            t = 0.0
            for _ in range(4):
                t, _ = g.run(5, t)
                net.harvest(g)
        net.fit_envelope(0.0)
        net.fit_scaling()
        for lr in (1e-3, 3e-4, 1e-4):
            net.train(800, batch=8192, lr=lr)
        res, face_ms = {}, {}
        for name, prec, sur in (("fp64", "fp64", False), ("fp32", "fp32", False), ("fp32nn", "fp32", True)):
            with Context(mri_params(n, prec, sur)) as g:
                if sur:
                    g.attach_surrogate(net)
                g.upload(u0)
                g.boundary(0.0, 0.0)
                g.run(3, 0.0)
                g.profile(True)
                g.profile_read()
                g.run(20, 0.0)
                prof = g.profile_read()
                res[name] = g.download()[3:-3, 3:-3, 3:-3, :8]
                face_ms[name] = {k: v[0] / 20 for k, v in prof.items() if k in ("riemann_flux_emf", "nn_faces",
                                                                                 "nn_fallback")}
    err = {k: {v: l1_rel(res[k][..., q], res["fp64"][..., q]) for q, v in ((0, "rho"), (5, "Bx"), (6, "By"), (7, "Bz"))}
           for k in ("fp32", "fp32nn")}
    gain = {v: err["fp32nn"][v] / max(err["fp32"][v], 1e-300) for v in err["fp32"]}
    print("relative L1 vs FP64 after 20 steps:", err)
    print("error of the learned flux over that of exact HLLD (FP32):", gain)
    print("Riemann/face kernels, ms per step:", face_ms)
    assert max(err["fp32"].values()) < 1e-4
    assert max(err["fp32nn"].values()) < 1e-1
    assert all(np.isfinite(list(gain.values())))


def test_surrogate_step_with_fallback():
    """The network inside the FP32 step: some faces fall back to HLLD, the state stays
    close to the plain FP64 run and div B stays at round-off."""
    with FluxNet(seed=2) as net:
        train_on_ot(net)
        net.set_gates(jump=0.1, compress=0.1)
        res = {}
        for prec, sur in (("fp64", False), ("fp32", False), ("fp32", True)):
            p = ot_params(32, prec, sur)
            with Context(p) as g:
                if sur:
                    g.attach_surrogate(net)
                g.upload(condinit(p, "orszag_tang"))
                g.boundary(0.0, 0.0)
                g.run(20, 0.0)
                res[(prec, sur)] = g.download()
                if sur:
                    faces, fallback = g.surrogate_stats()
                    hist = g.history()
        print("faces", faces, "fallback", fallback, "fraction", fallback / faces)
        assert faces == 20 * 3 * 32 * 32 * 33
        assert 0 < fallback < faces
        a64 = res[("fp64", False)][3:-3, 3:-3, 3:-3]
        for key in (("fp32", False), ("fp32", True)):
            a = res[key][3:-3, 3:-3, 3:-3]
            errs = [l1_rel(a[..., v], a64[..., v]) for v in (0, 4, 5, 6)]
            print(key, "L1 rel rho E Bx By", ["%.2e" % e for e in errs])
        a = res[("fp32", True)][3:-3, 3:-3, 3:-3]
        for v in (0, 4, 5, 6):
            assert l1_rel(a[..., v], a64[..., v]) < 2e-2
        assert abs(hist[8]) < 1e-10


def test_surrogate_in_2d():
    """The learned flux on the 2D field loop (NDIM = 2 face records with the B_z flux):
    trained on its own interfaces, finite, div B at round-off, close to the FP64 run."""
    def loop(precision, surrogate=False):
        return Params(ndim=2, nx=64, ny=32, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7,
                      precision=precision, surrogate=surrogate)
    with FluxNet(seed=4) as net:
        p = loop("fp32")
        u0 = condinit(p, "field_loop")
        with Context(p) as g:
            g.upload(u0)
            g.boundary(0.0, 0.0)
            t = 0.0
            for _ in range(3):
                t, _ = g.run(5, t)
                net.harvest(g)
        net.fit_envelope(0.0)
        net.fit_scaling()
        for lr in (1e-3, 3e-4, 1e-4):
            net.train(300, batch=4096, lr=lr)
        out = {}
        for prec, sur in (("fp64", False), ("fp32", True)):
            q = loop(prec, sur)
            with Context(q) as g:
                if sur:
                    g.attach_surrogate(net)
                g.upload(u0)
                g.boundary(0.0, 0.0)
                g.run(20, 0.0)
                out[prec] = g.download()
                if sur:
                    faces, fallback = g.surrogate_stats()
        a, b = out["fp32"][3:-3, 3:-3, 0], out["fp64"][3:-3, 3:-3, 0]
        assert faces == 20 * (65 * 32 + 64 * 33) and fallback < faces
        assert np.isfinite(a[..., :8]).all()
        errs = [l1_rel(a[..., v], b[..., v]) for v in (0, 4, 5, 6)]
        print("2D loop, faces", faces, "fallback", fallback, "L1 rel rho E Bx By", ["%.2e" % e for e in errs])
        assert max(errs) < 2e-2
        bx, by = out["fp32"][..., 5], out["fp32"][..., 6]
        divb = (bx[4:-2, 3:-3, 0] - bx[3:-3, 3:-3, 0]) + (by[3:-3, 4:-2, 0] - by[3:-3, 3:-3, 0])
        # CT keeps div B at the round-off of the FP32 increments (about 1e-8 of |B| per face difference)
        assert np.max(np.abs(divb)) < 1e-6 * max(np.max(np.abs(bx)), 1e-30)


def effective_face_fluxes(g, p, dt):
    """Face records of the last godunov of a 3D context as (faces, 5) effective fluxes: mass,
    energy and the three momentum fluxes, the normal one with p*_T added back (the 1D
    solvers that carry p*_T separately leave it out of the normal momentum flux)."""
    nf = (p.nx + 1) * (p.ny + 1) * (p.nz + 1)
    dx, dy, dz = (p.xmax - p.xmin) / p.nx, (p.ymax - p.ymin) / p.ny, (p.zmax - p.zmin) / p.nz
    ds = (dy * dz, dx * dz, dx * dy)
    k, j, i = np.meshgrid(np.arange(1, p.nz + 2), np.arange(1, p.ny + 2), np.arange(1, p.nx + 2), indexing="ij")
    valid = ((j <= p.ny) & (k <= p.nz), (i <= p.nx) & (k <= p.nz), (i <= p.nx) & (j <= p.ny))
    out = []
    for d in range(3):
        rec = g.debug_array(d, 6 * nf).reshape(p.nz + 1, p.ny + 1, p.nx + 1, 6)
        eff = rec[..., :5].copy()
        eff[..., 2 + d] += rec[..., 5] * ds[d] * dt
        out.append(eff[valid[d]])
    return np.concatenate(out)


def test_face_network_kernel_against_hlld_and_llf():
    """The inference kernel of the step (k_nn_faces) on its own: after one godunov from the
    same state, the faces it accepted (its count agrees with the kernel's own) carry fluxes
    much closer to HLLD than LLF's, as the held-out test of the network predicts; the faces
    it sent back carry the HLLD flux.  A wrong weight or bias operand in the kernel would
    either move the accepted fluxes away from HLLD or get nearly every face sent back."""
    with FluxNet(seed=2) as net:
        train_on_ot(net)
        net.set_gates(jump=0.1, compress=0.1)
        eff, stats = {}, None
        for name, riemann, sur in (("hlld", "hlld", False), ("llf", "llf", False), ("nn", "hlld", True)):
            p = Params(**{**ot_params(32, "fp32", sur).__dict__, "riemann": riemann})
            with Context(p) as g:
                if sur:
                    g.attach_surrogate(net)
                g.upload(condinit(p, "orszag_tang"))
                g.boundary(0.0, 0.0)
                dt = g.compute_dt()
                g.godunov(dt, 0.0)
                eff[name] = effective_face_fluxes(g, p, dt)
                if sur:
                    stats = g.surrogate_stats()
        faces, fallback = stats
        assert faces == eff["nn"].shape[0]
        dn = np.abs(eff["nn"] - eff["hlld"]).sum(axis=1)
        dl = np.abs(eff["llf"] - eff["hlld"]).sum(axis=1)
        accepted = dn > 1e-3 * dl + 1e-30
        print("faces", faces, "fallback", fallback, "classified accepted", int(accepted.sum()))
        assert abs(int(accepted.sum()) - (faces - fallback)) <= 0.01 * faces
        assert faces - fallback >= 0.1 * faces
        ratio = dn[accepted].sum() / dl[accepted].sum()
        print("accepted faces: L1(network - HLLD) / L1(LLF - HLLD) =", ratio)
        assert ratio < 0.5
        # faces sent back carry HLLD (the same solver in another kernel)
        back = ~accepted
        assert np.abs(eff["nn"][back] - eff["hlld"][back]).sum() <= 1e-4 * np.abs(eff["hlld"][back]).sum()
