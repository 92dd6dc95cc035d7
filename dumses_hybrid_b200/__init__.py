"""dumses_hybrid_b200: the DUMSES-Hybrid Godunov MHD step on B200 (sm_100a).

Python mirror of the reference's operator interface for the hot path.  The
reference calls argument-less Fortran subroutines on module globals from its
driver loop (src/dumses.f90:82-120); the same calls exist here as methods of
:class:`Context`, which wraps one context of the C-ABI library
``libdumses_gpu.so`` (include/dumses_gpu.h):

    reference                         here
    ---------------------------------  ------------------------------------
    call compute_dt(dt)                dt = ctx.compute_dt()
    call godunov                       ctx.godunov(dt, time)
    if (fargo) call fargo_update       ctx.fargo_update(dt)
    call boundary                      ctx.boundary(time, dt)
    call dissipation (nu or eta > 0)   ctx.dissipation(time, dt)
    call history (MRI problem)         ctx.history()
    !$acc update host(uin)             uin = ctx.download()

Arrays use the reference layout: numpy arrays of shape
(nx+6, ny+6, nz+6, 11) in Fortran order (uin(iu1:iu2,ju1:ju2,ku1:ku2,1:11)).

There is no CPU fallback: if the library is missing or no GPU is visible the
calls raise.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import re
from dataclasses import dataclass

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
# DG_LIBRARY selects another build of the library, e.g. the bounds-checked libdumses_gpu_chk.so
LIB_PATH = pathlib.Path(os.environ["DG_LIBRARY"]) if os.environ.get("DG_LIBRARY") else PKG / "libdumses_gpu.so"

DG_OK = 0
ERRORS = {-1: "DG_ERR_ARG", -2: "DG_ERR_CUDA", -3: "DG_ERR_NOMEM", -4: "DG_ERR_TIMEOUT", -5: "DG_ERR_STATE",
          -6: "DG_ERR_DT", -7: "DG_ERR_NODEVICE", -8: "DG_ERR_UNSUPPORTED"}
RIEMANN = {"llf": 2, "hll": 3, "hlld": 4, "upwind": 5, "hlla": 8}
HISTORY_VARIANTS = {"mri": 0, "default": 1}  # DG_HISTORY_MRI, DG_HISTORY_DEFAULT
BC = {"periodic": 0, "zero_gradient": 1, "shearingbox": 2}
IC = {"field_loop": 1, "orszag_tang": 2, "mri": 3, "mri_test": 4}
PREC = {"fp64": 0, "fp32": 1}


class DgParams(ctypes.Structure):
    """ctypes mirror of ``dg_params`` (include/dumses_gpu.h)."""
    _fields_ = [("ndim", ctypes.c_int), ("iso", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("nz", ctypes.c_int), ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymin", ctypes.c_double), ("ymax", ctypes.c_double), ("zmin", ctypes.c_double),
                ("zmax", ctypes.c_double), ("gamma", ctypes.c_double), ("ciso", ctypes.c_double),
                ("omega0", ctypes.c_double), ("courant", ctypes.c_double), ("slope_type", ctypes.c_int),
                ("iriemann", ctypes.c_int), ("iriemann2d", ctypes.c_int), ("bc", ctypes.c_int * 3),
                ("fargo", ctypes.c_int), ("precision", ctypes.c_int), ("surrogate", ctypes.c_int),
                ("device", ctypes.c_int), ("nu", ctypes.c_double), ("eta", ctypes.c_double),
                ("nzslice", ctypes.c_int), ("zposition", ctypes.c_int), ("reserved", ctypes.c_int * 4)]


class DgDumpInfo(ctypes.Structure):
    """ctypes mirror of ``dg_dump_info`` (include/dumses_gpu.h)."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nxslice", ctypes.c_int),
                ("nyslice", ctypes.c_int), ("nzslice", ctypes.c_int), ("time", ctypes.c_double),
                ("dt", ctypes.c_double), ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double),
                ("ymax", ctypes.c_double), ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
                ("gamma", ctypes.c_double), ("ciso", ctypes.c_double), ("uin_bytes", ctypes.c_longlong)]


class DumsesError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load_library(path: str | pathlib.Path | None = None) -> ctypes.CDLL:
    """Load libdumses_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python -m dumses_hybrid_b200.build`")
    lib = ctypes.CDLL(str(p))
    c_p = ctypes.POINTER(DgParams)
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    fp = ctypes.POINTER(ctypes.c_float)
    sig = {
        "dg_default_params": (None, [c_p]),
        "dg_uin_size": (ctypes.c_longlong, [c_p]),
        "dg_init": (ctypes.c_int, [c_p, ctypes.POINTER(vp)]),
        "dg_finalize": (ctypes.c_int, [vp]),
        "dg_upload": (ctypes.c_int, [vp, dp]),
        "dg_download": (ctypes.c_int, [vp, dp]),
        "dg_compute_dt": (ctypes.c_int, [vp, dp]),
        "dg_godunov": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double]),
        "dg_fargo_update": (ctypes.c_int, [vp, ctypes.c_double]),
        "dg_boundary": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double]),
        "dg_run": (ctypes.c_int, [vp, ctypes.c_int, dp, dp]),
        "dg_dissipation": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double]),
        "dg_step": (ctypes.c_int, [vp, dp, dp]),
        "dg_history": (ctypes.c_int, [vp, dp]),
        "dg_history_variant": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "dg_dump_header": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(DgDumpInfo)]),
        "dg_dump_write": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_double, ctypes.c_double]),
        "dg_dump_read": (ctypes.c_int, [vp, ctypes.c_char_p, dp, dp]),
        "dg_dump_write_host": (ctypes.c_int, [ctypes.c_char_p, c_p, ctypes.c_double, ctypes.c_double, dp]),
        "dg_dump_read_host": (ctypes.c_int, [ctypes.c_char_p, c_p, dp, dp, dp]),
        "dg_sync": (ctypes.c_int, [vp]),
        "dg_kernel_launches": (ctypes.c_longlong, [vp]),
        "dg_stream": (vp, [vp]),
        "dg_last_error": (ctypes.c_char_p, []),
        "dg_history_noalloc": (ctypes.c_int, [c_p, vp, vp, vp]),
        "dg_halo_count": (ctypes.c_longlong, [vp]),
        "dg_halo_pack": (ctypes.c_int, [vp, ctypes.c_int, vp]),
        "dg_halo_unpack": (ctypes.c_int, [vp, ctypes.c_int, vp]),
        "dg_history_columns": (ctypes.c_int, [vp, dp]),
        "dg_history_share": (ctypes.c_int, [vp, dp, dp]),
        "dg_profile": (ctypes.c_int, [vp, ctypes.c_int]),
        "dg_profile_read": (ctypes.c_int, [vp, dp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
        "dg_profile_slot_name": (ctypes.c_char_p, [ctypes.c_int]),
        "dg_debug_copy": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
        "dg_condinit": (ctypes.c_int, [c_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong, dp]),
        "dg_nn_param_count": (ctypes.c_longlong, []),
        "dg_nn_shape": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
        "dg_nn_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(vp)]),
        "dg_nn_destroy": (ctypes.c_int, [vp]),
        "dg_nn_set_samples": (ctypes.c_int, [vp, fp, fp, ctypes.c_longlong]),
        "dg_nn_reserve_samples": (ctypes.c_int, [vp, ctypes.c_longlong]),
        "dg_nn_sample_count": (ctypes.c_longlong, [vp]),
        "dg_nn_samples_copy": (ctypes.c_int, [vp, ctypes.c_longlong, ctypes.c_longlong, fp, fp]),
        "dg_nn_harvest": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
        "dg_nn_train": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, fp]),
        "dg_nn_gradients": (ctypes.c_int, [vp, fp, fp, ctypes.c_int, fp, fp]),
        "dg_nn_forward": (ctypes.c_int, [vp, fp, ctypes.c_longlong, fp]),
        "dg_nn_get_params": (ctypes.c_int, [vp, fp, ctypes.c_longlong]),
        "dg_nn_set_params": (ctypes.c_int, [vp, fp, ctypes.c_longlong]),
        "dg_nn_fit_envelope": (ctypes.c_int, [vp, ctypes.c_float]),
        "dg_nn_fit_scaling": (ctypes.c_int, [vp]),
        "dg_nn_set_gates": (ctypes.c_int, [vp, ctypes.c_float, ctypes.c_float]),
        "dg_attach_surrogate": (ctypes.c_int, [vp, vp]),
        "dg_wait_selftest": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, dp]),
        "dg_debug_oob_count": (ctypes.c_longlong, []),
        "dg_surrogate_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    if path is None:
        _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != DG_OK:
        raise DumsesError(rc, load_library().dg_last_error().decode())


@dataclass
class Params:
    """The reference's &scheme_params / &model_params plus NDIM and ISO."""
    ndim: int = 3
    iso: int = 0
    nx: int = 256
    ny: int = 256
    nz: int = 256
    xmin: float = 0.0
    xmax: float = 1.0
    ymin: float = -0.5
    ymax: float = 0.5
    zmin: float = 0.0
    zmax: float = 1.0
    gamma: float = 5.0 / 3.0
    ciso: float = 0.0
    omega0: float = 0.0
    courant: float = 0.7
    slope_type: int = 2
    riemann: str = "hlld"
    riemann2d: str = "hlld"
    bdtypex: str = "periodic"
    bdtypey: str = "periodic"
    bdtypez: str = "periodic"
    fargo: bool = False
    precision: str = "fp64"
    surrogate: bool = False
    device: int = 0
    nu: float = 0.0
    eta: float = 0.0
    nzslice: int = 1      # z slabs of a decomposed box (nz = this slab's share)
    zposition: int = 0    # this slab's place, 0 .. nzslice-1

    def to_c(self) -> DgParams:
        p = DgParams()
        p.ndim, p.iso, p.nx, p.ny, p.nz = self.ndim, int(self.iso), self.nx, self.ny, self.nz
        p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax = self.xmin, self.xmax, self.ymin, self.ymax, self.zmin, self.zmax
        p.gamma, p.ciso, p.omega0, p.courant = self.gamma, self.ciso, self.omega0, self.courant
        p.slope_type = self.slope_type
        p.iriemann, p.iriemann2d = RIEMANN[self.riemann], RIEMANN[self.riemann2d]
        p.bc[0], p.bc[1], p.bc[2] = BC[self.bdtypex], BC[self.bdtypey], BC[self.bdtypez]
        p.fargo, p.precision, p.surrogate, p.device = int(self.fargo), PREC[self.precision], int(self.surrogate), self.device
        p.nu, p.eta = self.nu, self.eta
        p.nzslice, p.zposition = self.nzslice, self.zposition
        return p

    @property
    def shape(self) -> tuple[int, int, int, int]:
        return (self.nx + 6, self.ny + 6 if self.ndim > 1 else 1, self.nz + 6 if self.ndim == 3 else 1, 11)


def _strip_namelist_comments(text: str) -> str:
    """Drop Fortran comments ('!' to the end of the line, outside quoted strings)."""
    out = []
    for line in text.splitlines():
        quote = None
        for k, ch in enumerate(line):
            if quote:
                if ch == quote:
                    quote = None
            elif ch in "'\"":
                quote = ch
            elif ch == "!":
                line = line[:k]
                break
        out.append(line)
    return "\n".join(out)


def read_namelist(path: str | pathlib.Path, ndim: int = 3, iso: int = 0) -> Params:
    """Build :class:`Params` from a reference ``input`` namelist file
    (&scheme_params, &model_params; init.f90:153-173), applying the reference
    defaults (init.f90:244-302) for keys the file does not set."""
    text = _strip_namelist_comments(pathlib.Path(path).read_text())
    kv = {}
    for m in re.finditer(r"([A-Za-z0-9_]+)\s*=\s*('[^']*'|\"[^\"]*\"|[^,\s/]+)", text):
        kv[m.group(1).lower()] = m.group(2).strip("'\"")

    def num(s: str) -> float:
        return float(s.lower().replace("d", "e"))

    p = Params(ndim=ndim, iso=iso)
    for key in ("nx", "ny", "nz", "slope_type"):
        if key in kv:
            setattr(p, key, int(kv[key]))
    for key in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "gamma", "ciso", "courant", "nu", "eta"):
        if key in kv:
            setattr(p, key, num(kv[key]))
    if "omega0" in kv:
        p.omega0 = num(kv["omega0"])
    for key in ("riemann", "riemann2d", "bdtypex", "bdtypey", "bdtypez"):
        if key in kv:
            setattr(p, key, kv[key].strip().lower())
    if "fargo" in kv:
        p.fargo = kv["fargo"].strip(".").lower().startswith("t")
    if ndim < 3:
        p.nz = 1
    return p


def condinit(params: Params, ic: str, beta: float = 1000.0, amp: float = 0.0, seed: int = 0) -> np.ndarray:
    """Initial conditions in the reference layout (host-side, no GPU needed)."""
    lib = load_library()
    cp = params.to_c()
    u = np.zeros(params.shape, dtype=np.float64, order="F")
    _check(lib.dg_condinit(ctypes.byref(cp), IC[ic], beta, amp, seed, u.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return u


def dump_filename(ndump: int, mype: int = 0, base: str | pathlib.Path = ".", make_dir: bool = True) -> pathlib.Path:
    """Path of dump `ndump` of rank `mype` as the reference names it: get_filename
    (src/modules/file.f90) gives output_NNNNNN/data.RRRRRR, output.f90:225 adds .bin."""
    d = pathlib.Path(base) / f"output_{ndump % 1000000:06d}"
    if make_dir:
        d.mkdir(parents=True, exist_ok=True)
    return d / f"data.{mype % 1000000:06d}.bin"


def dump_header(path: str | pathlib.Path) -> dict:
    """Header records of a 'binary' dump (output.f90:228-231) and the byte length of its uin record."""
    info = DgDumpInfo()
    _check(load_library().dg_dump_header(str(path).encode(), ctypes.byref(info)))
    return {name: getattr(info, name) for name, _ in DgDumpInfo._fields_}


def write_dump(path: str | pathlib.Path, params: Params, uin: np.ndarray, time: float, dt: float) -> None:
    """Write a host uin array as a 'binary' dump (output.f90:224-235)."""
    if uin.shape != params.shape or uin.dtype != np.float64 or not uin.flags.f_contiguous:
        raise ValueError(f"uin must be a Fortran-ordered float64 array of shape {params.shape}")
    cp = params.to_c()
    _check(load_library().dg_dump_write_host(str(path).encode(), ctypes.byref(cp), time, dt,
                                             uin.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))


def read_dump(path: str | pathlib.Path, params: Params) -> tuple[np.ndarray, float, float]:
    """Read a 'binary' dump of the grid of `params` (restart.f90:212-221): (uin, time, dt)."""
    cp = params.to_c()
    u = np.zeros(params.shape, dtype=np.float64, order="F")
    t, dt = ctypes.c_double(), ctypes.c_double()
    _check(load_library().dg_dump_read_host(str(path).encode(), ctypes.byref(cp), ctypes.byref(t), ctypes.byref(dt),
                                            u.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return u, t.value, dt.value


HISTORY_KEYS = ("time", "dt", "mass", "maxwell", "reynolds", "max+rey", "magp", "meanBx", "meanBy", "meanBz", "divB")


def _fortran_1pe(x: float, w: int) -> str:
    """Fortran edit 1PEw.5: one digit before the point, five after; a three-digit
    exponent drops the E (d.ddddd+ddd), as the Fortran standard prescribes."""
    s = f"{x:.5E}"
    mant, exp = s.split("E")
    if len(exp) > 3:  # sign + three digits
        s = mant + exp
    return s.rjust(w)


def history_header() -> str:
    """Header line of the MRI history file, format ('# ', A11, 1X, A12, 1X, 9(A14,1X))
    (src/problem/mri/history.f90:152-154)."""
    k = HISTORY_KEYS
    return "# " + k[0].rjust(11) + " " + k[1].rjust(12) + " " + "".join(n.rjust(14) + " " for n in k[2:])


def history_line(time: float, dt: float, sums: np.ndarray) -> str:
    """One line of the MRI history file for the sums of :meth:`Context.history`, format
    (1X, 1PE12.5, 1X, 1PE12.5, 1X, 9(E14.5,1X)) (history.f90:166-168); the scale factor
    1P carries over to the E14.5 fields."""
    vals = [float(v) for v in sums]
    return " " + _fortran_1pe(time, 12) + " " + _fortran_1pe(dt, 12) + " " + "".join(
        _fortran_1pe(v, 14) + " " for v in vals)


def write_history(path: str | pathlib.Path, time: float, dt: float, sums: np.ndarray) -> None:
    """Append one line to history.txt as the MRI history routine does: a new file (or
    time = 0) starts with the header line (history.f90:150-164)."""
    path = pathlib.Path(path)
    fresh = time == 0.0 or not path.exists()
    with open(path, "w" if fresh else "a") as f:
        if fresh:
            f.write(history_header() + "\n")
        f.write(history_line(time, dt, sums) + "\n")


class Context:
    """One device state of the MHD step (a dg_ctx of the C-ABI)."""

    def __init__(self, params: Params):
        self.params = params
        self.lib = load_library()
        self._cp = params.to_c()
        h = ctypes.c_void_p()
        _check(self.lib.dg_init(ctypes.byref(self._cp), ctypes.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.dg_finalize(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(a: np.ndarray):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def upload(self, uin: np.ndarray) -> None:
        if uin.shape != self.params.shape or uin.dtype != np.float64 or not uin.flags.f_contiguous:
            raise ValueError(f"uin must be a Fortran-ordered float64 array of shape {self.params.shape}")
        _check(self.lib.dg_upload(self.h, self._ptr(uin)))

    def download(self) -> np.ndarray:
        u = np.zeros(self.params.shape, dtype=np.float64, order="F")
        _check(self.lib.dg_download(self.h, self._ptr(u)))
        return u

    def download_into(self, uin: np.ndarray) -> None:
        """Download into a caller-owned Fortran-ordered float64 array (e.g. pinned memory)."""
        if uin.shape != self.params.shape or uin.dtype != np.float64 or not uin.flags.f_contiguous:
            raise ValueError(f"uin must be a Fortran-ordered float64 array of shape {self.params.shape}")
        _check(self.lib.dg_download(self.h, self._ptr(uin)))

    def compute_dt(self) -> float:
        dt = ctypes.c_double()
        _check(self.lib.dg_compute_dt(self.h, ctypes.byref(dt)))
        return dt.value

    def godunov(self, dt: float, time: float) -> None:
        _check(self.lib.dg_godunov(self.h, dt, time))

    def fargo_update(self, dt: float) -> None:
        _check(self.lib.dg_fargo_update(self.h, dt))

    def boundary(self, time: float, dt: float) -> None:
        _check(self.lib.dg_boundary(self.h, time, dt))

    def dissipation(self, time: float, dt: float) -> None:
        """Viscosity and resistivity after boundary (physics.f90:272-664); a no-op when nu = eta = 0."""
        _check(self.lib.dg_dissipation(self.h, time, dt))

    def run(self, nsteps: int, time: float) -> tuple[float, float]:
        t, dt = ctypes.c_double(time), ctypes.c_double(0.0)
        _check(self.lib.dg_run(self.h, nsteps, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def history(self, variant: str = "mri") -> np.ndarray:
        """The 9 history sums of the current state: variant "mri" (src/problem/mri/history.f90,
        dg_history) or "default" (src/subroutines/history.f90, the problems without their own
        history routine)."""
        out = np.zeros(9)
        if variant == "mri":
            _check(self.lib.dg_history(self.h, self._ptr(out)))
        else:
            _check(self.lib.dg_history_variant(self.h, HISTORY_VARIANTS[variant], self._ptr(out)))
        return out

    def sync(self) -> None:
        _check(self.lib.dg_sync(self.h))

    def dump(self, path: str | pathlib.Path, time: float, dt: float) -> None:
        """Write the state as a 'binary' dump (output.f90:224-235), streamed from the device."""
        _check(self.lib.dg_dump_write(self.h, str(path).encode(), time, dt))

    def restart(self, path: str | pathlib.Path) -> tuple[float, float]:
        """Load a 'binary' dump of this grid (restart.f90:212-221); returns (time, dt)."""
        t, dt = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.dg_dump_read(self.h, str(path).encode(), ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def debug_array(self, which: int, size: int) -> np.ndarray:
        """Copy a device work array of the last step (see dg_debug_copy)."""
        out = np.zeros(size)
        n = ctypes.c_longlong()
        _check(self.lib.dg_debug_copy(self.h, which, self._ptr(out), size, ctypes.byref(n)))
        return out[: n.value]

    def profile(self, on: bool = True) -> None:
        """Record CUDA events around every kernel of this context."""
        _check(self.lib.dg_profile(self.h, int(on)))

    def profile_read(self) -> dict[str, tuple[float, int]]:
        """{kernel slot: (total ms, launches)} since the last read."""
        n = 15
        ms = np.zeros(n)
        cnt = (ctypes.c_longlong * n)()
        _check(self.lib.dg_profile_read(self.h, self._ptr(ms), cnt, n))
        return {self.lib.dg_profile_slot_name(k).decode(): (float(ms[k]), int(cnt[k])) for k in range(n) if cnt[k]}

    # ---- z-slab decomposition (see dumses_hybrid_b200.slabs) ----
    @property
    def halo_count(self) -> int:
        """Doubles in one z halo of this context (3 planes of every stored state plane)."""
        return int(self.lib.dg_halo_count(self.h))

    def halo_pack(self, side: int, dev_ptr: int) -> None:
        """Copy the slab's 3 lowest (side 0) or highest (side 1) active planes to a device buffer."""
        _check(self.lib.dg_halo_pack(self.h, side, ctypes.c_void_p(dev_ptr)))

    def halo_unpack(self, side: int, dev_ptr: int) -> None:
        """Copy a neighbour's halo into the 3 ghost planes below (side 0) or above (side 1)."""
        _check(self.lib.dg_halo_unpack(self.h, side, ctypes.c_void_p(dev_ptr)))

    def history_columns(self) -> np.ndarray:
        """This slab's per-x-column sums of v_x and v_y, shape (nx, 2)."""
        col = np.zeros(2 * self.params.nx)
        _check(self.lib.dg_history_columns(self.h, self._ptr(col)))
        return col.reshape(self.params.nx, 2)

    def history_share(self, colmean: np.ndarray) -> np.ndarray:
        """This slab's share of the 9 history values, given the box's column means (nx, 2)."""
        cm = np.ascontiguousarray(colmean, dtype=np.float64).reshape(-1)
        out = np.zeros(9)
        _check(self.lib.dg_history_share(self.h, self._ptr(cm), self._ptr(out)))
        return out

    @property
    def stream(self) -> int:
        return int(self.lib.dg_stream(self.h) or 0)

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.dg_kernel_launches(self.h))

    def attach_surrogate(self, net: "FluxNet | None") -> None:
        """Use `net` for the faces of this FP32 context (made with surrogate=True); None detaches."""
        _check(self.lib.dg_attach_surrogate(self.h, net.h if net is not None else None))

    def surrogate_stats(self) -> tuple[int, int]:
        """(faces seen by the network, faces that fell back to HLLD) since the last call."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        _check(self.lib.dg_surrogate_stats(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value


N_IN, N_OUT = 17, 8


def network_shape(lib=None) -> tuple[int, int]:
    """(hidden width, hidden layers) of the network the library was built with."""
    lib = lib or load_library()
    w, d = ctypes.c_int(), ctypes.c_int()
    _check(lib.dg_nn_shape(ctypes.byref(w), ctypes.byref(d)))
    return w.value, d.value


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class FluxNet:
    """The learned face-flux network (a dg_nn of the C-ABI): 17 inputs, `depth` hidden layers
    of `width` SmeLU units (the library's build fixes them; 64 x 2 by default), 8 outputs,
    BF16 weights with FP32 accumulation, trained on the device.  Parameters are a flat
    float32 vector in the order W1[17][width], b1, the hidden W[width][width], b pairs,
    then W[width][8], b; `shapes` lists the (inputs, outputs) of each weight layer."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.lib = load_library()
        h = ctypes.c_void_p()
        _check(self.lib.dg_nn_create(device, seed, ctypes.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.dg_nn_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def param_count(self) -> int:
        return int(self.lib.dg_nn_param_count())

    @property
    def shape(self) -> tuple[int, int]:
        """(hidden width, hidden layers) of the library's network."""
        return network_shape(self.lib)

    @property
    def shapes(self) -> list[tuple[int, int]]:
        w, d = self.shape
        return [(N_IN, w)] + [(w, w)] * (d - 1) + [(w, N_OUT)]

    def params(self) -> np.ndarray:
        p = np.zeros(self.param_count, dtype=np.float32)
        _check(self.lib.dg_nn_get_params(self.h, _fptr(p), p.size))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.lib.dg_nn_set_params(self.h, _fptr(p), p.size))

    def set_samples(self, x: np.ndarray, t: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        _check(self.lib.dg_nn_set_samples(self.h, _fptr(x), _fptr(t), x.shape[0]))

    @property
    def sample_count(self) -> int:
        return int(self.lib.dg_nn_sample_count(self.h))

    def samples(self, first: int = 0, count: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        n = self.sample_count - first if count is None else count
        x = np.zeros((n, N_IN), dtype=np.float32)
        t = np.zeros((n, N_OUT), dtype=np.float32)
        _check(self.lib.dg_nn_samples_copy(self.h, first, n, _fptr(x), _fptr(t)))
        return x, t

    def harvest(self, ctx: Context, stride: int = 1) -> int:
        """Append the interfaces of an FP32 context's current state, with HLLD labels."""
        n = ctypes.c_longlong()
        _check(self.lib.dg_nn_harvest(ctx.h, self.h, stride, ctypes.byref(n)))
        return n.value

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3) -> float:
        loss = ctypes.c_float()
        _check(self.lib.dg_nn_train(self.h, steps, batch, lr, ctypes.byref(loss)))
        return loss.value

    def gradients(self, x: np.ndarray, t: np.ndarray) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.param_count, dtype=np.float32)
        loss = ctypes.c_float()
        _check(self.lib.dg_nn_gradients(self.h, _fptr(x), _fptr(t), x.shape[0], ctypes.byref(loss), _fptr(g)))
        return loss.value, g

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], N_OUT), dtype=np.float32)
        _check(self.lib.dg_nn_forward(self.h, _fptr(x), x.shape[0], _fptr(y)))
        return y

    def fit_envelope(self, margin: float = 0.0) -> None:
        _check(self.lib.dg_nn_fit_envelope(self.h, margin))

    def fit_scaling(self) -> None:
        """Standardise inputs and outputs by the current samples (call before training)."""
        _check(self.lib.dg_nn_fit_scaling(self.h))

    def set_gates(self, jump: float = 0.1, compress: float = 0.1) -> None:
        _check(self.lib.dg_nn_set_gates(self.h, jump, compress))
