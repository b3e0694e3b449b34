"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the checker of the
CUDA path.  Wraps
  * liboracle.so  -- the C restatement of the reference path (itlbm_oracle.c), and
  * _ref/libref_ops.so, _ref/libref_incl.so -- the reference itself, compiled from its sources by
    `make -C oracle ref` (present where that recipe ran; it travels with the repository snapshot).
The diagnostic structures are the ones of include/itlbm.h, taken from the package binding.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import sys
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REPO = ORACLE_DIR.parent
PKG_DIR = REPO / "interfacial-tension-operators-lbm_b200"
NVEL = 19


def load_package():
    """Import the package binding (a directory whose name is not an identifier) as `itlbm_b200`."""
    if "itlbm_b200" in sys.modules:
        return sys.modules["itlbm_b200"]
    spec = importlib.util.spec_from_file_location("itlbm_b200", PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["itlbm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_pkg = load_package()
DropDiag, StripDiag = _pkg.DropDiag, _pkg.StripDiag

_P = C.POINTER
_dp = _P(C.c_double)
_orc = None


def _ptr(a):
    return a.ctypes.data_as(_dp)


def orc():
    global _orc
    if _orc is None:
        path = ORACLE_DIR / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C {ORACLE_DIR}`")
        L = C.CDLL(str(path))
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        sig = {
            "orc_create": (vp, [i, i, i, d, d, d, d, d]),
            "orc_destroy": (None, [vp]),
            "orc_init_drop": (None, [vp, d, d, d, d, d]),
            "orc_init_strip": (None, [vp, i, i]),
            "orc_set_pops": (None, [vp, _dp, _dp]),
            "orc_get_pops": (None, [vp, i, _dp, _dp]),
            "orc_get_force": (None, [vp, _dp]),
            "orc_get_gm": (None, [vp, _dp]),
            "orc_step": (None, [vp, i]),
            "orc_set_threads": (None, [i]),
            "orc_diag_drop": (i, [vp, i, d, d, d, _P(DropDiag)]),
            "orc_diag_strip": (i, [vp, i, i, i, _P(StripDiag)]),
            "orc_perturbacao": (None, [i, d, d, _dp, _dp]),
            "orc_source": (None, [_dp, _dp, d, d, _dp]),
            "orc_calcula_forca": (None, [i, d, d, i, i, _dp, _dp, _dp]),
            "orc_colisao_comum": (None, [i, d, d, d, d, _dp, _dp, _dp, _dp]),
            "orc_fields": (None, [vp, i, _dp, _dp, _dp, _dp, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _orc = L
    return _orc


def set_threads(n):
    orc().orc_set_threads(int(n))


K_PERFIL = 2.0 * np.log(9.0) / 3.45  # Imm_OPS.cpp:199 with ESPESSURA_INI = 3.45


class OracleCase:
    """The C restatement of one case (AoS populations, reference layout)."""

    def __init__(self, nx, ny, tipo, chi=0.5, xi=1.569988, tau=1.0, beta=0.8, A=0.225):
        self.nx, self.ny, self.n, self.tipo = nx, ny, nx * ny, tipo
        self._h = orc().orc_create(nx, ny, tipo, chi, xi, tau, beta, A)

    def init_drop(self, radius=0.0, k_perfil=K_PERFIL, v0=0.0, rho_R=1.0, rho_B=1.0):
        radius = radius if radius > 0 else 0.25 * self.nx
        orc().orc_init_drop(self._h, radius, k_perfil, v0, rho_R, rho_B)
        return self

    def init_strip(self, p, q):
        orc().orc_init_strip(self._h, p, q)
        return self

    def set_pops(self, fR, fB):
        fR = np.ascontiguousarray(fR, dtype=np.float64)
        fB = np.ascontiguousarray(fB, dtype=np.float64)
        orc().orc_set_pops(self._h, _ptr(fR), _ptr(fB))

    def pops(self, which=0):
        fR, fB = np.empty(self.n * NVEL), np.empty(self.n * NVEL)
        orc().orc_get_pops(self._h, which, _ptr(fR), _ptr(fB))
        return fR, fB

    def force(self):
        F = np.empty(3 * self.n)
        orc().orc_get_force(self._h, _ptr(F))
        return F

    def gm(self):
        g = np.empty(3 * self.n)
        orc().orc_get_gm(self._h, _ptr(g))
        return g

    def step(self, n=1):
        orc().orc_step(self._h, int(n))

    def fields(self, form=0):
        """rec_density / rec_velocity (form 0) or the perfil.dat columns (form 1) of the post-collision
        populations of the last step."""
        out = {k: np.empty(self.n) for k in ("rho_R", "rho_B", "ux", "uy", "uz")}
        orc().orc_fields(self._h, int(form), *[_ptr(out[k]) for k in ("rho_R", "rho_B", "ux", "uy", "uz")])
        return out

    def diag_drop(self, step, v0=0.0, x_ini=None, y_ini=None):
        d = DropDiag()
        x_ini = self.nx // 2 if x_ini is None else x_ini
        y_ini = self.ny // 2 if y_ini is None else y_ini
        orc().orc_diag_drop(self._h, step, v0, float(x_ini), float(y_ini), C.byref(d))
        return d

    def diag_strip(self, step, p, q):
        d = StripDiag()
        orc().orc_diag_strip(self._h, step, p, q, C.byref(d))
        return d

    def close(self):
        if self._h:
            orc().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def perturbacao(tipo, chi, A, g, f):
    f = np.array(f, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    orc().orc_perturbacao(tipo, chi, A, _ptr(g), _ptr(f))
    return f


def source(F, u, rho, tau):
    S = np.empty(NVEL)
    orc().orc_source(_ptr(np.ascontiguousarray(F, dtype=np.float64)),
                     _ptr(np.ascontiguousarray(u, dtype=np.float64)), rho, tau, _ptr(S))
    return S


def calcula_forca(tipo, xi, sigma, nx, ny, fR, fB):
    F = np.empty(3 * nx * ny)
    orc().orc_calcula_forca(tipo, xi, sigma, nx, ny, _ptr(np.ascontiguousarray(fR)),
                            _ptr(np.ascontiguousarray(fB)), _ptr(F))
    return F


# ---- the reference itself (oracle/_ref) -------------------------------------------------------
REF_DIR = ORACLE_DIR / "_ref"


def ref_available():
    return (REF_DIR / "libref_ops.so").exists() and (REF_DIR / "libref_incl.so").exists()


_ref_ops = _ref_incl = None


def _load_ref():
    global _ref_ops, _ref_incl
    if _ref_ops is None:
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        L = C.CDLL(str(REF_DIR / "libref_ops.so"))
        for name, res, args in [
            ("ref_ops_create", vp, [i, i, i, d, d, d, d, d, d, d, d, d, d, i]),
            ("ref_ops_set_pops", None, [vp, _dp, _dp]),
            ("ref_ops_step", None, [vp, i]),
            ("ref_ops_get_pops", None, [vp, i, _dp, _dp]),
            ("ref_ops_get_force", None, [vp, _dp]),
            ("ref_ops_diag", i, [vp, i, d, d, d, _P(DropDiag)]),
            ("ref_ops_write_fields", i, [vp, i, C.c_char_p]),
            ("ref_ops_destroy", None, [vp]),
        ]:
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _ref_ops = L
        L2 = C.CDLL(str(REF_DIR / "libref_incl.so"))
        for name, res, args in [
            ("ref_incl_create", vp, [i, i, d, d, d, d, d, i, i, i]),
            ("ref_incl_step", None, [vp, i]),
            ("ref_incl_get_pops", None, [vp, i, _dp, _dp]),
            ("ref_incl_diag", i, [vp, i, _P(StripDiag)]),
            ("ref_incl_write_perfil", i, [vp, C.c_char_p]),
            ("ref_incl_destroy", None, [vp]),
        ]:
            f = getattr(L2, name)
            f.restype, f.argtypes = res, args
        _ref_incl = L2
    return _ref_ops, _ref_incl


class RefDrop:
    """The reference's own Imm_OPS step, through oracle/_ref/libref_ops.so."""

    def __init__(self, nx, ny, tipo, chi=0.5, xi=1.569988, tau=1.0, beta=0.8, A=0.225, radius=0.0,
                 k_perfil=K_PERFIL, v0=0.0, rho_R=1.0, rho_B=1.0, threads=0):
        L, _ = _load_ref()
        self.nx, self.ny, self.n = nx, ny, nx * ny
        radius = radius if radius > 0 else 0.25 * nx
        self._h = L.ref_ops_create(nx, ny, tipo, chi, xi, tau, beta, A, radius, k_perfil, v0, rho_R,
                                   rho_B, threads)

    def step(self, n=1):
        _ref_ops.ref_ops_step(self._h, int(n))

    def set_pops(self, fR, fB):
        _ref_ops.ref_ops_set_pops(self._h, _ptr(np.ascontiguousarray(fR)), _ptr(np.ascontiguousarray(fB)))

    def pops(self, which=0):
        fR, fB = np.empty(self.n * NVEL), np.empty(self.n * NVEL)
        _ref_ops.ref_ops_get_pops(self._h, which, _ptr(fR), _ptr(fB))
        return fR, fB

    def force(self):
        F = np.empty(3 * self.n)
        _ref_ops.ref_ops_get_force(self._h, _ptr(F))
        return F

    def diag(self, step, v0=0.0, x_ini=None, y_ini=None):
        d = DropDiag()
        x_ini = self.nx // 2 if x_ini is None else x_ini
        y_ini = self.ny // 2 if y_ini is None else y_ini
        _ref_ops.ref_ops_diag(self._h, step, v0, float(x_ini), float(y_ini), C.byref(d))
        return d

    def write_fields(self, step, directory):
        """rho_R<step>.vtk, rho_B<step>.vtk and vel_<step>.vtk of the post-collision populations, written
        into `directory` by the reference's rec_density / rec_velocity."""
        if not _ref_ops.ref_ops_write_fields(self._h, int(step), str(directory).encode()):
            raise RuntimeError(f"cannot write the fields into {directory}")

    def close(self):
        if self._h:
            _ref_ops.ref_ops_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefStrip:
    """The reference's own Imm_INCL step, through oracle/_ref/libref_incl.so."""

    def __init__(self, N, tipo, p, q, chi=0.5, xi=1.569988, tau=1.0, beta=0.8, A=0.225, threads=0):
        _, L = _load_ref()
        self.N, self.n, self.p, self.q = N, N * N, p, q
        self._h = L.ref_incl_create(N, tipo, chi, xi, tau, beta, A, p, q, threads)

    def step(self, n=1):
        _ref_incl.ref_incl_step(self._h, int(n))

    def pops(self, which=0):
        fR, fB = np.empty(self.n * NVEL), np.empty(self.n * NVEL)
        _ref_incl.ref_incl_get_pops(self._h, which, _ptr(fR), _ptr(fB))
        return fR, fB

    def diag(self, step):
        d = StripDiag()
        _ref_incl.ref_incl_diag(self._h, step, C.byref(d))
        return d

    def write_perfil(self, directory):
        """perfil.dat of the post-collision populations, written into `directory` by mede_inclinada."""
        if not _ref_incl.ref_incl_write_perfil(self._h, str(directory).encode()):
            raise RuntimeError(f"cannot write perfil.dat into {directory}")

    def close(self):
        if self._h:
            _ref_incl.ref_incl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefStepper:
    """The reference's own step loop (Imm_OPS.cpp:252-287) on one drop case, through
    oracle/_ref/libref_ops_fast.so (built from the reference's sources with its own flags), run on
    `threads` host threads (0 = all cores).  A CPU baseline, never a product path."""

    def __init__(self, nx, ny, tipo=3, chi=0.5, xi=1.569988, tau=1.0, beta=0.8, A=0.225, radius=0.0,
                 threads=0):
        import os
        L = C.CDLL(str(REF_DIR / "libref_ops_fast.so"))
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        L.ref_ops_create.restype, L.ref_ops_create.argtypes = vp, [i, i, i, d, d, d, d, d, d, d, d, d, d, i]
        L.ref_ops_step.restype, L.ref_ops_step.argtypes = None, [vp, i]
        L.ref_ops_destroy.restype, L.ref_ops_destroy.argtypes = None, [vp]
        self._L = L
        self.threads = threads if threads > 0 else (os.cpu_count() or 1)
        self.nodes = nx * ny
        radius = radius if radius > 0 else 0.25 * nx
        self._h = L.ref_ops_create(nx, ny, tipo, chi, xi, tau, beta, A, radius, K_PERFIL, 0.0, 1.0, 1.0,
                                   self.threads)

    def step(self, n):
        """n steps; returns the wall time in seconds."""
        import time
        t0 = time.perf_counter()
        self._L.ref_ops_step(self._h, n)
        return time.perf_counter() - t0

    def close(self):
        if self._h:
            self._L.ref_ops_destroy(self._h)
            self._h = None


class RefStripStepper:
    """The reference's own Imm_INCL step loop (Imm_INCL.cpp:358-442) on one inclined-strip case, through
    oracle/_ref/libref_incl_fast.so (the reference's own flags), on `threads` host threads (0 = all
    cores).  A CPU baseline, never a product path."""

    def __init__(self, N, tipo=3, p=1, q=0, chi=0.5, xi=1.569988, tau=1.0, beta=0.8, A=0.225, threads=0):
        import os
        L = C.CDLL(str(REF_DIR / "libref_incl_fast.so"))
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        L.ref_incl_create.restype, L.ref_incl_create.argtypes = vp, [i, i, d, d, d, d, d, i, i, i]
        L.ref_incl_step.restype, L.ref_incl_step.argtypes = None, [vp, i]
        L.ref_incl_destroy.restype, L.ref_incl_destroy.argtypes = None, [vp]
        self._L = L
        self.threads = threads if threads > 0 else (os.cpu_count() or 1)
        self.nodes = N * N
        self._h = L.ref_incl_create(N, tipo, chi, xi, tau, beta, A, p, q, self.threads)

    def step(self, n):
        """n steps; returns the wall time in seconds."""
        import time
        t0 = time.perf_counter()
        self._L.ref_incl_step(self._h, n)
        return time.perf_counter() - t0

    def close(self):
        if self._h:
            self._L.ref_incl_destroy(self._h)
            self._h = None


def time_reference_step(nx, ny, tipo=3, chi=0.5, xi=1.569988, tau=1.0, beta=0.8, A=0.225, radius=0.0,
                        steps=10, warmup=1, threads=0):
    """Time the reference's own step loop on the host cores.  Returns (MLUPS, seconds, threads)."""
    r = RefStepper(nx, ny, tipo, chi, xi, tau, beta, A, radius, threads)
    if warmup:
        r.step(warmup)
    dt = r.step(steps)
    r.close()
    return nx * ny * steps / dt / 1e6, dt, r.threads
