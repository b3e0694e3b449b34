"""ctypes binding of libitlbm (include/itlbm.h) for tests, the benchmark and scripting.

The product is the C ABI in libitlbm.so (CUDA kernels for sm_100a plus their C++ host side) and the
host programs in bin/.  This module only mirrors the ABI in Python: the structures of itlbm.h, the
operator parser with le_operador's behaviour (Operadores_tensao.cpp:66-86), and a `Case` object that
owns one simulation case.  There is no CPU fallback: every call goes to the library, and loading
fails loudly when libitlbm.so has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libitlbm.so"
BIN_DIR = PKG_DIR / "bin"

NVEL = 19
N_ANG = 256

# operator codes (OP_P1..OP_F3, Operadores_tensao.cpp:45-49)
OP_P1, OP_P3, OP_F1, OP_F2, OP_F3 = 1, 3, 11, 12, 13
GEOM_DROP, GEOM_STRIP = 0, 1
PREC_F64, PREC_F32, PREC_F32_FOLD = 0, 1, 2
FIELDS_VTK, FIELDS_PROFILE = 0, 1
STEP_KEEP_AUX = 1

ERRORS = {
    0: "ok", -1: "invalid argument", -2: "out of memory", -3: "CUDA error", -4: "no CUDA device",
    -5: "non-finite state", -6: "admission refused", -7: "wait timed out", -8: "parse error",
    -9: "I/O error", -10: "invalid state",
}


class Operador(C.Structure):
    _fields_ = [("tipo", C.c_int), ("chi", C.c_double), ("xi", C.c_double), ("nome", C.c_char * 16)]

    def __repr__(self):
        return f"Operador({self.nome.decode()}, tipo={self.tipo}, chi={self.chi}, xi={self.xi})"


class CaseDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("op", Operador), ("tau", C.c_double),
        ("beta", C.c_double), ("A_fact", C.c_double), ("rho_R", C.c_double), ("rho_B", C.c_double),
        ("geometry", C.c_int), ("radius", C.c_double), ("k_profile", C.c_double), ("v0", C.c_double),
        ("p", C.c_int), ("q", C.c_int), ("precision", C.c_int),
    ]


_D = C.c_double
DROP_DIAG_FIELDS = [
    ("ok", C.c_int), ("step", C.c_int),
    ("x0", _D), ("y0", _D), ("area", _D), ("raio", _D), ("raio_grad", _D), ("raio_linha", _D),
    ("massa_R", _D), ("massa_B", _D), ("qx", _D), ("qy", _D), ("qz", _D), ("u_max", _D), ("u_rms", _D),
    ("p_in", _D), ("p_out", _D), ("sd_in", _D), ("sd_out", _D), ("delta_p", _D), ("sigma", _D),
    ("p_centro", _D), ("p_canto", _D), ("sigma_linha", _D),
    ("K_perfil", _D), ("r_perfil", _D), ("res_perfil", _D), ("esp_perfil", _D),
    ("n_perfil", C.c_int), ("n_in", C.c_int), ("n_out", C.c_int), ("n_fluid", C.c_int), ("n_ruim", C.c_int),
    ("mean_x", _D), ("mean_y", _D), ("mean_z", _D), ("drop_x", _D), ("drop_y", _D),
    ("max_ref", _D), ("rms_ref", _D), ("max_mean", _D), ("rms_mean", _D), ("max_lab", _D), ("rms_lab", _D),
    ("min_f", _D), ("min_rho", _D), ("min_phi", _D), ("max_phi", _D), ("axis_ratio", _D),
    ("center_dx", _D), ("center_dy", _D), ("x_unwrapped", _D),
    ("negative_total", C.c_longlong), ("negative_color", C.c_longlong), ("bad", C.c_int),
    ("R0", _D), ("a2", _D), ("a4", _D), ("a8", _D), ("rmin", _D), ("rmax", _D),
]
STRIP_DIAG_FIELDS = [
    ("ok", C.c_int), ("step", C.c_int),
    ("sigma_pop", _D), ("int_grad", _D), ("K", _D), ("res", _D), ("d0", _D),
    ("u_max", _D), ("u_rms", _D), ("un_max", _D), ("ut_max", _D),
    ("massa_R", _D), ("massa_B", _D), ("qx", _D), ("qy", _D), ("min_f", _D), ("SFx", _D), ("SFy", _D),
    ("neg_total", C.c_longlong), ("neg_cor", C.c_longlong), ("n_ruim", C.c_int), ("n_ajuste", C.c_int),
]


class DropDiag(C.Structure):
    _fields_ = DROP_DIAG_FIELDS

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StripDiag(C.Structure):
    _fields_ = STRIP_DIAG_FIELDS

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SnapHeader(C.Structure):
    """Header of a case snapshot (itlbm_case_save / itlbm_batch_save)."""
    _fields_ = [("magic", C.c_char * 8), ("version", C.c_int), ("desc", CaseDesc), ("steps", C.c_longlong)]


class BatchConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_cases", C.c_int), ("chunk", C.c_int),
                ("diag_every", C.c_int), ("ctas_per_sm", C.c_int)]


EV_DIAG, EV_DONE, EV_UNSTABLE = 0, 1, 2


class BatchEvent(C.Structure):
    _fields_ = [("tag", C.c_longlong), ("kind", C.c_int), ("geometry", C.c_int), ("step", C.c_int),
                ("t_submit", C.c_double), ("t_event", C.c_double), ("drop", DropDiag), ("strip", StripDiag)]


class BatchStats(C.Structure):
    _fields_ = [("active", C.c_int), ("pending", C.c_int), ("finished", C.c_int),
                ("node_updates", C.c_longlong), ("device_ms", C.c_double), ("hbm_used", C.c_size_t),
                ("replays", C.c_int), ("captures", C.c_int), ("diag_ms", C.c_double),
                ("advance_ms", C.c_double), ("admit_ms", C.c_double), ("capture_ms", C.c_double),
                ("launch_mode", C.c_int), ("held", C.c_int), ("narrow_edges", C.c_int)]


class ItlbmError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({code})")
        self.code = code


_lib = None


def lib():
    """Load libitlbm.so (raises when it has not been built: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
    L = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    vp, dp, ip = C.c_void_p, P(C.c_double), P(C.c_int)
    sig = {
        "itlbm_version": (C.c_char_p, []),
        "itlbm_strerror": (C.c_char_p, [C.c_int]),
        "itlbm_last_error": (C.c_char_p, []),
        "itlbm_device_count": (C.c_int, [ip]),
        "itlbm_operador_parse": (C.c_int, [C.c_char_p, P(Operador)]),
        "itlbm_operador_read": (C.c_int, [C.c_char_p, P(Operador)]),
        "itlbm_case_create": (C.c_int, [P(CaseDesc), P(vp)]),
        "itlbm_case_destroy": (None, [vp]),
        "itlbm_case_step": (C.c_int, [vp, C.c_int, C.c_int, vp]),
        "itlbm_case_sync": (C.c_int, [vp]),
        "itlbm_case_steps_done": (C.c_longlong, [vp]),
        "itlbm_case_diag_drop": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, P(DropDiag), vp]),
        "itlbm_case_diag_drop_static": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, P(DropDiag), vp]),
        "itlbm_case_diag_strip": (C.c_int, [vp, C.c_int, P(StripDiag), vp]),
        "itlbm_case_read_pops": (C.c_int, [vp, C.c_int, dp, dp]),
        "itlbm_case_write_pops": (C.c_int, [vp, dp, dp]),
        "itlbm_case_read_fields": (C.c_int, [vp, dp, dp, dp, dp, dp, dp]),
        "itlbm_case_read_profile": (C.c_int, [vp, dp, dp, dp, dp]),
        "itlbm_case_save": (C.c_int, [vp, C.c_char_p]),
        "itlbm_case_load": (C.c_int, [C.c_char_p, P(vp)]),
        "itlbm_snapshot_info": (C.c_int, [C.c_char_p, P(CaseDesc), P(C.c_longlong)]),
        "itlbm_batch_save": (C.c_int, [vp, C.c_longlong, C.c_char_p]),
        "itlbm_batch_submit_saved": (C.c_int, [vp, C.c_char_p, C.c_int, C.c_longlong]),
        "itlbm_batch_create": (C.c_int, [P(BatchConfig), P(vp)]),
        "itlbm_batch_destroy": (None, [vp]),
        "itlbm_batch_submit": (C.c_int, [vp, P(CaseDesc), C.c_int, C.c_longlong]),
        "itlbm_batch_advance": (C.c_int, [vp, vp]),
        "itlbm_batch_poll": (C.c_int, [vp, P(BatchEvent), C.c_int]),
        "itlbm_batch_stats_get": (C.c_int, [vp, P(BatchStats)]),
        "itlbm_batch_hold_finished": (C.c_int, [vp, C.c_int]),
        "itlbm_batch_read_fields": (C.c_int, [vp, C.c_longlong, C.c_int, dp, dp, dp, dp, dp]),
        "itlbm_batch_release": (C.c_int, [vp, C.c_longlong]),
        "itlbm_dev_perturbacao": (C.c_int, [P(Operador), C.c_double, C.c_int, dp, dp]),
        "itlbm_dev_source": (C.c_int, [C.c_int, dp, dp, dp, C.c_double, dp]),
        "itlbm_dev_calcula_forca": (C.c_int, [P(Operador), C.c_double, C.c_int, C.c_int, dp, dp, dp]),
        "itlbm_dev_colisao_comum": (C.c_int, [P(Operador), C.c_double, C.c_double, C.c_double,
                                              C.c_int, dp, dp, dp, dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code, what):
    if code != 0:
        msg = lib().itlbm_last_error().decode(errors="replace")
        raise ItlbmError(code, f"{what} [{msg}]")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def le_operador(text: str) -> Operador:
    """Parse one operador.txt line the way le_operador does (Operadores_tensao.cpp:66-86)."""
    op = Operador()
    check(lib().itlbm_operador_parse(text.encode(), C.byref(op)), "operador")
    return op


def make_op(tipo, chi=0.5, xi=1.569988, nome=None):
    op = Operador()
    op.tipo, op.chi, op.xi = tipo, chi, xi
    names = {OP_P1: "P1", OP_P3: "P3", OP_F1: "F1", OP_F2: "F2", OP_F3: "F3"}
    op.nome = (nome or names[tipo]).encode()
    return op


def desc(nx, ny, op, tau=1.0, beta=0.8, A_fact=0.225, rho_R=1.0, rho_B=1.0, geometry=GEOM_DROP,
         radius=0.0, k_profile=2.0 * np.log(9.0) / 3.45, v0=0.0, p=1, q=0, precision=PREC_F64):
    d = CaseDesc()
    d.nx, d.ny, d.op, d.tau, d.beta, d.A_fact = nx, ny, op, tau, beta, A_fact
    d.rho_R, d.rho_B, d.geometry, d.radius, d.k_profile = rho_R, rho_B, geometry, radius, k_profile
    d.v0, d.p, d.q, d.precision = v0, p, q, precision
    return d


class Case:
    """One case on the current device (itlbm_case_* of include/itlbm.h)."""

    def __init__(self, d: CaseDesc):
        self.desc = d
        self.n = d.nx * d.ny
        h = C.c_void_p()
        check(lib().itlbm_case_create(C.byref(d), C.byref(h)), "itlbm_case_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().itlbm_case_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def step(self, nsteps=1, keep_aux=False, stream=None):
        check(lib().itlbm_case_step(self._h, nsteps, STEP_KEEP_AUX if keep_aux else 0, stream),
              "itlbm_case_step")

    def sync(self):
        check(lib().itlbm_case_sync(self._h), "itlbm_case_sync")

    @property
    def steps_done(self):
        return lib().itlbm_case_steps_done(self._h)

    def diag_drop(self, step, x_ini=None, y_ini=None, stream=None) -> DropDiag:
        out = DropDiag()
        x_ini = self.desc.nx // 2 if x_ini is None else x_ini
        y_ini = self.desc.ny // 2 if y_ini is None else y_ini
        check(lib().itlbm_case_diag_drop(self._h, step, float(x_ini), float(y_ini), C.byref(out), stream),
              "itlbm_case_diag_drop")
        return out

    def save(self, path):
        check(lib().itlbm_case_save(self._h, str(path).encode()), "itlbm_case_save")

    @classmethod
    def load(cls, path):
        """A case restored from a snapshot written by save() (or by Batch.save)."""
        hd = SnapHeader()
        with open(path, "rb") as f:
            C.memmove(C.byref(hd), f.read(C.sizeof(SnapHeader)), C.sizeof(SnapHeader))
        h = C.c_void_p()
        check(lib().itlbm_case_load(str(path).encode(), C.byref(h)), "itlbm_case_load")
        c = cls.__new__(cls)
        c.desc = hd.desc
        c.n = hd.desc.nx * hd.desc.ny
        c._h = h
        return c

    def diag_drop_static(self, step, x_ini=None, y_ini=None, stream=None) -> DropDiag:
        """diag_drop on the library's fixed device scratch (no allocation; cases of at most
        512 x 512 nodes; concurrent calls on one device race)."""
        out = DropDiag()
        x_ini = self.desc.nx // 2 if x_ini is None else x_ini
        y_ini = self.desc.ny // 2 if y_ini is None else y_ini
        check(lib().itlbm_case_diag_drop_static(self._h, step, float(x_ini), float(y_ini), C.byref(out),
                                                stream), "itlbm_case_diag_drop_static")
        return out

    def diag_strip(self, step, stream=None) -> StripDiag:
        out = StripDiag()
        check(lib().itlbm_case_diag_strip(self._h, step, C.byref(out), stream), "itlbm_case_diag_strip")
        return out

    def read_pops(self, which=0):
        fR = np.empty(self.n * NVEL)
        fB = np.empty(self.n * NVEL)
        check(lib().itlbm_case_read_pops(self._h, which, _dp(fR), _dp(fB)), "itlbm_case_read_pops")
        return fR, fB

    def write_pops(self, fR, fB):
        fR = np.ascontiguousarray(fR, dtype=np.float64)
        fB = np.ascontiguousarray(fB, dtype=np.float64)
        check(lib().itlbm_case_write_pops(self._h, _dp(fR), _dp(fB)), "itlbm_case_write_pops")

    def read_fields(self, force=False):
        n = self.n
        out = {k: np.empty(n) for k in ("rho_R", "rho_B", "ux", "uy", "uz")}
        F = np.empty(3 * n) if force else None
        check(lib().itlbm_case_read_fields(self._h, *[_dp(out[k]) for k in ("rho_R", "rho_B", "ux", "uy", "uz")],
                                           _dp(F) if force else None), "itlbm_case_read_fields")
        if force:
            out["force"] = F
        return out

    def read_profile(self):
        """The per-node values of perfil.dat (rho_R, rho_B and the mixture velocity ux, uy)."""
        n = self.n
        out = {k: np.empty(n) for k in ("rho_R", "rho_B", "ux", "uy")}
        check(lib().itlbm_case_read_profile(self._h, *[_dp(out[k]) for k in ("rho_R", "rho_B", "ux", "uy")]),
              "itlbm_case_read_profile")
        return out


class Batch:
    """Many cases stepped together (itlbm_batch_* of include/itlbm.h)."""

    def __init__(self, hbm_budget=0, max_cases=0, chunk=0, diag_every=0, ctas_per_sm=0):
        cfg = BatchConfig(hbm_budget, max_cases, chunk, diag_every, ctas_per_sm)
        h = C.c_void_p()
        check(lib().itlbm_batch_create(C.byref(cfg), C.byref(h)), "itlbm_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().itlbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, d: CaseDesc, n_steps: int, tag: int):
        check(lib().itlbm_batch_submit(self._h, C.byref(d), n_steps, tag), "itlbm_batch_submit")

    def save(self, tag, path):
        check(lib().itlbm_batch_save(self._h, tag, str(path).encode()), "itlbm_batch_save")

    def submit_saved(self, path, n_steps, tag):
        check(lib().itlbm_batch_submit_saved(self._h, str(path).encode(), n_steps, tag), "itlbm_batch_submit_saved")

    def advance(self):
        r = lib().itlbm_batch_advance(self._h, None)
        if r < 0:
            check(r, "itlbm_batch_advance")
        return r

    def poll(self, max_events=4096):
        buf = (BatchEvent * max_events)()
        n = lib().itlbm_batch_poll(self._h, buf, max_events)
        if n < 0:
            check(n, "itlbm_batch_poll")
        return [buf[i] for i in range(n)]

    def hold_finished(self, on=True):
        check(lib().itlbm_batch_hold_finished(self._h, 1 if on else 0), "itlbm_batch_hold_finished")

    def read_fields(self, tag, n, form=FIELDS_VTK):
        """Fields of an active case after a diagnostic step, or of a held finished case (n nodes)."""
        out = {k: np.empty(n) for k in ("rho_R", "rho_B", "ux", "uy", "uz")}
        check(lib().itlbm_batch_read_fields(self._h, tag, form, *[_dp(out[k]) for k in ("rho_R", "rho_B", "ux", "uy",
                                                                                        "uz")]),
              "itlbm_batch_read_fields")
        return out

    def release(self, tag):
        check(lib().itlbm_batch_release(self._h, tag), "itlbm_batch_release")

    def stats(self) -> BatchStats:
        st = BatchStats()
        check(lib().itlbm_batch_stats_get(self._h, C.byref(st)), "itlbm_batch_stats_get")
        return st


def dev_perturbacao(op, A, g, f):
    g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1, 3)
    f = np.array(f, dtype=np.float64).reshape(-1, NVEL)
    check(lib().itlbm_dev_perturbacao(C.byref(op), A, g.shape[0], _dp(g), _dp(f)), "itlbm_dev_perturbacao")
    return f


def dev_source(F, u, rho, tau):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1, 3)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
    rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
    S = np.empty((F.shape[0], NVEL))
    check(lib().itlbm_dev_source(F.shape[0], _dp(F), _dp(u), _dp(rho), tau, _dp(S)), "itlbm_dev_source")
    return S


def dev_calcula_forca(op, sigma, nx, ny, fR, fB):
    fR = np.ascontiguousarray(fR, dtype=np.float64)
    fB = np.ascontiguousarray(fB, dtype=np.float64)
    F = np.empty(3 * nx * ny)
    check(lib().itlbm_dev_calcula_forca(C.byref(op), sigma, nx, ny, _dp(fR), _dp(fB), _dp(F)),
          "itlbm_dev_calcula_forca")
    return F


def dev_colisao_comum(op, tau, A_fact, beta, fR, fB, gm, F=None):
    fR = np.array(fR, dtype=np.float64).reshape(-1, NVEL)
    fB = np.array(fB, dtype=np.float64).reshape(-1, NVEL)
    gm = np.ascontiguousarray(gm, dtype=np.float64).reshape(-1, 3)
    Fp = None
    if F is not None:
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1, 3)
        Fp = _dp(F)
    check(lib().itlbm_dev_colisao_comum(C.byref(op), tau, A_fact, beta, fR.shape[0], _dp(fR), _dp(fB),
                                        _dp(gm), Fp), "itlbm_dev_colisao_comum")
    return fR, fB


def header_symbols(header=PKG_DIR.parent / "include" / "itlbm.h"):
    """Names of the functions declared in include/itlbm.h."""
    import re
    text = Path(header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(itlbm_[a-z0-9_]+)\s*\(", text)))
