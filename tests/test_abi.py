"""The C ABI library loads and exports every entry point of include/itlbm.h (no GPU needed)."""
import ctypes
import re
import subprocess

import pytest


def test_library_exports_header(itlbm):
    lib = itlbm.lib()
    declared = itlbm.header_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, f"declared in include/itlbm.h but not exported: {missing}"


def test_exports_are_c_symbols(itlbm):
    out = subprocess.run(["nm", "-D", "--defined-only", str(itlbm.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(itlbm_[a-z0-9_]+)$", out, flags=re.M))
    assert set(itlbm.header_symbols()) <= exported


def test_struct_layouts_match_header(itlbm):
    # sizes of the ABI structures as compiled into the library (ctypes mirrors them)
    assert ctypes.sizeof(itlbm.Operador) == 40
    assert ctypes.sizeof(itlbm.CaseDesc) % 8 == 0
    names = [f for f, _ in itlbm.DROP_DIAG_FIELDS]
    assert len(names) == len(set(names))


@pytest.mark.parametrize("text,tipo,chi,xi,nome", [
    ("P1", 1, 0.5, 1.569988, "P1"),
    ("P3 0.5", 3, 0.5, 1.569988, "P3"),
    ("P3 -0.4\n", 3, -0.4, 1.569988, "P3"),
    ("P3", 3, 0.5, 1.569988, "P3"),
    ("P3\n2", 3, 2.0, 1.569988, "P3"),
    ("F1", 11, 0.5, 1.569988, "F1"),
    ("F2  ", 12, 0.5, 1.569988, "F2"),
    ("F3 1.569988", 13, 0.5, 1.569988, "F3"),
    ("F3 3", 13, 0.5, 3.0, "F3"),
    ("F3 abc", 13, 0.5, 1.569988, "F3"),
])
def test_le_operador(itlbm, text, tipo, chi, xi, nome):
    """itlbm_operador_parse follows le_operador (Operadores_tensao.cpp:66-86)."""
    op = itlbm.le_operador(text)
    assert (op.tipo, op.chi, op.xi, op.nome.decode()) == (tipo, chi, xi, nome)


@pytest.mark.parametrize("text", ["", "   \n", "P2", "p3 0.5", "F4", "X"])
def test_le_operador_rejects(itlbm, text):
    with pytest.raises(itlbm.ItlbmError) as e:
        itlbm.le_operador(text)
    assert e.value.code == -8


def test_operador_read_missing_file(itlbm, tmp_path):
    op = itlbm.Operador()
    rc = itlbm.lib().itlbm_operador_read(str(tmp_path / "nope.txt").encode(), ctypes.byref(op))
    assert rc == -9


def test_strerror_and_version(itlbm):
    L = itlbm.lib()
    assert L.itlbm_version().startswith(b"itlbm")
    assert L.itlbm_strerror(-2) == b"out of memory"
    assert L.itlbm_strerror(0) == b"ok"
