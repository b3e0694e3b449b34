"""itlbm_case_diag_drop_static: the drop diagnostic on the library's fixed device scratch.

It runs the kernels of itlbm_case_diag_drop, so both calls must give the same measures on the same
state (compared here with a relative tolerance of 1e-12 and an absolute floor of 1e-14, although the
reductions are deterministic and the results are expected to be identical).  The call allocates no
device memory, rejects cases larger than its scratch, and needs nothing zeroed between calls.
"""
import ctypes as C
import math

import pytest

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-12, 1e-14


def make_case(itlbm, nx, ny, tipo, chi=0.0, xi=0.0, A=0.1, tau=0.8, radius=None, v0=0.0, prec=0):
    op = itlbm.make_op(tipo, chi, xi)
    r = min(nx, ny) / 4.0 if radius is None else radius
    d = itlbm.desc(nx, ny, op, tau=tau, beta=0.8, A_fact=A, radius=r,
                   k_profile=2.0 * math.log(9.0) / 3.45, v0=v0, precision=prec)
    return itlbm.Case(d)


def assert_same(a, b):
    da, db = a.as_dict(), b.as_dict()
    for k, va in da.items():
        vb = db[k]
        if hasattr(va, "__len__"):
            for x, y in zip(va, vb):
                assert (math.isnan(x) and math.isnan(y)) or abs(x - y) <= ATOL + RTOL * abs(x), (k, x, y)
        elif isinstance(va, float):
            assert (math.isnan(va) and math.isnan(vb)) or abs(va - vb) <= ATOL + RTOL * abs(va), (k, va, vb)
        else:
            assert va == vb, (k, va, vb)


def free_bytes():
    rt = C.CDLL("libcudart.so.12")
    free, total = C.c_size_t(0), C.c_size_t(0)
    assert rt.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
    return free.value


@pytest.mark.parametrize("nx,ny,tipo,chi,xi,A,prec,v0", [
    (96, 96, 3, 0.5, 0.0, 0.225, 0, 0.0),      # class P, FP64
    (80, 72, 12, 0.0, 0.0, 0.1, 1, 0.05),      # class F (force kept), FP32, translating
    (4096, 64, 13, 0.0, 1.569988, 0.1, 1, 0.0),  # the largest side the scratch admits
])
def test_static_equals_allocating(gpu, nx, ny, tipo, chi, xi, A, prec, v0):
    c = make_case(gpu, nx, ny, tipo, chi, xi, A, radius=min(nx, ny) / 4.0, v0=v0, prec=prec)
    try:
        for step_to in (60, 137):  # two diagnostics in a row, with steps between them
            c.step(step_to - c.steps_done, keep_aux=True)
            k = c.steps_done - 1
            ref = c.diag_drop(k)
            s1 = c.diag_drop_static(k)
            s2 = c.diag_drop_static(k)  # again on the same state: nothing left over from s1
            assert_same(ref, s1)
            assert_same(s1, s2)
            assert s1.step == k
    finally:
        c.close()


def test_static_allocates_nothing(gpu):
    warm = make_case(gpu, 40, 40, 3, 0.5, A=0.225)
    c = make_case(gpu, 512, 512, 1, A=0.225, prec=1)  # exactly the node limit
    try:
        warm.step(3, keep_aux=True)
        warm.diag_drop_static(2)  # first call on the device: looks the scratch up
        c.step(5, keep_aux=True)
        gpu.lib().itlbm_case_sync(c._h)
        before = free_bytes()
        d = c.diag_drop_static(4)
        after = free_bytes()
        assert d.ok == 1
        # the allocating form would have taken 6 doubles a node (12.6 MB) for this case
        assert after == before, (before, after)
        assert_same(c.diag_drop(4), d)
    finally:
        c.close()
        warm.close()


@pytest.mark.parametrize("nx,ny", [(1024, 600), (8192, 16), (513, 512)])
def test_static_rejects_large_cases(gpu, nx, ny):
    c = make_case(gpu, nx, ny, 3, 0.5, A=0.225, radius=6.0, prec=1)
    try:
        c.step(2, keep_aux=True)
        out = gpu.DropDiag()
        rc = gpu.lib().itlbm_case_diag_drop_static(c._h, 1, nx / 2, ny / 2, C.byref(out), None)
        assert rc == -1  # ITLBM_E_ARG
        msg = gpu.lib().itlbm_last_error().decode()
        assert "static scratch" in msg and str(nx) in msg
        c.diag_drop(1)  # the allocating form still serves it (raises on an error code)
    finally:
        c.close()


def test_static_state_errors(gpu):
    c = make_case(gpu, 48, 48, 11, A=0.1)  # class F
    try:
        out = gpu.DropDiag()
        assert gpu.lib().itlbm_case_diag_drop_static(c._h, 0, 24.0, 24.0, C.byref(out), None) == -10
        c.step(3)  # aux not kept: a class-F diagnostic cannot run
        assert gpu.lib().itlbm_case_diag_drop_static(c._h, 2, 24.0, 24.0, C.byref(out), None) == -10
        assert gpu.lib().itlbm_case_diag_drop_static(None, 2, 24.0, 24.0, C.byref(out), None) == -1
    finally:
        c.close()
