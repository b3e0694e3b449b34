"""The FP32 step runs as a marching kernel (strips of 32 columns walked in slabs of 4 rows, rows
copied into shared memory by TMA).  It evaluates every node with the arithmetic of the FP32 tile
kernel, in the same order, so the two must agree BIT FOR BIT: populations at the top of each step,
post-collision populations, the kept force and the diagnostics.  The cases cover partial strips and
segments (nx not a multiple of 32, ny not a multiple of 4 or of the 64-row segment), boxes smaller
than a strip, several segments, both halo widths (1 for P1, P3, F3; 2 for F1, F2) and both
geometries."""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPS = [("P1", 1, 0.5, 1.569988, 0.225), ("P3", 3, 0.5, 1.569988, 0.225), ("F1", 11, 0.5, 1.569988, 0.1),
       ("F2", 12, 0.5, 1.569988, 0.1), ("F3", 13, 0.5, 1.569988, 0.1)]


def make(itlbm, kernel, nx, ny, tipo, chi, xi, A, geometry=0, p=1, q=0, v0=0.0, tau=0.8):
    os.environ["ITLBM_STEP_KERNEL"] = kernel
    try:
        op = itlbm.make_op(tipo, chi, xi)
        d = itlbm.desc(nx, ny, op, tau=tau, A_fact=A, radius=min(nx, ny) / 4.0,
                       k_profile=2.0 * math.log(9.0) / 3.45, v0=v0, geometry=geometry, p=p, q=q,
                       precision=itlbm.PREC_F32)
        return itlbm.Case(d)
    finally:
        os.environ.pop("ITLBM_STEP_KERNEL", None)


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("name,tipo,chi,xi,A", OPS, ids=[o[0] for o in OPS])
@pytest.mark.parametrize("nx,ny,v0", [
    (37, 29, 0.05),    # partial strip, ny % 4 = 1, translating
    (7, 5, 0.0),       # smaller than a strip: every halo column wraps
    (64, 64, 0.0),     # exactly two strips and one segment
    (100, 131, 0.02),  # three segments, the last one partial (3 rows)
    (33, 3, 0.0),      # fewer rows than a slab
])
def test_march_equals_tiles(gpu, name, tipo, chi, xi, A, nx, ny, v0):
    ct = make(gpu, "tile", nx, ny, tipo, chi, xi, A, v0=v0)
    cm = make(gpu, "march", nx, ny, tipo, chi, xi, A, v0=v0)
    try:
        assert same(ct.read_pops(0), cm.read_pops(0))
        for c in (ct, cm):
            c.step(1)
        assert same(ct.read_pops(0), cm.read_pops(0)), "after 1 step"
        for c in (ct, cm):
            c.step(38)
            c.step(1, keep_aux=True)
        assert same(ct.read_pops(0), cm.read_pops(0)), "after 40 steps"
        assert same(ct.read_pops(1), cm.read_pops(1)), "post-collision"
        ft, fm = ct.read_fields(force=True), cm.read_fields(force=True)
        for k in ft:
            assert np.array_equal(ft[k], fm[k]), k
        dt, dm = ct.diag_drop(39).as_dict(), cm.diag_drop(39).as_dict()
        for k, v in dt.items():
            assert v == dm[k] or (v != v and dm[k] != dm[k]), k
    finally:
        ct.close()
        cm.close()


@pytest.mark.parametrize("name,tipo,chi,xi,A", OPS, ids=[o[0] for o in OPS])
@pytest.mark.parametrize("N,p,q", [(48, 2, 1), (70, 1, 1)])
def test_march_equals_tiles_strip(gpu, name, tipo, chi, xi, A, N, p, q):
    ct = make(gpu, "tile", N, N, tipo, chi, xi, A, geometry=1, p=p, q=q)
    cm = make(gpu, "march", N, N, tipo, chi, xi, A, geometry=1, p=p, q=q)
    try:
        for c in (ct, cm):
            c.step(29)
            c.step(1, keep_aux=True)
        assert same(ct.read_pops(0), cm.read_pops(0))
        st, sm = ct.diag_strip(29).as_dict(), cm.diag_strip(29).as_dict()
        for k, v in st.items():
            assert v == sm[k] or (v != v and sm[k] != sm[k]), k
    finally:
        ct.close()
        cm.close()


def test_march_large_case_conserves(gpu):
    """A 1000 x 700 drop (32 strips, 11 segments) for 200 steps: both kernels agree bit for bit."""
    ct = make(gpu, "tile", 1000, 700, 3, 0.5, 1.569988, 0.225)
    cm = make(gpu, "march", 1000, 700, 3, 0.5, 1.569988, 0.225)
    try:
        for c in (ct, cm):
            c.step(200)
        assert same(ct.read_pops(0), cm.read_pops(0))
    finally:
        ct.close()
        cm.close()
