"""The batched engine: every case gives the same bits alone and in a mixed batch (cases of
different sizes, operators, storage forms -- FP64, FP32, FP32 fold -- and geometries, admitted at
different times), its
diagnostics fall on the reference's steps (every 500 steps and the last), and the admission
budget is honoured."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mkdesc(itlbm, nx, tipo, chi=0.5, xi=1.569988, A=0.1, tau=0.8, prec=0, geometry=0, p=1, q=0, v0=0.0):
    op = itlbm.make_op(tipo, chi, xi)
    return itlbm.desc(nx, nx, op, tau=tau, A_fact=A, precision=prec, geometry=geometry, p=p, q=q, v0=v0)


MIX = [  # (nx, tipo, chi, A, prec, geometry, pq, steps)
    (48, 3, 0.5, 0.225, 0, 0, (1, 0), 1001),
    (37, 12, 0.5, 0.1, 1, 0, (1, 0), 777),
    (64, 11, 0.5, 0.1, 1, 1, (2, 1), 600),
    (33, 13, 0.5, 0.1, 0, 0, (1, 0), 1200),
    (80, 1, 0.5, 0.225, 1, 0, (1, 0), 501),
    (40, 3, 2.0, 0.225, 0, 1, (1, 1), 1),
    (45, 3, 0.5, 0.225, 2, 0, (1, 0), 650),   # the fold: a third work table, run as its own chain
    (56, 12, 0.5, 0.1, 2, 1, (1, 2), 900),
]


def run_alone(itlbm, d, steps):
    """Same schedule as the batch: diagnostics at multiples of 500 and at the last step."""
    rows = []
    with itlbm.Case(d) as c:
        s = 0
        while s < steps:
            nxt = min(((s + 499) // 500) * 500, steps - 1)
            c.step(nxt - s + 1, keep_aux=True)
            rows.append(c.diag_drop(nxt).as_dict() if d.geometry == 0 else c.diag_strip(nxt).as_dict())
            s = nxt + 1
        return rows, c.read_pops(0)


def test_batch_equals_alone(gpu):
    descs = [mkdesc(gpu, nx, t, chi, A=A, prec=pr, geometry=g, p=pq[0], q=pq[1]) for nx, t, chi, A, pr, g, pq, _ in MIX]
    alone = [run_alone(gpu, d, m[-1]) for d, m in zip(descs, MIX)]
    with gpu.Batch(chunk=200) as b:
        # half submitted now, half after the first round
        for k in range(0, len(MIX), 2):
            b.submit(descs[k], MIX[k][-1], k)
        b.advance()
        for k in range(1, len(MIX), 2):
            b.submit(descs[k], MIX[k][-1], k)
        events = []
        for _ in range(200):
            b.advance()
            events += b.poll()
            st = b.stats()
            if st.active == 0 and st.pending == 0:
                break
        assert st.finished == len(MIX)
    for k, (rows, _) in enumerate(alone):
        diag = [e for e in events if e.tag == k and e.kind == gpu.EV_DIAG]
        done = [e for e in events if e.tag == k and e.kind == gpu.EV_DONE]
        assert len(done) == 1 and done[0].step == MIX[k][-1]
        assert [e.step for e in diag] == [r["step"] for r in rows]
        for e, r in zip(diag, rows):
            got = (e.drop if MIX[k][5] == 0 else e.strip).as_dict()
            assert got == r, (k, {f: (got[f], r[f]) for f in r if got[f] != r[f]})


def test_admission_budget(gpu):
    d = mkdesc(gpu, 256, 3, A=0.225, prec=1)
    per_case = 2 * 2 * 19 * 256 * 256 * 4
    with gpu.Batch(hbm_budget=int(2.5 * per_case), chunk=100) as b:
        for k in range(5):
            b.submit(d, 150, k)
        b.advance()
        st = b.stats()
        assert st.active == 2 and st.pending == 3 and st.hbm_used <= 2.5 * per_case
        for _ in range(50):
            b.advance()
            st = b.stats()
            if st.finished == 5:
                break
        assert st.finished == 5 and st.hbm_used == 0
        with pytest.raises(gpu.ItlbmError) as e:
            b.submit(mkdesc(gpu, 1024, 3, prec=1), 10, 99)
        assert e.value.code == -6


def test_unstable_case_retires(gpu):
    """P3 chi = -0.4, tau = 0.51, sigma = 1 blows up at step 500 (stored batch E4): reported unstable
    there, the other case carries on."""
    bad = mkdesc(gpu, 100, 3, chi=-0.4, A=9 * 1.0 / (4 * 0.51), tau=0.51, prec=0)
    good = mkdesc(gpu, 48, 3, A=0.225, tau=1.0, prec=0)
    with gpu.Batch(chunk=500) as b:
        b.submit(bad, 20000, 1)
        b.submit(good, 1500, 2)
        ev = []
        for _ in range(100):
            b.advance()
            ev += b.poll()
            if b.stats().finished == 2:
                break
    kinds = {(e.tag, e.kind) for e in ev}
    assert (1, gpu.EV_UNSTABLE) in kinds and (2, gpu.EV_DONE) in kinds
    assert [e.step for e in ev if e.tag == 1 and e.kind == gpu.EV_UNSTABLE] == [500]


def test_many_cases_start_clean(gpu):
    """120 cases admitted at once (sizes 64-320, all operators, both precisions): every case's
    initial state is in place before its first step, so none is flagged at the step-0 diagnostic,
    and a sample of them give the same diagnostic bits as alone.  (The initial states are copied on
    the batch's own stream; a copy on the legacy stream is not ordered before a non-blocking
    stream's kernels.)"""
    rng = np.random.default_rng(7)
    specs = []
    for k in range(120):
        nx = int(rng.integers(64, 321))
        tipo, chi = [(1, 0.5), (3, 0.5), (3, 2.0), (11, 0.5), (12, 0.5), (13, 0.5)][k % 6]
        A = 0.225 if tipo < 11 else 0.1
        specs.append(mkdesc(gpu, nx, tipo, chi, A=A, prec=k % 2))
    flagged, rows = [], {}
    with gpu.Batch(chunk=50, diag_every=10 ** 6) as b:
        for k, d in enumerate(specs):
            b.submit(d, 10 ** 6, k)
        b.advance()
        for e in b.poll():
            if e.kind == gpu.EV_UNSTABLE:
                flagged.append(e.tag)
            elif e.kind == gpu.EV_DIAG:
                rows[e.tag] = e.drop.as_dict()
    assert not flagged, flagged
    assert len(rows) == len(specs)
    for k in (0, 1, 57, 118, 119):
        with gpu.Case(specs[k]) as c:
            c.step(1, keep_aux=True)
            alone = c.diag_drop(0).as_dict()
        for key in ("massa_R", "massa_B", "u_max", "raio", "delta_p", "min_f"):
            assert alone[key] == rows[k][key] or abs(alone[key] - rows[k][key]) <= 1e-12 * abs(alone[key]) + 1e-15, (k, key)


def test_launch_shapes_agree(gpu):
    """The autotuned batch (ctas_per_sm = 0), one CTA per tile (-1) and persistent CTAs (4 per SM) run
    the same kernels on the same tiles: the same bits.  The tuned batch reports the shape it chose."""
    cases = [(48, 3, 0.5, 0.225, 1, 0, (1, 0)), (40, 12, 0.5, 0.1, 0, 0, (1, 0)),
             (56, 11, 0.5, 0.1, 2, 1, (2, 1)), (37, 13, 0.5, 0.1, 1, 0, (1, 0))]
    descs = [mkdesc(gpu, nx, t, chi, A=A, prec=pr, geometry=g, p=pq[0], q=pq[1])
             for nx, t, chi, A, pr, g, pq in cases]
    rows, modes = {}, {}
    for cps in (0, -1, 4):
        with gpu.Batch(chunk=64, ctas_per_sm=cps) as b:
            for k, d in enumerate(descs):
                b.submit(d, 129, k)
            events = []
            for _ in range(20):
                b.advance()
                events += b.poll()
                st = b.stats()
                if st.active == 0 and st.pending == 0:
                    break
            modes[cps] = st.launch_mode
        rows[cps] = [(e.tag, e.step, (e.drop if cases[e.tag][5] == 0 else e.strip).as_dict())
                     for e in events if e.kind == gpu.EV_DIAG]
    assert len(rows[0]) == 2 * len(cases)  # the diagnostics at steps 0 and 128
    assert rows[0] == rows[-1] == rows[4]
    assert modes[-1] == -1 and modes[4] == 4 and modes[0] in (-1, 0)


def test_held_cases_give_their_final_fields(gpu):
    """With hold_finished, a retired case keeps its state until released and its final fields equal
    those of the same case run alone, bit for bit (both velocity forms); it is off the work
    table, so the others advance as before, and its memory counts until release."""
    mix = [(40, 12, 0.1, 0, 0, (1, 0), 501, 0.05), (36, 3, 0.225, 0, 1, (2, 1), 600, 0.0),
           (44, 13, 0.1, 1, 0, (1, 0), 700, 0.1), (48, 11, 0.1, 0, 0, (1, 0), 1300, 0.0)]
    descs = [mkdesc(gpu, nx, t, A=A, prec=pr, geometry=g, p=pq[0], q=pq[1], v0=v0)
             for nx, t, A, pr, g, pq, _, v0 in mix]
    alone = []
    for d, m in zip(descs, mix):
        with gpu.Case(d) as c:
            c.step(m[6], keep_aux=True)
            alone.append((c.read_fields(), c.read_profile()))
    got = {}
    with gpu.Batch(chunk=250) as b:
        b.hold_finished(True)
        for k, d in enumerate(descs):
            b.submit(d, mix[k][6], k)
        for _ in range(100):
            b.advance()
            for e in b.poll():
                if e.kind == gpu.EV_DIAG:
                    continue
                assert e.kind == gpu.EV_DONE
                n = descs[e.tag].nx * descs[e.tag].ny
                used = b.stats().hbm_used
                got[e.tag] = (b.read_fields(e.tag, n, gpu.FIELDS_VTK), b.read_fields(e.tag, n, gpu.FIELDS_PROFILE))
                assert b.stats().held >= 1
                b.release(e.tag)
                assert b.stats().hbm_used < used
                with pytest.raises(gpu.ItlbmError):
                    b.release(e.tag)
            st = b.stats()
            if st.active == 0 and st.pending == 0 and st.held == 0:
                break
    assert sorted(got) == list(range(len(mix)))
    for k, m in enumerate(mix):
        (fa, pa), (fb, pb) = alone[k], got[k]
        for key in ("rho_R", "rho_B", "ux", "uy", "uz"):
            assert np.array_equal(fa[key], fb[key]), (k, key)
        for key in ("rho_R", "rho_B", "ux", "uy"):
            assert np.array_equal(pa[key], pb[key]), (k, key)


def test_tilings_agree_and_are_reported(gpu):
    """The batch's autotuner times narrow edge tiles against 32 x 8 tiles throughout on its first full
    replay (the windows switch tilings in the middle of it) and reports its choice; no bit changes:
    every diagnostic equals that of the same case run alone."""
    cases = [(45, 3, 0.225, 1, 0, (1, 0)), (58, 12, 0.1, 1, 0, (1, 0)), (40, 11, 0.1, 2, 1, (2, 1)),
             (71, 13, 0.1, 0, 0, (1, 0)), (33, 1, 0.225, 1, 0, (1, 0)), (48, 12, 0.1, 2, 0, (1, 0))]
    descs = [mkdesc(gpu, nx, t, A=A, prec=pr, geometry=g, p=pq[0], q=pq[1]) for nx, t, A, pr, g, pq in cases]
    alone = [run_alone(gpu, d, 300)[0] for d in descs]
    with gpu.Batch(chunk=160) as b:
        for k, d in enumerate(descs):
            b.submit(d, 300, k)
        events = []
        for _ in range(20):
            b.advance()
            events += b.poll()
            st = b.stats()
            if st.active == 0 and st.pending == 0:
                break
        assert st.narrow_edges in (0, 1) and st.launch_mode in (-1, 0)
    for k, c in enumerate(cases):
        rows = [(e.drop if c[4] == 0 else e.strip).as_dict() for e in events if e.tag == k and e.kind == gpu.EV_DIAG]
        assert rows == alone[k], k
