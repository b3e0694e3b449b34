"""Error of the FP32 storage forms against the plain FP64 path, per observable, on the third reference
configuration.  The FP64 path is bit-identical to the reference's own step (test_gpu_parity.py,
test_gpu_config2.py), so its results stand for the reference here.

* Translating drop: 512 x 512 x 1 periodic, R = 30, uniform initial velocity v0 in {0.05, ..., 0.25}
  along x, operators F2 and P3 chi = 0.5, tau = 0.8, sigma = 0.1, 20 000 steps, logistic initial
  profile (Imm_OPS.cpp:199).  Diagnostics at steps 4 999, 9 999, 14 999 and 19 999.
* Static drop: 4096 x 4096 x 1, R = 400, P3 chi = 0.5 and F2, 4 000 steps.

Observables (laplace.dat, iso.dat and galilean.dat columns): the Laplace pressure jump delta_p, the
measured tension sigma = R delta_p (Other_functions.cpp:530-553), the peak spurious velocity |u - v0|max
(Galilean_diagnostics.cpp:68-104), the equimolar radius, the drop-frame slip center_dx
(Galilean_diagnostics.cpp:93-95) and the interface mode amplitudes |a2|, |a4|, |a8| / R0
(Operadores_tensao.cpp:382-449).  Bars, for every operator and both FP32 forms: delta_p within 0.5 %,
peak spurious velocity within 5 %; the other errors are stated (printed, and written as JSON to
$ITLBM_REPORT_DIR/fp32_errors.json when that variable is set) with the bounds asserted in check().
"""
import json
import math
import os

import pytest

from test_gpu_parity import gpu_case

pytestmark = pytest.mark.gpu

SIGMA = 0.1
OPERATORS = [("P3 0.5", 3, 0.5, 1.569988), ("F2", 12, 0.5, 1.569988)]
PRECISIONS = [("fp32", 1), ("fold", 2)]
REPORT = []


def amplitude(tipo, tau):
    return SIGMA if tipo >= 11 else 9.0 * SIGMA / (4.0 * tau)


def rel(a, b):
    return abs(a - b) / abs(b) if b != 0 else abs(a - b)


def errors(d, ref):
    """Per-observable error of diagnostic d against the FP64 diagnostic ref."""
    return {
        "delta_p": rel(d.delta_p, ref.delta_p),
        "sigma": rel(d.sigma, ref.sigma),
        "u_max": rel(d.u_max, ref.u_max),
        "raio": rel(d.raio, ref.raio),
        "slip": abs(d.center_dx - ref.center_dx),
        "a2": abs(d.a2 - ref.a2),
        "a4": abs(d.a4 - ref.a4),
        "a8": abs(d.a8 - ref.a8),
    }


def run_lockstep(gpu, nx, R, v0, tipo, chi, xi, tau, diag_steps):
    A = amplitude(tipo, tau)
    cases = {"fp64": gpu_case(gpu, nx, nx, tipo, chi, xi, A, tau=tau, radius=R, v0=v0)}
    for label, prec in PRECISIONS:
        cases[label] = gpu_case(gpu, nx, nx, tipo, chi, xi, A, tau=tau, radius=R, v0=v0, prec=prec)
    worst = {label: {} for label, _ in PRECISIONS}
    last = {}
    for s in diag_steps:
        for c in cases.values():
            c.step(s + 1 - c.steps_done, keep_aux=True)
        d = {k: c.diag_drop(s) for k, c in cases.items()}
        assert all(x.ok for x in d.values()), s
        for label, _ in PRECISIONS:
            for k, e in errors(d[label], d["fp64"]).items():
                worst[label][k] = max(worst[label].get(k, 0.0), e)
        last = d
    for c in cases.values():
        c.close()
    return worst, last


def record(row):
    REPORT.append(row)
    print(json.dumps(row))
    out = os.environ.get("ITLBM_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "fp32_errors.json"), "w") as f:
            json.dump(REPORT, f, indent=1)


def check(worst):
    """The bars: the Laplace jump and the peak spurious velocity as the path's specification states them
    (0.5 %, 5 %); the other observables at a few times their largest error measured on B200 (delta_p
    6e-5, sigma 6e-5, radius 1e-6, slip 0.014 lattice units, |a_k| / R0 2.5e-5)."""
    for label, w in worst.items():
        assert w["delta_p"] <= 5e-3, (label, w)
        assert w["u_max"] <= 0.05, (label, w)
        assert w["sigma"] <= 5e-3, (label, w)
        assert w["raio"] <= 1e-5, (label, w)
        assert w["slip"] <= 0.05, (label, w)  # lattice units, after up to 5 000 of travel
        for k in ("a2", "a4", "a8"):
            assert w[k] <= 1e-4, (label, k, w)


@pytest.mark.parametrize("name,tipo,chi,xi", OPERATORS, ids=[o[0] for o in OPERATORS])
@pytest.mark.parametrize("v0", [0.05, 0.10, 0.15, 0.20, 0.25])
def test_translating_drop_512(gpu, name, tipo, chi, xi, v0):
    worst, last = run_lockstep(gpu, 512, 30.0, v0, tipo, chi, xi, 0.8, [4999, 9999, 14999, 19999])
    f64 = last["fp64"]
    record({"case": f"512^2 R=30 v0={v0} {name} tau=0.8, 20000 steps", "errors": worst,
            "fp64": {"delta_p": f64.delta_p, "sigma": f64.sigma, "u_max": f64.u_max, "raio": f64.raio,
                     "center_dx": f64.center_dx, "a2": f64.a2, "a4": f64.a4, "a8": f64.a8}})
    check(worst)


@pytest.mark.parametrize("name,tipo,chi,xi", OPERATORS, ids=[o[0] for o in OPERATORS])
def test_static_drop_4096(gpu, name, tipo, chi, xi):
    worst, last = run_lockstep(gpu, 4096, 400.0, 0.0, tipo, chi, xi, 0.8, [3999])
    f64 = last["fp64"]
    record({"case": f"4096^2 R=400 static {name} tau=0.8, 4000 steps", "errors": worst,
            "fp64": {"delta_p": f64.delta_p, "sigma": f64.sigma, "u_max": f64.u_max, "raio": f64.raio,
                     "center_dx": f64.center_dx, "a2": f64.a2, "a4": f64.a4, "a8": f64.a8}})
    check(worst)
