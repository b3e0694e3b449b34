"""The analytic operator checks of the reference (verifica_operadores.cpp, E0) on the oracle's
per-site functions, against the tolerances the reference uses and the numbers it printed
(E0_resultado.txt, committed as tests/golden/e0_resultado.json)."""
import math

import numpy as np
import pytest

# D3Q19 (def_lattice_d3q19, LBM_functions.cpp:366-497)
C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1],
              [-1, 0, 1], [0, -1, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1]], dtype=float)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
CASES = [(1, 0.5, 0.0, "P1"), (3, -0.4, 1.0, "P3 chi=-2/5 (RP)"), (3, 0.5, 1.0, "P3 chi=1/2 (LKR)"),
         (3, 2.0, 1.0, "P3 chi=2 (LVK)")]
A, MG = 0.37, 0.81  # verifica_operadores.cpp:42


def perturb(fn, tipo, chi, g):
    return fn(tipo, chi, A, np.asarray(g, dtype=float), np.zeros(19))


@pytest.mark.parametrize("tipo,chi,lam,name", CASES)
def test_class_p_moments(oracle, tipo, chi, lam, name):
    """M0 = 0, M1 = 0, M2 = (2/9) A |g| (nn - lambda I), tolerance 1e-14 (verifica_operadores.cpp:187-234)."""
    rng = np.random.default_rng(7)
    e0 = e1 = e2 = 0.0
    for _ in range(200):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        f = oracle.perturbacao(tipo, chi, A, MG * n, np.zeros(19))
        M0, M1, M2 = f.sum(), C.T @ f, (C.T * f) @ C
        e0, e1 = max(e0, abs(M0)), max(e1, abs(M1).max())
        e2 = max(e2, abs(M2 - 2 / 9 * A * MG * (np.outer(n, n) - lam * np.eye(3))).max())
    assert e0 <= 1e-14 and e1 <= 1e-14 and e2 <= 1e-14


@pytest.mark.parametrize("tipo,chi,lam,name", CASES)
def test_m4_table(oracle, golden, tipo, chi, lam, name):
    """M4_nnnn / (A|g|) against the in-plane angle, as printed in E0_resultado.txt:20-24."""
    row = []
    for th in (0.0, 15.0, 22.5, 30.0, 45.0):
        t = th * math.pi / 180.0
        n = np.array([math.cos(t), math.sin(t), 0.0])
        f = oracle.perturbacao(tipo, chi, A, MG * n, np.zeros(19))
        cn = C[:, 0] * n[0] + C[:, 1] * n[1]
        row.append((f * cn ** 4).sum() / (A * MG))
    assert np.allclose(row, golden["e0"]["m4"][name], atol=6e-7)


@pytest.mark.parametrize("chi", [-0.4, 0.5, 2.0, 7.0])
def test_nz1_fold(oracle, chi):
    """P3(chi) folded in z equals the D2Q9 member chi + 2 (verifica_operadores.cpp:265-307), 1e-15."""
    g = np.array([MG * math.cos(0.3), MG * math.sin(0.3), 0.0])
    f = oracle.perturbacao(3, chi, A, g, np.zeros(19))
    f9 = np.zeros((3, 3))
    for i in range(19):
        f9[int(C[i, 0]) + 1, int(C[i, 1]) + 1] += f[i]
    c2x = chi + 2.0
    B9 = [-c2x / (3 * (c2x + 2)), c2x / (6 * (c2x + 2)), 1 / (6 * (c2x + 2))]
    err = 0.0
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            s = abs(a) + abs(b)
            w9 = 4 / 9 if s == 0 else (1 / 9 if s == 1 else 1 / 36)
            cg = a * g[0] + b * g[1]
            err = max(err, abs(A * MG * (w9 * cg * cg / (MG * MG) - B9[s]) - f9[a + 1, b + 1]))
    assert err <= 1e-15


def test_guo_source_moments(oracle):
    """sum S = 0 and sum S c = (1 - 1/2tau) F (verifica_operadores.cpp:309-323), 1e-16."""
    tau, rho, F, u = 0.8, 1.03, [1.3e-3, -2.1e-3, 0.0], [0.02, -0.01, 0.0]
    S = oracle.source(F, u, rho, tau)
    assert abs(S.sum()) <= 1e-16
    M1 = C.T @ S
    assert abs(M1[0] - (1 - 0.5 / tau) * F[0]) <= 1e-16
    assert abs(M1[1] - (1 - 0.5 / tau) * F[1]) <= 1e-16


def tanh_fields(nx, ny, xi, disc, R=60.0):
    x, y = np.meshgrid(np.arange(nx), np.arange(ny))
    if disc:
        s = R - np.hypot(x - nx / 2.0, y - ny / 2.0)
    else:
        ax = np.abs(x - nx / 2.0)
        s = np.where(ax < nx / 4.0, nx / 4.0 - ax, -(ax - nx / 4.0))
    ph = np.tanh(s / xi).ravel()
    fR = (W[None, :] * 0.5 * (1 + ph)[:, None]).ravel()
    fB = (W[None, :] * 0.5 * (1 - ph)[:, None]).ravel()
    return fR, fB


def force_checks(F, nx, ny, sigma, R):
    F = F.reshape(-1, 3)
    return F


@pytest.mark.parametrize("xi", [1.569988, 3.0, 6.0])
@pytest.mark.parametrize("tipo", [11, 12, 13])
def test_class_f_on_tanh_profiles(oracle, golden, tipo, xi):
    """verifica_operadores.cpp:325-403: flat profile max|F|/(sigma/xi) ~ 0, disc sum F_r dr/(sigma/R) - 1."""
    nx = ny = 256
    sigma, R = 0.1, 60.0
    fR, fB = tanh_fields(nx, ny, xi, False)
    F = oracle.calcula_forca(tipo, xi, sigma, nx, ny, fR, fB).reshape(-1, 3)
    fmax = (abs(F[:, 0]) + abs(F[:, 1])).max()
    fR, fB = tanh_fields(nx, ny, xi, True, R)
    F = oracle.calcula_forca(tipo, xi, sigma, nx, ny, fR, fB).reshape(-1, 3)
    x, y = np.meshgrid(np.arange(nx), np.arange(ny))
    dx, dy = (x - nx / 2.0).ravel(), (y - ny / 2.0).ravel()
    r = np.hypot(dx, dy)
    m = r >= 1e-9
    soma = (-(F[m, 0] * dx[m] + F[m, 1] * dy[m]) / r[m] / (2 * math.pi * r[m])).sum()
    tol_p = 0.2 / xi ** 2 if tipo == 13 else 1e-3
    tol_d = 1.5 * (xi / R) ** 2 + 5e-4 + (0.25 / xi ** 2 if tipo == 13 else 0.0)
    plano, disco = fmax / (sigma / xi), soma / (sigma / R) - 1.0
    assert abs(plano) <= tol_p and abs(disco) <= tol_d
    # the numbers the reference printed (E0_resultado.txt, 4 significant digits)
    name = {11: "F1 CSF", 12: "F2 div T", 13: "F3 mu grad phi"}[tipo]
    sec = f"{name}   ( xi = {xi:.3f} )"
    ref = {c["what"].split(":")[0]: c["erro"] for c in golden["e0"]["checks"] if c["section"] == sec}
    assert ref, sec
    assert math.isclose(disco, ref["disco"], rel_tol=2e-3, abs_tol=1e-6)
    assert abs(plano - ref["plano"]) <= max(2e-3 * abs(ref["plano"]), 1e-9)
