"""Incompressible MHD on the FFF basis: RK4(U, W, P, F) with W = B and no force, through
ts_rk4_step_mhd, against the FP64 oracle (relative L2 <= 1e-12 FP64, 1e-5 FP32), plus
the invariants of the ideal equations."""
import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def state(N, seed=0):
    g = R.Grid(N)
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), seed, 0.5)
    B = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 3.0), seed + 1, 0.3)
    return g, U, B


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((32, 32, 32), "reference"), ((32, 16, 64), "two_thirds"),
                                       ((64, 32, 16), "none"), ((64, 64, 64), "two_thirds")])
def test_mhd_step_matches_oracle(cuda, N, dealias, prec):
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g, U0, B0 = state(N)
    cfg = R.MHDConfig(g, nu=0.01, eta=0.02, dt=1e-3, dealias_mode=mode)
    Uo, Bo = U0.copy(), B0.copy()
    for _ in range(3):
        Uo, Bo = R.mhd_rk4_step(cfg, Uo, Bo)
    plan = tb.Plan(N, precision=prec, nu=0.01, kappa=0.02, dt=1e-3, dealias=dealias)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(U0).to(cuda).to(cdt)
    b = torch.from_numpy(B0).to(cuda).to(cdt)
    plan.rk4_step_mhd(u, b, 3)
    plan.status()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
    assert rel(b.cpu().numpy().astype(np.complex128), Bo) < tol


def test_ideal_mhd_invariants(cuda):
    """nu = eta = 0: total energy and cross helicity are kept to the time-stepping error;
    both fields stay solenoidal."""
    import torch
    import tarang_b200 as tb
    g, U0, B0 = state((32, 32, 32), seed=4)
    plan = tb.Plan(32, precision="f64", nu=0.0, kappa=0.0, dt=1e-3, dealias="two_thirds")
    u, b = torch.from_numpy(U0).to(cuda), torch.from_numpy(B0).to(cuda)
    e0 = plan.energy(u) + plan.energy(b)
    H0 = sum(R.cross_energy(g, U0[i], B0[i]) for i in range(3))
    plan.rk4_step_mhd(u, b, 10)
    un, bn = u.cpu().numpy(), b.cpu().numpy()
    e1 = plan.energy(u) + plan.energy(b)
    H1 = sum(R.cross_energy(g, un[i], bn[i]) for i in range(3))
    assert abs(e1 - e0) < 1e-5 * e0
    assert abs(H1 - H0) < 1e-5 * e0
    assert plan.max_div(u) < 1e-12 and plan.max_div(b) < 1e-12


def test_mhd_step_rejects_other_plans(cuda):
    import math
    import tarang_b200 as tb
    sff = tb.Plan(32, basis="SFF", kfactor=(math.pi, 2 * math.pi, 2 * math.pi))
    with pytest.raises(tb.TsError):
        sff.rk4_step_mhd(sff.field(3), sff.field(3), 1)
