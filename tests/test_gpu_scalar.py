"""Passive scalar on the FFF basis (program.kind SCALAR_INCOMPRESS): RK4(U,T,P,F) with no force,
through ts_rk4_step_scalar, against the FP64 oracle (relative L2 <= 1e-12 FP64, 1e-5 FP32)."""
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
    rng = np.random.default_rng(seed + 7)
    T = R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape)))
    return g, U, T


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((32, 32, 32), "reference"), ((32, 16, 64), "two_thirds"),
                                       ((64, 32, 16), "none"), ((64, 64, 64), "two_thirds")])
def test_scalar_step_matches_oracle(cuda, N, dealias, prec):
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g, U0, T0 = state(N)
    cfg = R.ScalarConfig(g, nu=0.01, kappa=0.02, dt=1e-3, dealias_mode=mode)
    Uo, To = U0.copy(), T0.copy()
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan = tb.Plan(N, precision=prec, nu=0.01, kappa=0.02, dt=1e-3, dealias=dealias)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(U0).to(cuda).to(cdt)
    T = torch.from_numpy(T0).to(cuda).to(cdt)
    plan.rk4_step_scalar(u, T, 3)
    plan.status()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
    assert rel(T.cpu().numpy().astype(np.complex128), To) < tol


def test_scalar_mean_kept_and_variance_decays(cuda):
    """The K = 0 mode of T has no advective or diffusive change; <T'^2> decays without forcing."""
    import torch
    import tarang_b200 as tb
    g, U0, T0 = state((32, 32, 32), seed=3)
    T0 = T0.copy()
    T0[0, 0, 0] = 0.25
    plan = tb.Plan(32, precision="f64", nu=0.01, kappa=0.05, dt=2e-3, dealias="two_thirds")
    u = torch.from_numpy(U0).to(cuda)
    T = torch.from_numpy(T0).to(cuda)
    e0 = plan.energy(T, 1)
    plan.rk4_step_scalar(u, T, 20)
    t = T.cpu().numpy()
    assert abs(t[0, 0, 0] - 0.25) < 1e-14
    assert plan.energy(T, 1) < e0
    assert plan.max_div(u) < 1e-12


def test_scalar_step_rejects_other_plans(cuda):
    import math
    import tarang_b200 as tb
    rot = tb.Plan(32, nlin_form="rotational")
    u, T = rot.field(3), rot.field(1)
    with pytest.raises(tb.TsError):
        rot.rk4_step_scalar(u, T, 1)
    sff = tb.Plan(32, basis="SFF", kfactor=(math.pi, 2 * math.pi, 2 * math.pi))
    with pytest.raises(tb.TsError):
        sff.rk4_step_scalar(sff.field(3), sff.field(1), 1)
