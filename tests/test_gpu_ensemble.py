"""Ensemble of RBC runs of uneven sizes (one CUDA graph launch per step) and the
non-power-of-two SFF sizes 48 / 96 (radix-3 FFT passes), through the C ABI."""
import ctypes
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

KF = (math.pi, 2 * math.pi, 2 * math.pi)


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def test_member_generator_is_deterministic():
    import tarang_b200 as tb
    a, b = tb.ensemble_members(), tb.ensemble_members()
    assert a == b and len(a) == 64
    assert {m[0] for m in a} == {32, 48, 64, 96, 128}
    assert all(1e5 <= m[1] <= 1e7 for m in a)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("N", [(48, 48, 48), (96, 32, 48), (32, 96, 96)])
def test_mixed_radix_rbc_matches_oracle(cuda, N, prec):
    """SFF path at sizes with a factor 3 against the FP64 oracle (relative L2 <= 1e-5 FP32, 1e-12 FP64)."""
    import torch
    import tarang_b200 as tb
    g = R.Grid(N, KF, "SFF")
    rng = np.random.default_rng(2)
    par = ["S", "C", "C"]
    U0 = np.stack([R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), par[i])) for i in range(3)])
    T0 = R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), "S"))
    cfg = R.RBCConfig(g, Ra=1e5, Pr=1.0, dt=1e-3, dealias_mode=1)
    plan = tb.Plan(N, basis="SFF", precision=prec, kfactor=KF, nu=cfg.nu, kappa=cfg.kappa, dt=1e-3)
    cdt = torch.complex64 if prec == "f32" else torch.complex128
    u = torch.from_numpy(U0.copy()).to(cuda).to(cdt)
    T = torch.from_numpy(T0.copy()).to(cuda).to(cdt)
    Uo, To = U0, T0
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan.rk4_step_rbc(u, T, 3)
    torch.cuda.synchronize()
    tol = 1e-5 if prec == "f32" else 1e-12
    assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
    assert rel(T.cpu().numpy().astype(np.complex128), To) < tol


@pytest.mark.gpu
def test_ensemble_equals_independent_runs(cuda):
    """Members advanced together in one graph match the same runs done one plan at a time, bit for bit."""
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    members = [(32, 1e5, 1.0), (48, 3e5, 1.0), ((64, 32, 32), 1e6, 1.0), (16, 2e6, 1.0)]
    ens = tb.Ensemble(members, dt=1e-3)
    ens.init_temperature(1e-3, 4.0, 3)
    ens.run(3)
    ens.run(8)   # one launch of the eight-step graph (each size group a chain of its own)
    Nu = ens.nusselt()
    lib = L.load()
    for m, (N, Ra, Pr) in enumerate(members):
        N = (N, N, N) if isinstance(N, int) else N
        plan = tb.Plan(N, basis="SFF", precision="f32", kfactor=KF, nu=math.sqrt(Pr / Ra), kappa=1 / math.sqrt(Pr * Ra),
                       dt=1e-3, Ra=Ra, Pr=Pr)
        u = plan.field(3)
        T = plan.field(1)
        plan.init_temperature_perturbation(1e-3, 4.0, 3 + m, T)
        plan.rk4_step_rbc(u, T, 11)
        torch.cuda.synchronize()
        # same kernels, same arithmetic per member: the states agree bit for bit
        ens.synchronize()
        assert torch.equal(ens.view(m, "U"), u) and torch.equal(ens.view(m, "T"), T)
        assert abs(plan.nusselt(u, T) - Nu[m]) <= 1e-13 * abs(Nu[m])
        assert abs(plan.energy(T) - ens.energy(m, "T")) <= 1e-13 * plan.energy(T)
        eu = plan.energy(u)
        assert abs(eu - ens.energy(m, "U")) <= 1e-13 * eu
    ens.close()
