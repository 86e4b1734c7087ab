"""SSS basis (sin/cos along every axis; basis/SSS/pencil): the transforms through
ts_fft_forward / ts_fft_inverse with parities [SC][SC][SC] against the oracle
(relative L2 <= 1e-13 FP64, 2e-6 FP32).  The coefficients are real and live in the
padded real layout (Nx, Ny, Nz + 2) of each component, as SSS_PENCIL stores them."""
import itertools
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu

KF = (math.pi, math.pi, math.pi)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("parity", ["".join(p) for p in itertools.product("SC", repeat=3)])
@pytest.mark.parametrize("N", [(16, 16, 16), (32, 16, 64), (48, 32, 32)])
def test_sss_transforms_match_oracle(cuda, N, parity, prec):
    import torch
    import tarang_b200 as tb
    g = R.Grid(N, KF, "SSS")
    plan = tb.Plan(N, basis="SSS", kfactor=KF, precision=prec)
    rng = np.random.default_rng(7)
    u = rng.standard_normal((2,) + N)
    rdt = torch.float64 if prec == "f64" else torch.float32
    real = torch.zeros((2, N[0], N[1], N[2] + 2), dtype=rdt, device=cuda)
    real[..., : N[2]] = torch.from_numpy(u).to(rdt)
    spec = plan.field(2)
    plan.forward(real, spec, parity=parity)
    torch.cuda.synchronize()
    coef = torch.view_as_real(spec).reshape(2, N[0], N[1], N[2] + 2)[..., : N[2]].cpu().numpy()
    ref = np.stack([R.forward(g, u[i], parity) for i in range(2)])
    tol = 1e-13 if prec == "f64" else 2e-6
    assert rel(coef, ref) < tol
    back = torch.zeros_like(real)
    plan.inverse(spec, back, parity=parity)
    torch.cuda.synchronize()
    ub = back.cpu().numpy()
    assert rel(ub[..., : N[2]], np.stack([R.inverse(g, ref[i], parity) for i in range(2)])) < tol


def test_sss_plan_rejects_other_calls(cuda):
    import tarang_b200 as tb
    plan = tb.Plan(32, basis="SSS", kfactor=KF)
    u = plan.field(3)
    with pytest.raises(tb.TsError):
        plan.rk4_step(u, 1)
    with pytest.raises(tb.TsError):
        plan.energy(u)
    with pytest.raises(tb.TsError):
        plan.forward(plan.field(1), plan.field(1), parity="SCF")
