"""SSF basis (sin/cos along x and y, Fourier along z; basis/SSF/pencil): the transforms
SSF_PENCIL::Forward_transform / Inverse_transform through ts_fft_forward / ts_fft_inverse
with the four parities, against the oracle (relative L2 <= 1e-13 FP64, 2e-6 FP32)."""
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu

KF = (math.pi, math.pi, 2 * math.pi)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("parity", ["SCF", "CSF", "SSF", "CCF"])
@pytest.mark.parametrize("N", [(16, 16, 16), (32, 16, 64), (48, 32, 16), (64, 96, 32)])
def test_ssf_transforms_match_oracle(cuda, N, parity, prec):
    import torch
    import tarang_b200 as tb
    g = R.Grid(N, KF, "SSF")
    plan = tb.Plan(N, basis="SSF", kfactor=KF, precision=prec)
    rng = np.random.default_rng(5)
    u = rng.standard_normal((2,) + N)
    rdt = torch.float64 if prec == "f64" else torch.float32
    real = torch.zeros((2, N[0], N[1], N[2] + 2), dtype=rdt, device=cuda)
    real[..., : N[2]] = torch.from_numpy(u).to(rdt)
    spec = plan.field(2)
    plan.forward(real, spec, parity=parity)
    torch.cuda.synchronize()
    ref = np.stack([R.forward(g, u[i], parity) for i in range(2)])
    tol = 1e-13 if prec == "f64" else 2e-6
    assert rel(spec.cpu().numpy(), ref) < tol
    back = torch.zeros_like(real)
    plan.inverse(spec, back, parity=parity)
    torch.cuda.synchronize()
    ub = back.cpu().numpy()
    assert rel(ub[..., : N[2]], np.stack([R.inverse(g, ref[i], parity) for i in range(2)])) < tol
    # the input of the inverse is not modified
    assert rel(spec.cpu().numpy(), ref) < tol


def test_ssf_plan_rejects_other_calls(cuda):
    import tarang_b200 as tb
    plan = tb.Plan(32, basis="SSF", kfactor=KF)
    u = plan.field(3)
    with pytest.raises(tb.TsError):
        plan.rk4_step_scalar(u, plan.field(1), 1)   # the passive-scalar step is FFF only
    with pytest.raises(tb.TsError):
        plan.rk4_step_mhd(u, plan.field(3), 1)
    with pytest.raises(tb.TsError):
        tb.Plan(32, basis="SSF", kfactor=KF, nlin_form="rotational")
    real = plan.field(1)
    with pytest.raises(tb.TsError):
        plan.forward(real, plan.field(1), parity="SFF")


def ssf_state(g, seed):
    """a random solenoidal field with the SSF parities (Vx = SCF, Vy = CSF, Vz = CCF)"""
    rng = np.random.default_rng(seed)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCF", "CSF", "CCF")])
    return R.project_rhs(g, U) * -1.0  # the projection keeps the solenoidal part


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((16, 16, 16), "reference"), ((32, 16, 32), "none"),
                                       ((48, 32, 16), "reference"), ((32, 32, 32), "two_thirds")])
def test_ssf_step_matches_oracle(cuda, N, dealias, prec):
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF, "SSF")
    U0 = 0.3 * ssf_state(g, 2)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=mode, nlin_form="conservative")
    W = U0.copy()
    for _ in range(3):
        W = R.rk4_step(cfg, W)
    plan = tb.Plan(N, basis="SSF", kfactor=KF, precision=prec, nu=0.01, dt=1e-3, dealias=dealias)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(U0).to(cuda).to(cdt)
    plan.rk4_step(u, 3)
    plan.status()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel(u.cpu().numpy().astype(np.complex128), W) < tol


def test_ssf_taylor_green_decays_exactly(cuda):
    """u = sin x cos y, v = -cos x sin y (Vx = SCF, Vy = CSF): the nonlinear term is a
    gradient, so the step is the exact viscous decay exp(-2 nu t)."""
    import torch
    import tarang_b200 as tb
    N = (16, 16, 16)
    g = R.Grid(N, (1.0, 1.0, 1.0), "SSF")
    x = (np.arange(16) + 0.5) * np.pi / 16
    z = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    U0 = np.stack([R.forward(g, np.sin(X) * np.cos(Y), "SCF"), R.forward(g, -np.cos(X) * np.sin(Y), "CSF"),
                   R.forward(g, np.zeros_like(X), "CCF")])
    plan = tb.Plan(N, basis="SSF", kfactor=(1.0, 1.0, 1.0), precision="f64", nu=0.05, dt=1e-2)
    u = torch.from_numpy(U0).to(cuda)
    plan.rk4_step(u, 5)
    assert np.max(np.abs(u.cpu().numpy() - U0 * np.exp(-0.05 * 2 * 5e-2))) < 1e-15


KF_RBC = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))   # SSF_PENCIL's RBC default


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((16, 16, 16), "reference"), ((32, 16, 32), "none"),
                                       ((48, 32, 16), "two_thirds"), ((32, 32, 32), "reference")])
def test_ssf_rbc_step_matches_oracle(cuda, N, dealias, prec):
    """RBC on SSF (ts_rk4_step_rbc on an SSF plan; T = SCF) over 3 steps against the oracle."""
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF_RBC, "SSF")
    U0 = 0.3 * ssf_state(g, 5)
    rng = np.random.default_rng(9)
    T0 = 0.3 * R.forward(g, rng.standard_normal(g.rshape), "SCF")
    cfg = R.RBCConfig(g, Ra=1e5, Pr=0.7, dt=1e-3, dealias_mode=mode)
    Uo, To = U0.copy(), T0.copy()
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan = tb.Plan(N, basis="SSF", kfactor=KF_RBC, precision=prec, nu=cfg.nu, kappa=cfg.kappa, dt=1e-3,
                   dealias=dealias, Ra=1e5, Pr=0.7)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(U0).to(cuda).to(cdt)
    T = torch.from_numpy(T0).to(cuda).to(cdt)
    plan.rk4_step_rbc(u, T, 3)
    plan.status()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
    assert rel(T.cpu().numpy().astype(np.complex128), To) < tol


def test_ssf_rbc_roll_follows_linear_theory(cuda):
    """One small roll (u_x, theta in sin(kx x) cos(ky y)) grows or decays as the linear
    system da/dt = (1 - kx^2/K^2) b - nu K^2 a, db/dt = a - kappa K^2 b predicts."""
    from scipy.linalg import expm
    import tarang_b200 as tb
    N = (16, 16, 16)
    eps, nu, kappa, dt, n = 1e-9, 0.01, 0.02, 2e-3, 25
    plan = tb.Plan(N, basis="SSF", kfactor=KF_RBC, nu=nu, kappa=kappa, dt=dt)
    u, T = plan.field(3), plan.field(1)
    kx, ky = KF_RBC[0], KF_RBC[1]
    u[0, 1, 1, 0] = eps
    u[1, 1, 1, 0] = -kx * eps / ky
    T.view(N[0], N[1], -1)[1, 1, 0] = 0.5 * eps
    plan.rk4_step_rbc(u, T, n)
    K2 = kx * kx + ky * ky
    a, b = expm(np.array([[-nu * K2, 1 - kx * kx / K2], [1.0, -kappa * K2]]) * n * dt) @ np.array([eps, 0.5 * eps])
    assert abs(u[0, 1, 1, 0].item() - a) < 1e-7 * eps
    assert abs(T.view(N[0], N[1], -1)[1, 1, 0].item() - b) < 1e-7 * eps


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_ssf_energy_and_nusselt_match_oracle(cuda, prec):
    """ts_energy with the SSF weights (Multiplicity_factor 4 / 2 / 1 / 1/2) and the Nusselt
    number 1 + 2 sqrt(Ra Pr) <U1, T> on an SSF plan, against the oracle."""
    import torch
    import tarang_b200 as tb
    N = (32, 16, 32)
    g = R.Grid(N, KF_RBC, "SSF")
    U = 0.3 * ssf_state(g, 3)
    rng = np.random.default_rng(4)
    T = 0.3 * R.forward(g, rng.standard_normal(g.rshape), "SCF")
    cfg = R.RBCConfig(g, Ra=2e5, Pr=0.7, dt=1e-3)
    plan = tb.Plan(N, basis="SSF", kfactor=KF_RBC, precision=prec, nu=cfg.nu, kappa=cfg.kappa, Ra=2e5, Pr=0.7)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(U).to(cuda).to(cdt)
    t = torch.from_numpy(T[None]).to(cuda).to(cdt)
    Ur = u.cpu().numpy().astype(np.complex128)   # the values the device holds
    Tr = t.cpu().numpy().astype(np.complex128)[0]
    tol = 1e-12 if prec == "f64" else 1e-6
    assert abs(plan.energy(u) / R.total_energy(g, Ur) - 1) < tol
    assert abs(plan.energy(t) / R.total_energy_scalar(g, Tr) - 1) < tol
    assert abs(plan.nusselt(u, t) - R.nusselt(cfg, Ur, Tr)) < tol * abs(R.nusselt(cfg, Ur, Tr))


def test_ssf_max_div_matches_oracle(cuda):
    """ts_max_div on an SSF plan: ~0 for a projected field, the oracle's value for a random one."""
    import torch
    import tarang_b200 as tb
    N = (32, 16, 32)
    g = R.Grid(N, KF, "SSF")
    rng = np.random.default_rng(12)
    V = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCF", "CSF", "CCF")])
    plan = tb.Plan(N, basis="SSF", kfactor=KF)
    assert abs(plan.max_div(torch.from_numpy(V).to(cuda)) / R.max_abs_div(g, V) - 1) < 1e-12
    W = -R.project_rhs(g, V)
    assert plan.max_div(torch.from_numpy(W).to(cuda)) < 1e-12 * R.max_abs_div(g, V)


@pytest.mark.parametrize("basis,N", [("SSF", (16, 32, 16)), ("SSF", (32, 16, 32)), ("SSS", (16, 32, 16)),
                                     ("SSS", (32, 16, 32))])
def test_sincos_shell_spectrum_matches_oracle(cuda, basis, N):
    """E(k) on SSF and SSS: the reference's shell loop over the complex array shape
    (universal_energy.cc:276-306) with the basis's grid wavenumbers (kx = lx, ky = ly, kz = lz),
    Multiplicity_factor (4 / 2 / 1 / 1/2) and Min_radius_outside; on SSS each pair of real z
    coefficients is one complex slot at kz = lz.  FP64 <= 1e-13, FP32 <= 1e-6."""
    import torch
    import tarang_b200 as tb
    kf = (math.pi, math.pi / math.sqrt(2.0), 0.7 * math.pi)
    g = R.Grid(N, kf, basis)
    rng = np.random.default_rng(4)
    par = ("SCF", "CSF", "CCF") if basis == "SSF" else ("SCC", "CSC", "CCS")
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in par])
    ref = R.shell_spectrum(g, U)
    for prec, tol in (("f64", 1e-13), ("f32", 1e-6)):
        plan = tb.Plan(N, basis=basis, precision=prec, kfactor=kf)
        assert plan.n_shells == len(ref)
        if basis == "SSS":
            P = np.zeros((3, N[0], N[1], N[2] + 2))
            P[..., :N[2]] = U
            u = torch.view_as_complex(torch.from_numpy(P.reshape(3, N[0], N[1], N[2] // 2 + 1, 2)).to(
                torch.float64 if prec == "f64" else torch.float32).contiguous()).to(cuda)
        else:
            u = torch.from_numpy(U).to(cuda).to(plan.torch_dtype())
        got = plan.shell_spectrum(u)
        assert rel(got, ref) < tol, (prec, rel(got, ref))
        plan.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dealias", ["reference", "none", "two_thirds"])
def test_ssf_flux_matches_oracle(cuda, prec, dealias):
    """Pi(R) on SSF, the reference's per-sphere algorithm (EnergyTr::Compute_flux,
    compute_flux.cc:51-65: one giver nonlinear term per sphere, summed outside it) against
    the oracle's flux_per_sphere: FP64 to 1e-12, FP32 to 2e-6 of max|Pi|."""
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    N = (16, 32, 16)
    kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    g = R.Grid(N, kf, "SSF")
    U = 0.3 * ssf_state(g, 13)
    radii = [1.0, 2.5, 4.0, 6.0, 9.0]
    want = R.flux_per_sphere(g, U, radii, mode)
    plan = tb.Plan(N, basis="SSF", precision=prec, kfactor=kf, dealias=dealias)
    u = torch.from_numpy(np.ascontiguousarray(U)).to(cuda).to(plan.torch_dtype())
    got = plan.flux(u, radii)
    tol = 1e-12 if prec == "f64" else 2e-6
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want)), (got, want)
    plan.close()
