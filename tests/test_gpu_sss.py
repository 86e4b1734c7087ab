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
        tb.Plan(32, basis="SSS", kfactor=KF, nlin_form="rotational")
    with pytest.raises(tb.TsError):
        plan.forward(plan.field(1), plan.field(1), parity="SCF")


def to_padded(A):
    """real coefficients (c, Nx, Ny, Nz) -> the padded real layout viewed as complex"""
    c, Nx, Ny, Nz = A.shape
    P = np.zeros((c, Nx, Ny, Nz + 2))
    P[..., :Nz] = A
    return P.view(np.complex128)


def from_padded(t, Nz):
    import torch
    a = torch.view_as_real(t).reshape(t.shape[0], t.shape[1], t.shape[2], -1).cpu().numpy().astype(np.float64)
    return a[..., :Nz]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((16, 16, 16), "reference"), ((32, 16, 32), "none"),
                                       ((32, 32, 16), "two_thirds")])
def test_sss_step_matches_oracle(cuda, N, dealias, prec):
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF, "SSS")
    rng = np.random.default_rng(4)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCC", "CSC", "CCS")])
    U0 = -0.3 * R.project_rhs(g, U)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=mode, nlin_form="conservative")
    W = U0.copy()
    for _ in range(3):
        W = R.rk4_step(cfg, W)
    plan = tb.Plan(N, basis="SSS", kfactor=KF, precision=prec, nu=0.01, dt=1e-3, dealias=dealias)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(to_padded(U0)).to(cuda).to(cdt) if prec == "f64" else \
        torch.view_as_complex(torch.from_numpy(to_padded(U0).view(np.float64).reshape(3, N[0], N[1], N[2] // 2 + 1, 2)
                                               .astype(np.float32)).contiguous()).to(cuda)
    plan.rk4_step(u, 3)
    plan.status()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel(from_padded(u, N[2]), W) < tol


def test_sss_taylor_green_decays_exactly(cuda):
    import torch
    import tarang_b200 as tb
    N = (16, 16, 16)
    g = R.Grid(N, (1.0, 1.0, 1.0), "SSS")
    x = (np.arange(16) + 0.5) * np.pi / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    U0 = np.stack([R.forward(g, np.sin(X) * np.cos(Y), "SCC"), R.forward(g, -np.cos(X) * np.sin(Y), "CSC"),
                   R.forward(g, np.zeros_like(X), "CCS")])
    plan = tb.Plan(N, basis="SSS", kfactor=(1.0, 1.0, 1.0), precision="f64", nu=0.05, dt=1e-2)
    u = torch.from_numpy(to_padded(U0)).to(cuda)
    plan.rk4_step(u, 5)
    assert np.max(np.abs(from_padded(u, 16) - U0 * np.exp(-0.05 * 2 * 5e-2))) < 1e-15


KF_RBC = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))   # SSS_PENCIL's RBC default


def _dev(A, cuda, prec):
    """real coefficients (c, Nx, Ny, Nz) -> the padded layout on the device, as complex"""
    import torch
    c, Nx, Ny, Nz = A.shape
    t = torch.from_numpy(to_padded(A).view(np.float64).reshape(c, Nx, Ny, Nz // 2 + 1, 2))
    return torch.view_as_complex(t.to(torch.float64 if prec == "f64" else torch.float32).contiguous()).to(cuda)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((16, 16, 16), "reference"), ((32, 16, 32), "none"),
                                       ((32, 32, 16), "two_thirds"), ((16, 32, 16), "reference")])
def test_sss_rbc_step_matches_oracle(cuda, N, dealias, prec):
    """RBC on SSS (ts_rk4_step_rbc on an SSS plan; T = SCC, real coefficients) over 3 steps."""
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF_RBC, "SSS")
    rng = np.random.default_rng(6)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCC", "CSC", "CCS")])
    U0 = -0.3 * R.project_rhs(g, U)
    T0 = 0.3 * R.forward(g, rng.standard_normal(g.rshape), "SCC")
    cfg = R.RBCConfig(g, Ra=1e5, Pr=0.7, dt=1e-3, dealias_mode=mode)
    Uo, To = U0.copy(), T0.copy()
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan = tb.Plan(N, basis="SSS", kfactor=KF_RBC, precision=prec, nu=cfg.nu, kappa=cfg.kappa, dt=1e-3,
                   dealias=dealias, Ra=1e5, Pr=0.7)
    u = _dev(U0, cuda, prec)
    T = _dev(T0[None], cuda, prec)
    plan.rk4_step_rbc(u, T, 3)
    plan.status()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel(from_padded(u, N[2]), Uo) < tol
    assert rel(from_padded(T, N[2])[0], To) < tol


def test_sss_rbc_roll_follows_linear_theory(cuda):
    """One small roll (u_x, theta in sin(kx x) cos(ky y) cos(kz z)) with u_y balancing the
    divergence: (a, b) follow da/dt = (1 - kx^2/K^2) b - nu K^2 a, db/dt = a - kappa K^2 b."""
    from scipy.linalg import expm
    import tarang_b200 as tb
    N = (16, 16, 16)
    eps, nu, kappa, dt, n = 1e-9, 0.01, 0.02, 2e-3, 25
    g = R.Grid(N, KF_RBC, "SSS")
    U0 = np.zeros((3,) + g.shape)
    T0 = np.zeros((1,) + g.shape)
    kx, ky, kz = KF_RBC
    U0[0, 1, 1, 1] = eps
    U0[1, 1, 1, 1] = -kx * eps / ky
    T0[0, 1, 1, 1] = 0.5 * eps
    plan = tb.Plan(N, basis="SSS", kfactor=KF_RBC, nu=nu, kappa=kappa, dt=dt)
    u, T = _dev(U0, cuda, "f64"), _dev(T0, cuda, "f64")
    plan.rk4_step_rbc(u, T, n)
    K2 = kx * kx + ky * ky + kz * kz
    a, b = expm(np.array([[-nu * K2, 1 - kx * kx / K2], [1.0, -kappa * K2]]) * n * dt) @ np.array([eps, 0.5 * eps])
    assert abs(from_padded(u, N[2])[0, 1, 1, 1] - a) < 1e-7 * eps
    assert abs(from_padded(T, N[2])[0, 1, 1, 1] - b) < 1e-7 * eps


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_sss_energy_and_nusselt_match_oracle(cuda, prec):
    """ts_energy on real SSS coefficients (weights 4 / 2 / 1 / 1/2, padding skipped) and the
    Nusselt number on an SSS plan, against the oracle; the energy equals <u^2>/2 in real space."""
    import tarang_b200 as tb
    N = (16, 32, 16)
    g = R.Grid(N, KF_RBC, "SSS")
    rng = np.random.default_rng(8)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCC", "CSC", "CCS")])
    U = -0.3 * R.project_rhs(g, U)
    T = 0.3 * R.forward(g, rng.standard_normal(g.rshape), "SCC")
    cfg = R.RBCConfig(g, Ra=2e5, Pr=0.7, dt=1e-3)
    plan = tb.Plan(N, basis="SSS", kfactor=KF_RBC, precision=prec, nu=cfg.nu, kappa=cfg.kappa, Ra=2e5, Pr=0.7)
    u, t = _dev(U, cuda, prec), _dev(T[None], cuda, prec)
    Ur, Tr = from_padded(u, N[2]), from_padded(t, N[2])[0]   # the values the device holds
    tol = 1e-12 if prec == "f64" else 1e-6
    assert abs(plan.energy(u) / R.total_energy(g, Ur) - 1) < tol
    assert abs(plan.energy(t) / R.total_energy_scalar(g, Tr) - 1) < tol
    assert abs(plan.nusselt(u, t) - R.nusselt(cfg, Ur, Tr)) < tol * abs(R.nusselt(cfg, Ur, Tr))
    ur = R.inverse(g, Tr, "SCC")
    assert abs(plan.energy(t) / (0.5 * np.mean(ur ** 2)) - 1) < tol


def test_sss_max_div_and_padding(cuda):
    """ts_max_div on an SSS plan against the oracle (~0 after projection), and the two padding
    reals per line change neither the energy nor the divergence."""
    import torch
    import tarang_b200 as tb
    N = (16, 32, 16)
    g = R.Grid(N, KF, "SSS")
    rng = np.random.default_rng(13)
    V = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCC", "CSC", "CCS")])
    plan = tb.Plan(N, basis="SSS", kfactor=KF)
    v = _dev(V, cuda, "f64")
    d0, e0 = plan.max_div(v), plan.energy(v)
    assert abs(d0 / R.max_abs_div(g, V) - 1) < 1e-12
    w = _dev(-R.project_rhs(g, V), cuda, "f64")
    assert plan.max_div(w) < 1e-12 * d0
    vr = torch.view_as_real(v).reshape(3, N[0], N[1], N[2] + 2)
    vr[..., N[2]:] = 7.0
    assert plan.max_div(v) == d0 and plan.energy(v) == e0


@pytest.mark.parametrize("pr,us", [("PRLARGE", "USMALL"), ("PRSMALL", "ULARGE"), ("PRSMALL", "USMALL")])
def test_sss_rbc_scalings_match_oracle(cuda, pr, us):
    """RBC on SSS under the other Pr_option / Uscaling combinations, FP64 <= 1e-12 after 3 steps."""
    import tarang_b200 as tb
    N = (16, 16, 16)
    g = R.Grid(N, KF_RBC, "SSS")
    rng = np.random.default_rng(8)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCC", "CSC", "CCS")])
    U0 = -0.3 * R.project_rhs(g, U)
    T0 = 0.3 * R.forward(g, rng.standard_normal(g.rshape), "SCC")
    cfg = R.RBCConfig(g, Ra=3e4, Pr=0.7, dt=1e-5 if us == "USMALL" else 1e-3, dealias_mode=1, pr_option=pr,
                      uscaling=us)
    Uo, To = U0.copy(), T0.copy()
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan = tb.Plan(N, basis="SSS", kfactor=KF_RBC, precision="f64", nu=cfg.nu, kappa=cfg.kappa, dt=cfg.dt,
                   dealias="reference", Ra=3e4, Pr=0.7, Pr_option=pr, Uscaling=us)
    u = _dev(U0, cuda, "f64")
    T = _dev(T0[None], cuda, "f64")
    plan.rk4_step_rbc(u, T, 3)
    plan.status()
    assert rel(from_padded(u, N[2]), Uo) < 1e-12
    assert rel(from_padded(T, N[2])[0], To) < 1e-12


def _sss_state(g, seed, width):
    """a random solenoidal field with the SSS parities, energy at |K| <~ width, unit norm"""
    rng = np.random.default_rng(seed)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), R.SSS_PARITY[v]) for v in ("Vx", "Vy", "Vz")])
    U = -np.exp(-(g.Kmag() / width) ** 2) * R.project_rhs(g, U)
    return U / np.sqrt(np.sum(U ** 2))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((16, 16, 16), "reference"), ((32, 16, 32), "none"),
                                       ((32, 32, 16), "two_thirds")])
def test_sss_flux_matches_oracle(cuda, N, dealias, prec):
    """Pi(R) on SSS, the reference's per-sphere algorithm (EnergyTr::Compute_flux,
    compute_flux.cc:51-65, with SSS_PENCIL's sphere fill and outside sum over the real
    coefficients, SSS_pencil_ET.cc:50-70, 662-678) against the oracle's flux_per_sphere:
    FP64 to 1e-12, FP32 to 2e-6 of max|Pi|; radii in any order."""
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF, "SSS")
    U = _sss_state(g, 23, 10.0)
    radii = [7.0, 1.0, 3.5, 10.0, 14.0, 20.0]
    want = R.flux_per_sphere(g, U, radii, mode)
    assert np.max(np.abs(want)) > 0
    plan = tb.Plan(N, basis="SSS", precision=prec, kfactor=KF, dealias=dealias)
    got = plan.flux(_dev(U, cuda, prec), radii)
    tol = 1e-12 if prec == "f64" else 2e-6
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want)), (got, want)
    plan.close()


@pytest.mark.parametrize("dealias", ["reference", "two_thirds"])
def test_sss_dealias_field_matches_oracle(cuda, dealias):
    """ts_dealias_field on SSS real coefficients: the oracle's dealias, bit for bit."""
    import tarang_b200 as tb
    mode = {"reference": 1, "two_thirds": 2}[dealias]
    N = (32, 16, 32)
    g = R.Grid(N, KF, "SSS")
    U = _sss_state(g, 5, 40.0)
    plan = tb.Plan(N, basis="SSS", precision="f64", kfactor=KF, dealias=dealias)
    u = _dev(U, cuda, "f64")
    plan.dealias(u)
    assert np.array_equal(from_padded(u, N[2]), R.dealias(g, U, mode))
    plan.close()
