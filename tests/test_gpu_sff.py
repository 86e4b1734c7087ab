"""GPU parity of the SFF / Boussinesq (RBC) path against the FP64 oracle, through the C ABI.

Tolerance: FP64 path relative L2 <= 1e-12 after 3 steps; FP32 path vs the FP64
path relative L2 <= 1e-5.
"""
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu

KF = (math.pi, 2 * math.pi, 2 * math.pi)


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def random_state(g, amp, seed):
    """Random fields with the SFF parities (u1 S, u2 C, u3 C, T S), reality-fixed."""
    rng = np.random.default_rng(seed)
    par = ["S", "C", "C"]
    U = np.stack([R.reality_fix(g, amp * R.forward(g, rng.standard_normal(g.rshape), par[i])) for i in range(3)])
    T = R.reality_fix(g, amp * R.forward(g, rng.standard_normal(g.rshape), "S"))
    return U, T


@pytest.mark.parametrize("N,dealias", [((16, 16, 16), "reference"), ((32, 16, 32), "two_thirds"), ((32, 32, 32), "reference")])
def test_rbc_step_matches_oracle_f64(cuda, N, dealias):
    import torch
    import tarang_b200 as tb
    mode = {"reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF, "SFF")
    U0, T0 = random_state(g, 0.3, 5)
    cfg = R.RBCConfig(g, Ra=1e5, Pr=1.0, dt=1e-3, dealias_mode=mode)
    plan = tb.Plan(N, basis="SFF", kfactor=KF, dealias=dealias, nu=cfg.nu, kappa=cfg.kappa, dt=1e-3,
                   Ra=1e5, Pr=1.0)
    u = torch.from_numpy(U0.copy()).to(cuda)
    T = torch.from_numpy(T0.copy()).to(cuda)
    Uo, To = U0.copy(), T0.copy()
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan.rk4_step_rbc(u, T, 3)
    torch.cuda.synchronize()
    assert rel(u.cpu().numpy(), Uo) < 1e-12
    assert rel(T.cpu().numpy(), To) < 1e-12
    assert abs(plan.nusselt(u, T) - R.nusselt(cfg, Uo, To)) < 1e-12
    assert abs(plan.energy(u) - R.total_energy(g, Uo)) < 1e-13 * R.total_energy(g, Uo)


def test_rbc_temperature_ic_matches_oracle(cuda):
    import tarang_b200 as tb
    g = R.Grid((32, 32, 32), KF, "SFF")
    plan = tb.Plan((32, 32, 32), basis="SFF", kfactor=KF)
    T = plan.field(1)
    plan.init_temperature_perturbation(1e-3, 4.0, 3, T)
    assert rel(T[0].cpu().numpy(), R.rbc_temperature_ic(g, 1e-3, 4.0, 3)) < 1e-14


def test_rbc_f32_vs_f64(cuda):
    import torch
    import tarang_b200 as tb
    N = (32, 32, 32)
    g = R.Grid(N, KF, "SFF")
    U0, T0 = random_state(g, 0.3, 9)
    kw = dict(basis="SFF", kfactor=KF, dealias="two_thirds", nu=math.sqrt(1 / 1e5), kappa=1 / math.sqrt(1e5),
              dt=1e-3, Ra=1e5, Pr=1.0)
    p64 = tb.Plan(N, precision="f64", **kw)
    p32 = tb.Plan(N, precision="f32", **kw)
    u64 = torch.from_numpy(U0.copy()).to(cuda)
    t64 = torch.from_numpy(T0.copy()).to(cuda)
    u32, t32 = u64.to(torch.complex64), t64.to(torch.complex64)
    for _ in range(5):
        p64.rk4_step_rbc(u64, t64, 1)
        p32.rk4_step_rbc(u32, t32, 1)
    torch.cuda.synchronize()
    assert rel(u32.to(torch.complex128).cpu().numpy(), u64.cpu().numpy()) < 1e-5
    assert rel(t32.to(torch.complex128).cpu().numpy(), t64.cpu().numpy()) < 1e-5


def test_rbc_linear_growth_above_critical(cuda):
    """Ra = 1e5 (above the free-slip onset ~3044 for this box) amplifies a small perturbation."""
    import torch
    import tarang_b200 as tb
    N = (16, 16, 16)
    plan = tb.Plan(N, basis="SFF", kfactor=KF, nu=math.sqrt(1 / 1e5), kappa=1 / math.sqrt(1e5), dt=2e-2,
                   Ra=1e5, Pr=1.0)
    u = plan.field(3)
    T = plan.field(1)
    plan.init_temperature_perturbation(1e-6, 1.5, 3, T)
    e0 = plan.energy(T)
    plan.rk4_step_rbc(u, T, 60)
    torch.cuda.synchronize()
    assert plan.energy(T) / e0 > 1.1


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("parity", ["SFF", "CFF"])
@pytest.mark.parametrize("N", [(16, 16, 16), (32, 16, 64), (64, 32, 16), (48, 16, 16)])
def test_sff_transforms_match_oracle(cuda, N, parity, prec):
    """SFF_PENCIL::Forward/Inverse_transform through ts_fft_forward / ts_fft_inverse (x parity S or C)."""
    import torch
    import tarang_b200 as tb
    g = R.Grid(N, KF, "SFF")
    plan = tb.Plan(N, basis="SFF", kfactor=KF, precision=prec)
    rng = np.random.default_rng(2)
    u = rng.standard_normal((2,) + N)
    rdt = torch.float64 if prec == "f64" else torch.float32
    real = torch.zeros((2, N[0], N[1], N[2] + 2), dtype=rdt, device=cuda)
    real[..., : N[2]] = torch.from_numpy(u).to(rdt)
    spec = plan.field(2)
    plan.forward(real, spec, parity=parity)
    torch.cuda.synchronize()
    par = parity[0]
    ref = np.stack([R.forward(g, u[i], par) for i in range(2)])
    tol = 1e-13 if prec == "f64" else 2e-6
    assert rel(spec.cpu().numpy(), ref) < tol
    back = torch.zeros_like(real)
    plan.inverse(spec, back, parity=parity)
    torch.cuda.synchronize()
    ub = back.cpu().numpy()
    assert rel(ub[..., : N[2]], np.stack([R.inverse(g, ref[i], par) for i in range(2)])) < tol
    assert np.all(ub[..., N[2]:] == 0)
    # the input of the inverse is not modified
    assert rel(spec.cpu().numpy(), ref) < tol


def test_sff_transform_rejects_wrong_parity(cuda):
    import torch
    import tarang_b200 as tb
    plan = tb.Plan((16, 16, 16), basis="SFF", kfactor=KF)
    real = torch.zeros((1, 16, 16, 18), dtype=torch.float64, device=cuda)
    with pytest.raises(tb.TsError):
        plan.forward(real, plan.field(1), parity="FFF")


SCALINGS = [("PRLARGE", "USMALL"), ("PRSMALL", "ULARGE"), ("PRSMALL", "USMALL")]


@pytest.mark.parametrize("pr,us", SCALINGS)
@pytest.mark.parametrize("basis", ["SFF", "SSF"])
def test_rbc_scalings_match_oracle(cuda, basis, pr, us):
    """The other Pr_option / Uscaling combinations: buoyancy coefficients (compute_force_RBC.cc:
    104-150), nu and kappa (Iscalar_main.cc:52-92) and the Nusselt factors (Correlation.cc:
    144-176) against the oracle: FP64 <= 1e-12 after 3 steps, FP32 <= 1e-5, Nusselt to 1e-12."""
    import torch
    import tarang_b200 as tb
    from tarang_b200.solver import rbc_diss_coefficients
    N = (16, 16, 16)
    kf = KF if basis == "SFF" else (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    g = R.Grid(N, kf, basis)
    Ra, Pr = 3e4, 0.7
    cfg = R.RBCConfig(g, Ra=Ra, Pr=Pr, dt=1e-5 if us == "USMALL" else 1e-3, dealias_mode=1, pr_option=pr,
                      uscaling=us)
    if basis == "SFF":
        U0, T0 = random_state(g, 0.3, 7)
    else:
        rng = np.random.default_rng(7)
        f = [0.3 * R.forward(g, rng.standard_normal(g.rshape), p) for p in ("SCF", "CSF", "CCF", "SCF")]
        U0, T0 = np.stack(f[:3]), f[3]
    Uo, To = U0, T0
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    nu, kappa = rbc_diss_coefficients(pr, us, Ra, Pr)
    assert (nu, kappa) == (cfg.nu, cfg.kappa)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-5)):
        plan = tb.Plan(N, basis=basis, precision=prec, kfactor=kf, dealias="reference", nu=nu, kappa=kappa,
                       dt=cfg.dt, Ra=Ra, Pr=Pr, Pr_option=pr, Uscaling=us)
        u = torch.from_numpy(np.ascontiguousarray(U0)).to(cuda).to(plan.torch_dtype())
        T = torch.from_numpy(np.ascontiguousarray(T0)[None]).to(cuda).to(plan.torch_dtype())
        plan.rk4_step_rbc(u, T, 3)
        plan.status()
        assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
        assert rel(T[0].cpu().numpy().astype(np.complex128), To) < tol
        if prec == "f64" and basis == "SFF":
            ref = R.nusselt(cfg, Uo, To)
            assert abs(plan.nusselt(u, T) - ref) < 1e-12 * max(1.0, abs(ref))
        plan.close()


@pytest.mark.parametrize("pr,us", [("PRZERO", "USMALL"), ("PRZERO", "ULARGE"), ("PRINFTY", "USMALL"),
                                   ("PRINFTY", "ULARGE")])
def test_rbc_slaved_scalings_match_oracle(cuda, pr, us):
    """PRZERO (T = U.V1 / K^2 after every stage) and PRINFTY (U = vs P(T x) / K^2) on SFF
    against the oracle (rbc_rk4_step_slaved): the slaved initial field of ts_rbc_slave, then
    3 steps, FP64 <= 1e-12 and FP32 <= 1e-5 in both fields, and the Nusselt number."""
    import torch
    import tarang_b200 as tb
    from tarang_b200.solver import rbc_diss_coefficients
    N = (16, 16, 16)
    g = R.Grid(N, KF, "SFF")
    Ra, Pr = 3e4, 0.7
    cfg = R.RBCConfig(g, Ra=Ra, Pr=Pr, dt=1e-5 if us == "USMALL" else 1e-3, dealias_mode=1, pr_option=pr,
                      uscaling=us)
    co = cfg.coeffs
    U0, T0 = random_state(g, 0.3, 11)
    if pr == "PRZERO":
        T0 = R.rbc_slave_temperature(g, U0)
    else:
        U0 = R.rbc_slave_velocity(g, T0, co["vs"])
    Uo, To = U0, T0
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    nu, kappa = rbc_diss_coefficients(pr, us, Ra, Pr)
    assert (nu, kappa) == (cfg.nu, cfg.kappa)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-5)):
        plan = tb.Plan(N, basis="SFF", precision=prec, kfactor=KF, dealias="reference", nu=nu, kappa=kappa,
                       dt=cfg.dt, Ra=Ra, Pr=Pr, Pr_option=pr, Uscaling=us)
        u = torch.from_numpy(np.ascontiguousarray(U0)).to(cuda).to(plan.torch_dtype())
        T = torch.from_numpy(np.ascontiguousarray(T0)[None]).to(cuda).to(plan.torch_dtype())
        # the slaved field as the reference sets it after an initial condition
        if pr == "PRZERO":
            T.zero_()
        else:
            u.zero_()
        plan.rbc_slave(u, T)
        assert rel(u.cpu().numpy().astype(np.complex128), U0) < tol
        assert rel(T[0].cpu().numpy().astype(np.complex128), T0) < tol
        plan.rk4_step_rbc(u, T, 3)
        plan.status()
        assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
        assert rel(T[0].cpu().numpy().astype(np.complex128), To) < tol
        if prec == "f64":
            ref = R.nusselt(cfg, Uo, To)
            assert abs(plan.nusselt(u, T) - ref) < 1e-12 * max(1.0, abs(ref))
        plan.close()


def test_rbc_slaved_scalings_refused_off_sff(cuda):
    """PRZERO / PRINFTY step on SFF only: an SSF plan refuses the step, an ensemble refuses
    the members, and ts_rbc_slave refuses the non-slaved scalings."""
    import torch
    import tarang_b200 as tb
    plan = tb.Plan((16, 16, 16), basis="SSF", kfactor=KF, Pr_option="PRZERO", Uscaling="USMALL", nu=1.0,
                   kappa=0.0)
    u = plan.field(3)
    T = plan.field(1)
    with pytest.raises(tb.TsError):
        plan.rk4_step_rbc(u, T, 1)
    plan.close()
    plan = tb.Plan((16, 16, 16), basis="SFF", kfactor=KF)
    u = plan.field(3)
    T = plan.field(1)
    with pytest.raises(tb.TsError):
        plan.rbc_slave(u, T)
    plan.close()
    for pr in ("PRZERO", "PRINFTY"):
        with pytest.raises(tb.TsError):
            tb.Ensemble([((16, 16, 16), 1e4, 1.0)], dt=1e-4, Pr_option=pr, Uscaling="USMALL")

@pytest.mark.parametrize("dealias", ["reference", "two_thirds"])
def test_rbc_two_dimensional_matches_oracle(cuda, dealias):
    """A two-dimensional RBC run (Ny = 1, program.two_dimension; the reference's RBC/2d and
    RBC_scaling/2d inputs are 32 x 1 x 32 on SFF): the y transforms are the identity and
    u2 stays zero. FP64 <= 1e-12 and FP32 <= 1e-5 against the oracle after 3 steps, and
    the Nusselt number."""
    import torch
    import tarang_b200 as tb
    mode = {"reference": 1, "two_thirds": 2}[dealias]
    N = (32, 1, 32)
    g = R.Grid(N, KF, "SFF")
    U0, T0 = random_state(g, 0.3, 9)
    U0[1] = 0
    cfg = R.RBCConfig(g, Ra=1e5, Pr=1.0, dt=1e-3, dealias_mode=mode)
    Uo, To = U0, T0
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    assert np.abs(Uo[1]).max() == 0.0
    for prec, tol in (("f64", 1e-12), ("f32", 1e-5)):
        plan = tb.Plan(N, basis="SFF", precision=prec, kfactor=KF, dealias=dealias, nu=cfg.nu, kappa=cfg.kappa,
                       dt=cfg.dt, Ra=cfg.Ra, Pr=cfg.Pr)
        u = torch.from_numpy(np.ascontiguousarray(U0)).to(cuda).to(plan.torch_dtype())
        T = torch.from_numpy(np.ascontiguousarray(T0)[None]).to(cuda).to(plan.torch_dtype())
        plan.rk4_step_rbc(u, T, 3)
        plan.status()
        assert rel(u.cpu().numpy().astype(np.complex128), Uo) < tol
        assert rel(T[0].cpu().numpy().astype(np.complex128), To) < tol
        assert float(u[1].abs().max()) == 0.0
        if prec == "f64":
            ref = R.nusselt(cfg, Uo, To)
            assert abs(plan.nusselt(u, T) - ref) < 1e-12 * max(1.0, abs(ref))
        plan.close()


def test_two_dimensional_refused_off_sff(cuda):
    """Ny = 1 is taken on SFF plans only."""
    import tarang_b200 as tb
    for basis in ("FFF", "SSF", "SSS"):
        with pytest.raises(tb.TsError):
            tb.Plan((32, 1, 32), basis=basis)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,dealias", [((16, 32, 16), "reference"), ((32, 16, 16), "none"),
                                       ((32, 32, 32), "two_thirds"), ((32, 1, 32), "reference")])
def test_sff_flux_matches_oracle(cuda, N, dealias, prec):
    """Pi(R) of the velocity on SFF, the reference's per-sphere algorithm (EnergyTr::Compute_flux,
    compute_flux.cc:51-65: one giver nonlinear term per sphere, summed outside it; the
    reference's RBC runs are on this basis) against the oracle's flux_per_sphere, in three
    dimensions and in two (Ny = 1): FP64 to 1e-12, FP32 to 2e-6 of max|Pi|; the radii
    in any order."""
    import torch
    import tarang_b200 as tb
    mode = {"none": 0, "reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF, "SFF")
    U, _ = random_state(g, 3.0, 17)
    if N[1] == 1:
        U[1] = 0
    U = -np.exp(-(g.Kmag() / 6.0) ** 2) * R.project_rhs(g, U)  # solenoidal, energy at |K| <~ 6
    U /= np.sqrt(np.sum(np.abs(U) ** 2))
    radii = [7.0, 1.0, 3.5, 8.0, 10.0, 14.0]
    want = R.flux_per_sphere(g, U, radii, mode)
    assert np.max(np.abs(want)) > 0
    plan = tb.Plan(N, basis="SFF", precision=prec, kfactor=KF, dealias=dealias, Ra=1e4, Pr=1.0, dt=1e-4)
    u = torch.from_numpy(np.ascontiguousarray(U)).to(cuda).to(plan.torch_dtype())
    got = plan.flux(u, radii)
    tol = 1e-12 if prec == "f64" else 2e-6
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want)), (got, want)
    plan.close()
