"""GPU discrete adjoint of the rotational IF-RK4 step, through the C ABI.

Tolerances: FP64 adjoint vs the FP64 oracle transpose, relative L2 <= 1e-11;
gradient vs central finite differences (eps = 1e-6, FP64) relative <= 1e-6;
FP32 adjoint vs FP64 adjoint, relative L2 <= 1e-4.
"""
import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def np_(t):
    return t.detach().cpu().numpy()


def setup(N, prec="f64", nu=0.01, dt=1e-2, reality=True):
    import tarang_b200 as tb
    g = R.Grid((N, N, N) if isinstance(N, int) else N)
    cfg = R.FluidConfig(g, nu=nu, dt=dt, dealias_mode=2, nlin_form="rotational", reality_fix=reality)
    plan = tb.Plan(N, precision=prec, nu=nu, dt=dt, dealias="two_thirds", nlin_form="rotational",
                   reality_fix=reality)
    return g, cfg, plan


@pytest.mark.parametrize("reality", [True, False])
@pytest.mark.parametrize("N", [32, (32, 16, 64), (512, 16, 32)])
def test_adjoint_step_matches_oracle(cuda, N, reality):
    import torch
    g, cfg, plan = setup(N, reality=reality)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    rng = np.random.default_rng(5)
    Lam = rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
    u = torch.from_numpy(V.copy()).to(cuda)
    un = torch.empty_like(u)
    st = torch.empty((9,) + g.shape, dtype=u.dtype, device=cuda)
    plan.rk4_step_keep(u, un, st)
    lam = torch.from_numpy(Lam.copy()).to(cuda)
    plan.adjoint_step(u, st, lam)
    torch.cuda.synchronize()
    # the kept stage fields and the new state are the forward step's
    S = R.rk4_stages(cfg, V)
    for i in range(3):
        assert rel(np_(st[3 * i:3 * i + 3]), S[i + 1]) < 1e-12
    assert rel(np_(un), R.rk4_step(cfg, V)) < 1e-12
    assert rel(np_(u), V) == 0.0
    assert rel(np_(lam), R.rk4_step_adjoint(cfg, V, Lam)) < 1e-11


def test_adjoint_window_matches_composed_steps(cuda):
    import torch
    g, cfg, plan = setup(32)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    rng = np.random.default_rng(9)
    Lam = rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
    n = 3
    states = [V]
    for _ in range(n - 1):
        states.append(R.rk4_step(cfg, states[-1]))
    ref = Lam.copy()
    for k in reversed(range(n)):
        ref = R.rk4_step_adjoint(cfg, states[k], ref)
    u = torch.from_numpy(V.copy()).to(cuda)
    lam = torch.from_numpy(Lam.copy()).to(cuda)
    work = torch.empty(plan.adjoint_work_bytes(n), dtype=torch.uint8, device=cuda)
    plan.adjoint_window(u, n, lam, work)
    torch.cuda.synchronize()
    assert rel(np_(lam), ref) < 1e-11
    assert rel(np_(u), V) == 0.0


def test_adjoint_rejects_unsupported(cuda):
    import torch
    import tarang_b200 as tb
    plan = tb.Plan(32, nlin_form="conservative")
    u = plan.field(3)
    st = torch.empty((9,) + plan.spec_shape, dtype=u.dtype, device=cuda)
    with pytest.raises(tb.TsError):
        plan.adjoint_step(u, st, u.clone())
    p2 = tb.Plan(32, nlin_form="rotational")
    work = torch.empty(p2.adjoint_work_bytes(2) - 16, dtype=torch.uint8, device=cuda)
    with pytest.raises(tb.TsError):
        p2.adjoint_window(u, 2, u.clone(), work)


def _fd_check(plan, u0, target, dirs, nsteps, window, eps):
    """gradient from autograd vs central differences of J along each direction; returns max rel err."""
    import torch
    import tarang_b200 as tb
    x = u0.clone().requires_grad_(True)
    J = tb.energy_norm_loss(tb.rk4_evolve(x, plan, nsteps, window), target)
    J.backward()
    plan.status()
    G = x.grad.detach()
    errs = []
    for v in dirs:
        def Jat(s):
            u = (u0 + s * v).contiguous()
            plan.rk4_step(u, nsteps)
            plan.status()
            return float(tb.energy_norm_loss(u, target))
        fd = (Jat(eps) - Jat(-eps)) / (2 * eps)
        ad = float(torch.sum((G * torch.conj(v)).real))
        errs.append((abs(fd - ad) / max(abs(fd), 1e-30), fd, ad))
    return errs, G


def test_gradient_matches_finite_differences_small(cuda):
    import torch
    import tarang_b200 as tb
    plan = tb.Plan(32, precision="f64", nu=0.01, dt=1e-2, dealias="two_thirds", nlin_form="rotational")
    u0, tgt = plan.field(3), plan.field(3)
    sp = tb.spectrum_k4_gauss(plan.n_shells, 4.0)
    plan.init_energy_spectrum(sp, 0, 0.5, u0)
    plan.init_energy_spectrum(sp, 1, 0.5, tgt)
    dirs = [plan.init_energy_spectrum(sp, 100 + i, 0.5, plan.field(3)) for i in range(3)]
    errs, _ = _fd_check(plan, u0, tgt, dirs, nsteps=10, window=4, eps=1e-6)
    assert max(e[0] for e in errs) < 1e-6, errs


def test_adjoint_config4_128(cuda):
    """128^3, nu = 5e-3, dt = 1e-3, 200 steps, checkpoints every 20; J = 1/2 ||u(T) - u_target||^2;
    gradient vs central differences along 8 seeded solenoidal directions (eps = 1e-6, FP64), and the
    FP32 adjoint against the FP64 one."""
    import torch
    import tarang_b200 as tb
    p64 = tb.Plan(128, precision="f64", nu=5e-3, dt=1e-3, dealias="two_thirds", nlin_form="rotational")
    sp = tb.spectrum_k4_gauss(p64.n_shells, 4.0)
    u0, tgt = p64.field(3), p64.field(3)
    p64.init_energy_spectrum(sp, 0, 0.5, u0)
    p64.init_energy_spectrum(sp, 1, 0.5, tgt)
    dirs = [p64.init_energy_spectrum(sp, 1000 + i, 0.5, p64.field(3)) for i in range(8)]
    errs, G64 = _fd_check(p64, u0, tgt, dirs, nsteps=200, window=20, eps=1e-6)
    assert max(e[0] for e in errs) < 1e-6, errs
    p32 = tb.Plan(128, precision="f32", nu=5e-3, dt=1e-3, dealias="two_thirds", nlin_form="rotational")
    x = u0.to(torch.complex64).requires_grad_(True)
    tb.energy_norm_loss(tb.rk4_evolve(x, p32, 200, 20), tgt.to(torch.complex64)).backward()
    assert rel(np_(x.grad).astype(np.complex128), np_(G64)) < 1e-4


@pytest.mark.parametrize("N", [(16, 32, 1024), (1024, 16, 32)])
def test_adjoint_step_f32_long_axes(cuda, N):
    """FP32 adjoint on 1024-point axes (two-warp z lines, split x pass) against the FP64 oracle."""
    import torch
    g, cfg, _ = setup(N)
    _, _, plan = setup(N, prec="f32")
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    rng = np.random.default_rng(11)
    Lam = rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
    u = torch.from_numpy(V.copy()).to(cuda).to(torch.complex64)
    st = torch.empty((9,) + g.shape, dtype=u.dtype, device=cuda)
    plan.rk4_step_keep(u, torch.empty_like(u), st)
    lam = torch.from_numpy(Lam.copy()).to(cuda).to(torch.complex64)
    plan.adjoint_step(u, st, lam)
    torch.cuda.synchronize()
    assert rel(np_(lam).astype(np.complex128), R.rk4_step_adjoint(cfg, V, Lam)) < 1e-4
