"""Parity at the benchmark's own sizes: one IF-RK4 step of the 256^3 forced workload (the
headline configuration: Carati supply on shell 3, eps = 0.1, nu = 1e-3, dt = 5e-4, two-thirds
dealiasing, IC k^4 exp(-2 (k/4)^2), E = 0.5, seed 0) and of 128^3 runs, GPU against the FP64
oracle.  Tolerances: FP64 relative L2 <= 1e-12, FP32 <= 1e-5 (the precision the FP32 path
is specified to), energy and max |div u| alongside.  The oracle step at 256^3 takes about
ten seconds per nonlinear form on the host's cores."""
import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _forcing(g):
    es = np.zeros(g.n_shells())
    es[3] = 0.1
    return es


@pytest.mark.parametrize("N", [128, 256])
def test_forced_step_matches_oracle_at_scale(cuda, N):
    import torch
    import tarang_b200 as tb
    g = R.Grid((N, N, N))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    es = _forcing(g)
    mis = g.modes_in_shell()
    for form in ("rotational", "conservative"):
        cfg = R.FluidConfig(g, nu=1e-3, dt=5e-4, dealias_mode=R.DEALIAS_TWO_THIRDS,
                            forcing=R.CaratiForcing(2.0, 3.0, es), nlin_form=form)
        ref = R.rk4_step(cfg, V, mis)
        E_ref = R.total_energy(g, ref)
        precs = ("f64", "f32") if (form == "rotational" or N == 128) else ("f64",)
        for prec in precs:
            plan = tb.Plan(N, precision=prec, nlin_form=form, dealias="two_thirds", nu=1e-3, dt=5e-4,
                           forcing=tb.Forcing(2.0, 3.0, es))
            u = torch.from_numpy(V).to(cuda).to(plan.torch_dtype())
            plan.rk4_step(u, 1)
            plan.status()
            got = u.cpu().numpy().astype(np.complex128)
            tol = 1e-12 if prec == "f64" else 1e-5
            assert rel(got, ref) < tol, (N, form, prec, rel(got, ref))
            assert abs(plan.energy(u) - E_ref) / E_ref < tol
            assert plan.max_div(u) < (1e-12 if prec == "f64" else 1e-5)
            plan.close()
            del u
            torch.cuda.empty_cache()


def test_adjoint_config_forward_step_matches_oracle_128(cuda):
    """The adjoint configuration's forward step (128^3, nu = 5e-3, dt = 1e-3, unforced,
    two-thirds, rotational), FP64 and FP32, against the oracle."""
    import torch
    import tarang_b200 as tb
    N = 128
    g = R.Grid((N, N, N))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=5e-3, dt=1e-3, dealias_mode=R.DEALIAS_TWO_THIRDS, nlin_form="rotational")
    ref = V
    for _ in range(2):
        ref = R.rk4_step(cfg, ref)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-5)):
        plan = tb.Plan(N, precision=prec, nlin_form="rotational", dealias="two_thirds", nu=5e-3, dt=1e-3)
        u = torch.from_numpy(V).to(cuda).to(plan.torch_dtype())
        plan.rk4_step(u, 2)
        plan.status()
        assert rel(u.cpu().numpy().astype(np.complex128), ref) < tol
        plan.close()
