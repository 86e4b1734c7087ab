"""Health reporting on the GPU, with the failures made on the host: a NaN written into a
state before a step (the device-side form of the reference's abort on a NaN total energy,
Ifluid_main.cc:127-129), and a bounded wait on an mbarrier that nothing completes (the
timeout path of every bulk-copy wait).  No test faults, traps or hangs the GPU."""
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu
KF = (math.pi, 2 * math.pi, 2 * math.pi)


def test_nan_in_state_is_reported_and_cleared(cuda):
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = tb.Plan(32, precision="f32", nlin_form="rotational", dealias="two_thirds", nu=1e-3, dt=5e-4)
    u = plan.field(3)
    plan.init_energy_spectrum(R.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    clean = u.clone()
    plan.rk4_step(u, 2)
    assert plan.status_code() == L.TS_OK
    u.copy_(clean)
    u[1, 3, 5, 2] = complex(float("nan"), 0.0)
    plan.rk4_step(u, 1)
    assert plan.status_code() == L.TS_ERR_NAN
    # the next stepping call reports it without stepping
    before = u.clone()
    with pytest.raises(L.TsError) as ei:
        plan.rk4_step(u, 1)
    assert ei.value.status == L.TS_ERR_NAN
    assert torch.equal(torch.isnan(u), torch.isnan(before))
    # a good state after clearing: steps again, and matches a fresh plan bit for bit
    plan.clear_status()
    u.copy_(clean)
    plan.rk4_step(u, 2)
    assert plan.status_code() == L.TS_OK
    p2 = tb.Plan(32, precision="f32", nlin_form="rotational", dealias="two_thirds", nu=1e-3, dt=5e-4)
    v = clean.clone()
    p2.rk4_step(v, 2)
    torch.cuda.synchronize()
    assert torch.equal(u, v)


def test_nan_in_rbc_temperature_is_reported(cuda):
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = tb.Plan(32, basis="SFF", precision="f64", kfactor=KF, Ra=1e5, Pr=1.0, dt=1e-3,
                   nu=math.sqrt(1 / 1e5), kappa=1 / math.sqrt(1e5))
    u, T = plan.field(3), plan.field(1)
    plan.init_temperature_perturbation(1e-3, 4.0, 3, T)
    T[0, 2, 1, 1] = complex(float("inf"), 0.0)
    plan.rk4_step_rbc(u, T, 1)
    assert plan.status_code() == L.TS_ERR_NAN
    plan.clear_status()
    assert plan.status_code() == L.TS_OK


def test_ensemble_flags_only_the_bad_member(cuda):
    """A NaN poked into one member's temperature before the run: only that member is flagged,
    and every other member's state is bit-identical to a clean run of the same ensemble."""
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    members = [(32, 1e5, 1.0), (32, 4e5, 1.0), (48, 3e5, 1.0), (16, 2e6, 1.0), (32, 1e6, 1.0)]
    bad = 1
    states = []
    for poison in (False, True):
        ens = tb.Ensemble(members, dt=1e-3, precision="f32")
        ens.init_temperature(1e-3, 4.0, 3)
        ens.synchronize()
        if poison:
            T = ens.view(bad, "T")
            T[0, 3, 2, 1] = complex(float("nan"), 0.0)
            torch.cuda.synchronize()
        ens.run(4)
        ens.synchronize()
        h = ens.health()
        if poison:
            assert h[bad] == L.TS_ERR_NAN
            assert all(h[m] == L.TS_OK for m in range(len(members)) if m != bad)
            # reported again until cleared on request
            assert ens.health(clear=True)[bad] == L.TS_ERR_NAN
            assert all(x == L.TS_OK for x in ens.health())
        else:
            assert all(x == L.TS_OK for x in h)
        states.append([(ens.view(m, "U").clone(), ens.view(m, "T").clone()) for m in range(len(members))])
        ens.close()
    for m in range(len(members)):
        if m == bad:
            assert not torch.isfinite(states[1][m][1]).all()
            continue
        assert torch.equal(states[0][m][0], states[1][m][0])
        assert torch.equal(states[0][m][1], states[1][m][1])


def test_bounded_wait_gives_up_and_the_context_stays_usable(cuda):
    """ts_plan_expire_wait: one block waits on an mbarrier nothing arrives on; the bounded wait
    gives up, sets the timeout bit, the kernel returns and the plan reports TS_ERR_TIMEOUT.
    After clearing, a step on the same plan matches the oracle."""
    import ctypes
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = tb.Plan(32, precision="f64", nu=1e-3, dt=5e-4, dealias="reference")
    L.check(plan.lib.ts_plan_expire_wait(plan.h, 1 << 14), "ts_plan_expire_wait")
    assert plan.status_code() == L.TS_ERR_TIMEOUT
    u = plan.field(3)
    with pytest.raises(L.TsError) as ei:
        plan.rk4_step(u, 1)
    assert ei.value.status == L.TS_ERR_TIMEOUT
    plan.clear_status()
    g = R.Grid((32, 32, 32))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    u = torch.from_numpy(V.copy()).to(cuda)
    plan.rk4_step(u, 1)
    assert plan.status_code() == L.TS_OK
    ref = R.rk4_step(R.FluidConfig(g, nu=1e-3, dt=5e-4, dealias_mode=1), V)
    got = u.cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    assert plan.lib.ts_plan_expire_wait(plan.h, 0) == L.TS_ERR_ARG
