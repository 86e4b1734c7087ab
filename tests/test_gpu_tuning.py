"""Launch tuning: every kernel candidate of every pass class computes the step
the oracle computes (FP64 oracle; FP32 candidates within relative L2 1e-5,
FP64 within 1e-11), the autotuner keeps the caller's fields and an ensemble's
states, and its cache round-trips."""
import json
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu

KF = (math.pi, 2 * math.pi, 2 * math.pi)
TOL = {"f32": 1e-5, "f64": 1e-11}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def tunings(plan):
    """(class index, variant, blocks) for every non-rule candidate of the plan, one class at a time"""
    out = []
    for c, (name, cand) in enumerate(plan.tuning_candidates().items()):
        for v in cand["variants"]:
            if v:
                out.append((c, v, 0))
        if cand["blocks"]:
            out += [(c, 0, 1), (c, 0, 3)]
    return out


def with_class(c, v, b):
    t = {"variant": [0] * 5, "blocks_per_sm": [0] * 5}
    t["variant"][c] = v
    t["blocks_per_sm"][c] = b
    return t


FFF_CASES = [
    ((256, 64, 32), "f32", "rotational", "two_thirds"),
    ((32, 256, 256), "f32", "rotational", "two_thirds"),
    ((32, 32, 1024), "f32", "rotational", "two_thirds"),
    ((1024, 16, 32), "f32", "conservative", "reference"),
    ((1024, 32, 32), "f32", "rotational", "two_thirds"),
    ((32, 1024, 32), "f32", "rotational", "two_thirds"),
    ((64, 64, 64), "f64", "conservative", "reference"),
    ((32, 128, 64), "f64", "rotational", "two_thirds"),
]


@pytest.mark.parametrize("N,prec,form,dealias", FFF_CASES)
def test_fff_candidates_match_oracle(cuda, N, prec, form, dealias):
    import torch
    import tarang_b200 as tb
    mode = {"reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=mode, nlin_form=form)
    W = V.copy()
    for _ in range(2):
        W = R.rk4_step(cfg, W)
    plan = tb.Plan(N, precision=prec, nu=0.01, dt=1e-3, dealias=dealias, nlin_form=form)
    cases = tunings(plan)
    assert cases, "every geometry has candidates"
    u0 = torch.from_numpy(V.astype(np.complex128 if prec == "f64" else np.complex64)).to(cuda)
    errs = {}
    for c, v, b in [(0, 0, 0)] + cases:
        plan.set_tuning(with_class(c, v, b))
        u = u0.clone()
        plan.rk4_step(u, 2)
        plan.status()
        errs[(c, v, b)] = rel(u.cpu().numpy(), W)
    bad = {k: e for k, e in errs.items() if not e < TOL[prec]}
    assert not bad, bad


SFF_CASES = [((64, 64, 32), "f32", "two_thirds"), ((48, 48, 48), "f32", "reference"),
             ((32, 32, 32), "f64", "reference"), ((128, 32, 16), "f32", "reference"),
             ((96, 48, 48), "f64", "reference")]


@pytest.mark.parametrize("N,prec,dealias", SFF_CASES)
def test_sff_candidates_match_oracle(cuda, N, prec, dealias):
    import torch
    import tarang_b200 as tb
    mode = {"reference": 1, "two_thirds": 2}[dealias]
    g = R.Grid(N, KF, "SFF")
    rng = np.random.default_rng(5)
    par = ["S", "C", "C"]
    U0 = np.stack([R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), par[i])) for i in range(3)])
    T0 = R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), "S"))
    cfg = R.RBCConfig(g, Ra=1e5, Pr=1.0, dt=1e-3, dealias_mode=mode)
    Uo, To = U0.copy(), T0.copy()
    for _ in range(2):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    plan = tb.Plan(N, basis="SFF", precision=prec, kfactor=KF, dealias=dealias, nu=cfg.nu, kappa=cfg.kappa,
                   dt=1e-3, Ra=1e5, Pr=1.0)
    cases = tunings(plan)
    assert cases
    cdt = np.complex128 if prec == "f64" else np.complex64
    errs = {}
    for c, v, b in [(0, 0, 0)] + cases:
        plan.set_tuning(with_class(c, v, b))
        u = torch.from_numpy(U0.astype(cdt)).to(cuda)
        T = torch.from_numpy(T0.astype(cdt)).to(cuda)
        plan.rk4_step_rbc(u, T, 2)
        plan.status()
        errs[(c, v, b)] = max(rel(u.cpu().numpy(), Uo), rel(T.cpu().numpy(), To))
    bad = {k: e for k, e in errs.items() if not e < TOL[prec]}
    assert not bad, bad


def test_set_tuning_rejects_missing_candidates(cuda):
    import tarang_b200 as tb
    plan = tb.Plan(64, precision="f32", nlin_form="rotational", dealias="two_thirds")
    cand = plan.tuning_candidates()
    assert not cand["z"]["blocks"] and cand["y_inv"]["blocks"]
    with pytest.raises(tb.TsError):
        plan.set_tuning(with_class(2, 0, 2))  # z takes no blocks-per-SM count
    with pytest.raises(tb.TsError):
        plan.set_tuning(with_class(0, 7, 0))
    # the FFF inverse x pass has four candidates in FP32 (3: the prefetching kernel), none at 4
    assert 3 in cand["x_inv"]["variants"] and 4 not in cand["x_inv"]["variants"]
    with pytest.raises(tb.TsError):
        plan.set_tuning(with_class(0, 4, 0))
    assert plan.tuning() == {"variant": [0] * 5, "blocks_per_sm": [0] * 5}


def test_plan_autotune_keeps_fields_and_caches(cuda, tmp_path):
    import torch
    import tarang_b200 as tb
    N = 64
    g = R.Grid((N, N, N))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=2, nlin_form="rotational")
    W = R.rk4_step(cfg, V.copy())
    plan = tb.Plan(N, precision="f32", nu=0.01, dt=1e-3, dealias="two_thirds", nlin_form="rotational")
    u = torch.from_numpy(V.astype(np.complex64)).to(cuda)
    before = u.clone()
    cache = str(tmp_path / "tuning.json")
    rep = plan.autotune(reps=2, cache=cache)
    assert torch.equal(u, before)
    for name in ("x_inv", "y_inv", "z", "y_fwd", "x_fwd"):
        assert rep[name]["tried"] and rep[name]["variant"] >= 0
    t = plan.tuning()
    assert rep["tuning"] == t == rep["final"]
    assert rep["confirm"]["kept"] in ("tuned", "rule")
    if rep["confirm"]["kept"] == "rule":
        assert t == {"variant": [0] * 5, "blocks_per_sm": [0] * 5}
    plan.rk4_step(u, 1)
    assert rel(u.cpu().numpy(), W) < 1e-5
    # a second plan of the same configuration takes the stored tuning without timing
    other = tb.Plan(N, precision="f32", nu=0.01, dt=1e-3, dealias="two_thirds", nlin_form="rotational")
    hit = other.autotune(cache=cache)
    assert hit["cached"] and other.tuning() == t
    assert json.load(open(cache))[plan.tuning_key()] == t


def test_ensemble_autotune_keeps_states(cuda):
    import tarang_b200 as tb
    members = [(32, 1e5, 1.0), (48, 1e6, 1.0), (32, 3e5, 1.0)]
    ens = tb.Ensemble(members, dt=1e-4, precision="f32")
    ens.init_temperature(1e-3, 4.0, 3)
    ens.run(2)
    e_before = [ens.energy(m) for m in range(3)]
    rep = ens.autotune(reps=1)
    assert len(rep["groups"]) == 2
    # the graph schedule of the size groups is chosen by timing both
    assert rep["schedule"] in ("parallel", "serial") and rep["parallel_ms"] > 0 and rep["serial_ms"] > 0
    assert [ens.energy(m) for m in range(3)] == e_before
    # tuned and untuned ensembles agree to FP32 rounding
    ref = tb.Ensemble(members, dt=1e-4, precision="f32")
    ref.init_temperature(1e-3, 4.0, 3)
    ref.run(2)
    ens.run(5)
    ref.run(5)
    for m in range(3):
        assert abs(ens.energy(m) - ref.energy(m)) <= 1e-5 * ref.energy(m)
    assert np.allclose(ens.nusselt(), ref.nusselt(), rtol=1e-5, atol=0)
    for k, grp in enumerate(rep["groups"]):
        m = 0 if grp["N"][0] == 32 else 1
        assert ens.tuning(m) == grp["tuning"]["final"]
