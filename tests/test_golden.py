"""Golden fixtures (tests/golden/fff16_forced_step.npz): the oracle reproduces them on CPU and
the CUDA path matches them on the GPU (FP64, relative L2 <= 1e-12)."""
import os

import numpy as np
import pytest

from oracle import tarang_ref as R

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load():
    return dict(np.load(os.path.join(HERE, "fff16_forced_step.npz")))


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_oracle_reproduces_golden():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    got = mg.compute()
    ref = load()
    for k in ("V0", "V1", "Ek1", "Pi1"):
        assert rel(got[k], ref[k]) < 1e-14, k


@pytest.mark.gpu
def test_cuda_matches_golden(cuda):
    import torch
    import tarang_b200 as tb
    ref = load()
    plan = tb.Plan(16, precision="f64", nu=0.01, dt=1e-3, dealias="reference",
                   forcing=tb.Forcing(2.0, 3.0, ref["energy_supply"]))
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    assert rel(u.cpu().numpy(), ref["V0"]) < 1e-13
    plan.rk4_step(u, 1)
    torch.cuda.synchronize()
    assert rel(u.cpu().numpy(), ref["V1"]) < 1e-12
    assert rel(plan.shell_spectrum(u), ref["Ek1"]) < 1e-12
    assert np.max(np.abs(plan.flux(u, ref["radii"]) - ref["Pi1"])) < 1e-12 * np.max(np.abs(ref["Pi1"]))
