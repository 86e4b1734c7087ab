"""Regenerate the golden fixtures of tests/golden from the FP64 oracle.

The reference ships no golden vectors (its tests are commented out), so these
fixtures pin the oracle itself: a 16^3 FFF field from this project's seeded
initial condition, one forced IF-RK4 step (reference-corner dealias), its
shell spectrum and sphere fluxes (the reference's per-sphere form,
compute_flux.cc:51-65).  The CPU tests check that the oracle still
reproduces them; the GPU tests check the CUDA path against them.
Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import tarang_ref as R  # noqa: E402

CASE = dict(N=16, k0=4.0, seed=0, energy=0.5, nu=0.01, dt=1e-3, f_in=2.0, f_out=3.0, eps=0.1,
            radii=[0.0, 2.0, 4.0, 8.0])


def compute():
    g = R.Grid((CASE["N"],) * 3)
    V0 = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), CASE["k0"]), CASE["seed"], CASE["energy"])
    es = np.zeros(g.n_shells())
    es[3] = CASE["eps"]
    cfg = R.FluidConfig(g, nu=CASE["nu"], dt=CASE["dt"], dealias_mode=R.DEALIAS_REFERENCE_CORNER,
                        forcing=R.CaratiForcing(CASE["f_in"], CASE["f_out"], es))
    V1 = R.rk4_step(cfg, V0)
    return dict(V0=V0, V1=V1, Ek1=R.shell_spectrum(g, V1), energy_supply=es,
                Pi1=R.flux_per_sphere(g, V1, CASE["radii"], R.DEALIAS_REFERENCE_CORNER),
                radii=np.array(CASE["radii"]))


if __name__ == "__main__":
    out = os.path.join(HERE, "fff16_forced_step.npz")
    np.savez_compressed(out, **compute())
    print("wrote", out)
