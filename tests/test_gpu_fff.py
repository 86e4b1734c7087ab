"""GPU parity of the FFF path against the FP64 oracle, through the C ABI.

Tolerances: FP64 path, relative L2 <= 1e-11 after a few steps (transform
round-off ~1e-15 per operation); FP32 path (FP32 transforms, FP64 sums and
integrating factor), relative L2 <= 1e-5 against the FP64 result of the same
nonlinear form.
"""
import math

import numpy as np
import pytest

from oracle import tarang_ref as R

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def to_np(t):
    return t.detach().cpu().numpy()


def plan_for(N, **kw):
    from tarang_b200 import Plan
    return Plan(N, **kw)


def oracle_ic(N, k0=4.0, seed=0, E=0.5):
    g = R.Grid((N, N, N) if isinstance(N, int) else N)
    return g, R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), k0), seed, E)


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N", [16, 32, 64, (32, 16, 64), (16, 64, 32)])
def test_fft_matches_numpy(cuda, prec, N):
    import torch
    Ns = (N, N, N) if isinstance(N, int) else N
    g = R.Grid(Ns)
    plan = plan_for(Ns, precision=prec)
    rng = np.random.default_rng(1)
    u = rng.standard_normal((2,) + Ns)
    rdt = torch.float64 if prec == "f64" else torch.float32
    real = torch.zeros((2, Ns[0], Ns[1], Ns[2] + 2), dtype=rdt, device=cuda)
    real[..., : Ns[2]] = torch.from_numpy(u).to(rdt)
    spec = plan.field(2)
    plan.forward(real, spec)
    torch.cuda.synchronize()
    ref = np.stack([R.forward(g, u[i]) for i in range(2)])
    tol = 1e-13 if prec == "f64" else 2e-6
    assert rel(to_np(spec), ref) < tol
    back = torch.zeros_like(real)
    plan.inverse(spec, back)
    torch.cuda.synchronize()
    ub = to_np(back)
    assert rel(ub[..., : Ns[2]], np.stack([R.inverse(g, ref[i]) for i in range(2)])) < tol
    assert np.all(ub[..., Ns[2]:] == 0)


def test_ic_matches_oracle(cuda):
    g, V = oracle_ic(32)
    plan = plan_for(32)
    u = plan.field(3)
    plan.init_energy_spectrum(R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5, u)
    assert rel(to_np(u), V) < 1e-13
    assert abs(plan.energy(u) - 0.5) < 1e-13


@pytest.mark.parametrize("dealias", ["reference", "two_thirds", "none"])
def test_nlin_matches_oracle(cuda, dealias):
    import torch
    mode = {"reference": 1, "two_thirds": 2, "none": 0}[dealias]
    g, V = oracle_ic(32, k0=8.0)
    plan = plan_for(32, dealias=dealias)
    u = torch.from_numpy(V.copy()).to(cuda)
    out = plan.field(3)
    plan.nlin(u, out)
    torch.cuda.synchronize()
    Vd = R.dealias(g, V, mode)
    ref = R.nlin_conservative(g, Vd)
    assert rel(to_np(out), ref) < 1e-13
    # the reference dealiases U in place (compute_nlin.cc:61-62)
    assert rel(to_np(u), Vd) == 0.0


@pytest.mark.parametrize("form", ["conservative", "rotational"])
@pytest.mark.parametrize("dealias", ["reference", "two_thirds"])
def test_rk4_matches_oracle_f64(cuda, form, dealias):
    import torch
    mode = {"reference": 1, "two_thirds": 2}[dealias]
    g, V = oracle_ic(32)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=mode, nlin_form=form)
    plan = plan_for(32, nu=0.01, dt=1e-3, dealias=dealias, nlin_form=form)
    u = torch.from_numpy(V.copy()).to(cuda)
    W = V.copy()
    for _ in range(3):
        W = R.rk4_step(cfg, W)
    plan.rk4_step(u, 3)
    torch.cuda.synchronize()
    assert rel(to_np(u), W) < 1e-12


def test_rk4_forced_matches_oracle_f64(cuda):
    import torch
    g, V = oracle_ic(32)
    es = np.zeros(g.n_shells())
    es[3] = 0.1
    forcing = R.CaratiForcing(2.0, 3.0, es)
    cfg = R.FluidConfig(g, nu=1e-3, dt=5e-4, dealias_mode=1, forcing=forcing)
    from tarang_b200 import Forcing
    plan = plan_for(32, nu=1e-3, dt=5e-4, forcing=Forcing(2.0, 3.0, es))
    u = torch.from_numpy(V.copy()).to(cuda)
    W = V.copy()
    for _ in range(3):
        W = R.rk4_step(cfg, W)
    plan.rk4_step(u, 3)
    torch.cuda.synchronize()
    assert rel(to_np(u), W) < 1e-12
    # the forcing injects energy: E grows against the unforced run
    W0 = V.copy()
    cfg0 = R.FluidConfig(g, nu=1e-3, dt=5e-4, dealias_mode=1)
    for _ in range(3):
        W0 = R.rk4_step(cfg0, W0)
    assert R.total_energy(g, W) > R.total_energy(g, W0)


def test_diagnostics_match_oracle(cuda):
    import torch
    g, V = oracle_ic(32)
    plan = plan_for(32, dealias="two_thirds")
    u = torch.from_numpy(V.copy()).to(cuda)
    assert abs(plan.energy(u) - R.total_energy(g, V)) < 1e-14
    Ek = plan.shell_spectrum(u)
    assert rel(Ek, R.shell_spectrum(g, V)) < 1e-13
    assert plan.max_div(u) < 1e-14
    radii = [0.0, 2.0, 4.0, 8.0, 10.5, 1e9]
    Pi = plan.flux(u, radii)
    ref = R.flux_one_pass(g, V, radii, 2)
    assert np.max(np.abs(Pi - ref)) < 1e-13 * max(1.0, np.max(np.abs(ref)))
    # per-sphere reference form agrees for the alias-free two-thirds field
    ref2 = R.flux_per_sphere(g, V, radii[:-1], 2)
    assert np.max(np.abs(Pi[:-1] - ref2)) < 1e-12


def test_f32_rotational_vs_f64(cuda):
    import torch
    g, V = oracle_ic(64)
    p64 = plan_for(64, precision="f64", nlin_form="rotational", dealias="two_thirds")
    p32 = plan_for(64, precision="f32", nlin_form="rotational", dealias="two_thirds")
    u64 = torch.from_numpy(V.copy()).to(cuda)
    u32 = u64.to(torch.complex64)
    for _ in range(5):
        p64.rk4_step(u64, 1)
        p32.rk4_step(u32, 1)
        torch.cuda.synchronize()
        e = rel(to_np(u32).astype(np.complex128), to_np(u64))
        assert e < 1e-5
        assert abs(p32.energy(u32) - p64.energy(u64)) / p64.energy(u64) < 1e-5


def test_config0_plain_small(cuda):
    """64^3, float64, nu = 0.01, dt = 1e-3, 100 steps, E(k), Pi(k) every 10 steps vs the oracle."""
    import torch
    g, V = oracle_ic(64)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=1)
    plan = plan_for(64, nu=0.01, dt=1e-3)
    u = torch.from_numpy(V.copy()).to(cuda)
    W = V.copy()
    radii = [0.0, 2.0, 4.0, 8.0, 16.0, 32.0]
    for step in range(1, 101):
        W = R.rk4_step(cfg, W)
        plan.rk4_step(u, 1)
        if step % 10 == 0:
            torch.cuda.synchronize()
            assert rel(to_np(u), W) < 1e-11
            assert rel(plan.shell_spectrum(u), R.shell_spectrum(g, W)) < 1e-11
            Pi = plan.flux(u, radii)
            # the reference's per-sphere form (the configuration's corner-box dealiasing)
            ref = R.flux_per_sphere(g, W, radii, 1)
            assert np.max(np.abs(Pi - ref)) < 1e-11 * max(1.0, np.max(np.abs(ref)))
    assert plan.max_div(u) < 1e-12


def test_host_pointer_step_matches_device(cuda):
    """The reference-facing call with host buffers (staged copies inside the call)."""
    import torch
    g, V = oracle_ic(32)
    plan = plan_for(32)
    host = np.ascontiguousarray(V.copy())
    dev = torch.from_numpy(V.copy()).to(cuda)
    plan.rk4_step(host, 2)
    plan.rk4_step(dev, 2)
    torch.cuda.synchronize()
    assert rel(host, to_np(dev)) == 0.0


@pytest.mark.parametrize("form", ["rotational", "conservative"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N", [(1024, 16, 32), (16, 1024, 32), (32, 16, 1024), (512, 32, 16)])
def test_rk4_long_axes(cuda, prec, N, form):
    """1024- and 512-point axes (their own tile widths and kernel variants) against the oracle."""
    import torch
    g = R.Grid(N)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=2, nlin_form=form)
    plan = plan_for(N, precision=prec, nu=0.01, dt=1e-3, dealias="two_thirds", nlin_form=form)
    dt = torch.complex128 if prec == "f64" else torch.complex64
    u = torch.from_numpy(V.copy()).to(cuda).to(dt)
    W = R.rk4_step(cfg, V)
    plan.rk4_step(u, 1)
    torch.cuda.synchronize()
    assert rel(u.cpu().numpy().astype(np.complex128), W) < (1e-12 if prec == "f64" else 1e-5)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_nlin_and_flux_long_x(cuda, prec):
    """Nx = 512 runs the split x pass (strided FFT + elementwise epilogue) in every mode."""
    import torch
    N = (512, 16, 32)
    g = R.Grid(N)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    plan = plan_for(N, precision=prec, dealias="two_thirds")
    dt = torch.complex128 if prec == "f64" else torch.complex64
    tol = 1e-12 if prec == "f64" else 2e-5
    u = torch.from_numpy(V.copy()).to(cuda).to(dt)
    out = plan.field(3)
    plan.nlin(u, out)
    torch.cuda.synchronize()
    assert rel(to_np(out).astype(np.complex128), R.nlin_conservative(g, R.dealias(g, V, 2))) < tol
    radii = [0.0, 2.0, 4.0, 8.0, 1e9]
    Pi = plan.flux(u, radii)
    ref = R.flux_one_pass(g, V, radii, 2)
    assert np.max(np.abs(Pi - ref)) < tol * 10 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_bitwise_reproducible(cuda, prec):
    """Same seed, same plan settings, fresh plans on memory that held other data:
    the initial condition, its energy and three steps agree bit for bit."""
    import torch
    outs = []
    for junk in (0.0, float("nan")):
        x = torch.full((1 << 26,), junk, dtype=torch.float64, device=cuda)
        del x
        torch.cuda.empty_cache()
        plan = plan_for(64, precision=prec, nlin_form="rotational", dealias="two_thirds")
        u = plan.field(3)
        plan.init_energy_spectrum(R.spectrum_k4_gauss(plan.n_shells, 4.0), 7, 0.5, u)
        e0 = plan.energy(u)
        plan.rk4_step(u, 3)
        torch.cuda.synchronize()
        outs.append((e0, u.clone(), plan.energy(u)))
        plan.close()
    assert outs[0][0] == outs[1][0]
    assert torch.equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


@pytest.mark.parametrize("dealias", ["two_thirds", "reference"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_shell_and_flux_sums_bitwise_reproducible(cuda, prec, dealias):
    """E(k), the raw shell sums and Pi(R) are added in a fixed order (no atomics on the sums):
    repeated calls, and fresh plans, give the same bits."""
    import torch
    radii = [0.0, 2.0, 4.0, 8.0, 12.0, 1e9]
    res = []
    for _ in range(2):
        plan = plan_for(64, precision=prec, dealias=dealias)
        u = plan.field(3)
        plan.init_energy_spectrum(R.spectrum_k4_gauss(plan.n_shells, 6.0), 11, 0.5, u)
        for _ in range(3):
            res.append((plan.shell_spectrum(u), plan.shell_sums(u)[0], plan.flux(u, radii)))
        plan.close()
        torch.cuda.empty_cache()
    for r in res[1:]:
        for a, b in zip(res[0], r):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("N,k0", [(32, 8.0), ((32, 16, 64), 4.0)])
@pytest.mark.parametrize("mode", [1, 0])
def test_flux_per_sphere_matches_oracle(cuda, N, k0, mode):
    """Pi(R) under the reference's corner-box dealiasing (and none) is the per-sphere algorithm of
    EnergyTr::Compute_flux (compute_flux.cc:51-65): one giver nonlinear term per sphere.  There the
    one-pass form differs from it by the aliased part of the products (about 8 % of max|Pi| at
    32^3, k0 = 8), so the test also checks that the GPU result is not the one-pass value."""
    import torch
    g, V = oracle_ic(N, k0=k0, seed=3)
    radii = [0.0, 2.0, 4.0, 8.0, 12.0, 1e9]
    ref = R.flux_per_sphere(g, V, radii, mode)
    one = R.flux_one_pass(g, V, radii, mode)
    scale = np.max(np.abs(ref))
    dl = {1: "reference", 0: "none"}[mode]
    for prec, tol in (("f64", 1e-12), ("f32", 2e-6)):
        plan = plan_for(N, precision=prec, dealias=dl)
        dt = torch.complex128 if prec == "f64" else torch.complex64
        u = torch.from_numpy(V.copy()).to(cuda).to(dt)
        Pi = plan.flux(u, radii)
        assert np.max(np.abs(Pi - ref)) < tol * scale, (prec, Pi, ref)
        # the state is not modified by the diagnostic
        assert torch.equal(u, torch.from_numpy(V.copy()).to(cuda).to(dt))
        plan.close()
    if mode == 1 and N == 32:
        assert np.max(np.abs(one - ref)) > 0.05 * scale


def test_flux_radii_limit(cuda):
    """At most 63 radii: more are refused with TS_ERR_ARG, not truncated."""
    plan = plan_for(16, precision="f64", dealias="two_thirds")
    u = plan.field(3)
    with pytest.raises(RuntimeError):
        plan.flux(u, np.arange(64, dtype=np.float64))
    assert len(plan.flux(u, np.arange(63, dtype=np.float64))) == 63


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_alloc_field_is_a_zeroed_plan_field(cuda, prec):
    """ts_alloc_field returns a zeroed device field of the plan's layout: energy 0, and the
    same initial condition and three steps on it as on a torch field, bit for bit; ts_free_field
    releases it; ncomp < 1 is refused."""
    import ctypes
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = plan_for(32, precision=prec, nlin_form="rotational", dealias="two_thirds")
    lib = plan.lib
    f = ctypes.c_void_p()
    L.check(lib.ts_alloc_field(plan.h, 3, ctypes.byref(f)), "ts_alloc_field")
    assert f.value
    e = ctypes.c_double(-1.0)
    L.check(lib.ts_energy(plan.h, f, 3, ctypes.byref(e)), "ts_energy")
    assert e.value == 0.0
    E = np.ascontiguousarray(R.spectrum_k4_gauss(plan.n_shells, 4.0))
    L.check(lib.ts_init_energy_spectrum(plan.h, E.ctypes.data_as(L._D), len(E), 5, 0.5, f), "ts_init_energy_spectrum")
    L.check(lib.ts_rk4_step(plan.h, f, 3), "ts_rk4_step")
    L.check(lib.ts_energy(plan.h, f, 3, ctypes.byref(e)), "ts_energy")
    u = plan.field(3)
    plan.init_energy_spectrum(E, 5, 0.5, u)
    plan.rk4_step(u, 3)
    torch.cuda.synchronize()
    assert e.value == plan.energy(u) and e.value > 0
    L.check(lib.ts_free_field(f), "ts_free_field")
    g = ctypes.c_void_p()
    assert lib.ts_alloc_field(plan.h, 0, ctypes.byref(g)) == L.TS_ERR_ARG and not g.value
