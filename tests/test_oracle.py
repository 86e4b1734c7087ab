"""Known-answer tests of the FP64 oracle (CPU only).

The reference ships no tests or golden vectors (its src/test is commented
out), so the oracle is pinned by (a) the reference's own analytic initial
conditions, whose spectral coefficients fix the transform convention
(ic_model.cc:55-140), and (b) analytic / self-consistency identities.
"""
import math

import numpy as np
import pytest

from oracle import tarang_ref as R


def tg_real(g, k0=1, amp=1.0):
    N = g.N[0]
    x = 2 * np.pi * np.arange(N) / N
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = amp * np.sin(k0 * X) * np.cos(k0 * Y) * np.cos(k0 * Z)
    v = -amp * np.cos(k0 * X) * np.sin(k0 * Y) * np.cos(k0 * Z)
    return np.stack([u, v, np.zeros_like(u)])


def fwd(g, ur):
    return np.stack([R.forward(g, ur[i]) for i in range(ur.shape[0])])


def test_taylor_green_coefficients_match_reference_ic():
    """Setup_Taylor_Green_field FFF (ic_model.cc:84-94): V1(+-k0,+-k0,k0) = -+i amp/8, V2 likewise."""
    g = R.Grid((16, 16, 16))
    k0, amp = 2, 0.7
    V = fwd(g, tg_real(g, k0, amp))
    ex = np.zeros_like(V)
    lx = lambda k: k % 16
    ex[0, lx(k0), lx(k0), k0] = -1j * amp / 8
    ex[0, lx(k0), lx(-k0), k0] = -1j * amp / 8
    ex[0, lx(-k0), lx(k0), k0] = 1j * amp / 8
    ex[0, lx(-k0), lx(-k0), k0] = 1j * amp / 8
    ex[1, lx(k0), lx(k0), k0] = 1j * amp / 8
    ex[1, lx(-k0), lx(k0), k0] = 1j * amp / 8
    ex[1, lx(k0), lx(-k0), k0] = -1j * amp / 8
    ex[1, lx(-k0), lx(-k0), k0] = -1j * amp / 8
    assert np.max(np.abs(V - ex)) < 1e-15


def test_abc_reference_ic_real_field():
    """Setup_ABC_field FFF (ic_model.cc:117-129): the kz-only modes carry amp*C, so the inverse
    transform gives u1 = amp (B cos y + 2 C sin z) (not a Beltrami field)."""
    g = R.Grid((16, 16, 16))
    A, B, C, amp = 0.3, 0.5, 0.7, 1.1
    V = np.zeros((3,) + g.shape, complex)
    V[0, 0, 1, 0] = amp * B / 2
    V[0, 0, 15, 0] = amp * B / 2
    V[0, 0, 0, 1] = -1j * amp * C
    u1 = R.inverse(g, V[0])
    x = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    assert np.max(np.abs(u1 - amp * (B * np.cos(Y) + 2 * C * np.sin(Z)))) < 1e-14


@pytest.mark.parametrize("N", [(16, 16, 16), (8, 16, 32)])
def test_roundtrip_and_parseval(N):
    g = R.Grid(N)
    rng = np.random.default_rng(0)
    u = rng.standard_normal(N)
    A = R.forward(g, u)
    assert np.max(np.abs(R.inverse(g, A) - u)) < 1e-13
    A[:, :, N[2] // 2] = 0  # Parseval holds for fields without the kz = Nz/2 plane
    ur = R.inverse(g, A)
    assert abs(R.total_energy_scalar(g, A) - (ur ** 2).sum() / (2 * np.prod(N))) < 1e-13


@pytest.mark.parametrize("par", ["S", "C"])
def test_sff_roundtrip_and_energy(par):
    g = R.Grid((16, 8, 16), (math.pi, 2 * math.pi, 2 * math.pi), "SFF")
    rng = np.random.default_rng(3)
    A = R.forward(g, rng.standard_normal(g.rshape), par)
    A[:, :, g.N[2] // 2] = 0
    ur = R.inverse(g, A, par)
    A2 = R.forward(g, ur, par)
    assert np.max(np.abs(A2 - A)) < 1e-13
    assert abs(R.total_energy_scalar(g, A) - (ur ** 2).sum() / (2 * ur.size)) < 1e-12


def test_derivative_of_single_mode():
    g = R.Grid((16, 16, 16))
    x = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(3 * X) * np.cos(2 * Z)
    A = R.forward(g, u)
    dx = R.inverse(g, R.xderiv(g, A))
    dz = R.inverse(g, R.zderiv(g, A))
    assert np.max(np.abs(dx - 3 * np.cos(3 * X) * np.cos(2 * Z))) < 1e-13
    assert np.max(np.abs(dz + 2 * np.sin(3 * X) * np.sin(2 * Z))) < 1e-13


def test_sff_x_derivative_parity():
    """SFF Xderiv: a sine series differentiates to a cosine series with +Kx (SFF_pencil_tr.cc:77-90)."""
    g = R.Grid((16, 8, 8), (math.pi, 2 * math.pi, 2 * math.pi), "SFF")
    xs = (np.arange(16) + 0.5) / 16
    X = xs[:, None, None] * np.ones((16, 8, 8))
    u = np.sin(3 * math.pi * X)
    A = R.forward(g, u, "S")
    du = R.inverse(g, R.xderiv(g, A, "S"), "C")
    assert np.max(np.abs(du - 3 * math.pi * np.cos(3 * math.pi * X))) < 1e-12


def test_projection_idempotent_and_solenoidal():
    g = R.Grid((16, 16, 16))
    rng = np.random.default_rng(1)
    N = np.stack([R.forward(g, rng.standard_normal((16, 16, 16))) for _ in range(3)])
    P1 = -R.project_rhs(g, N)
    P2 = -R.project_rhs(g, P1)
    assert np.max(np.abs(P1 - P2)) < 1e-15
    assert R.max_abs_div(g, P1) < 1e-14


def test_taylor_green_linear_decay():
    """Small amplitude TG decays as exp(-2 nu k^2 t) in energy, k^2 = 3 (the IF factor is exact)."""
    g = R.Grid((16, 16, 16))
    V = fwd(g, tg_real(g, 1, 1e-7))
    nu, dt, n = 0.05, 1e-2, 10
    cfg = R.FluidConfig(g, nu=nu, dt=dt, dealias_mode=R.DEALIAS_TWO_THIRDS)
    E0 = R.total_energy(g, V)
    for _ in range(n):
        V = R.rk4_step(cfg, V)
    assert abs(R.total_energy(g, V) / E0 - math.exp(-2 * nu * 3 * n * dt)) < 1e-9


def test_beltrami_field_decays_exactly():
    """A k=1 Beltrami field (omega = u) has u x omega = 0: after projection the nonlinear term
    vanishes, so u(t) = u(0) exp(-nu t)."""
    g = R.Grid((16, 16, 16))
    x = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    A, B, C = 0.9, 0.6, 0.4
    u = np.stack([A * np.sin(Z) + C * np.cos(Y), B * np.sin(X) + A * np.cos(Z), C * np.sin(Y) + B * np.cos(X)])
    V = fwd(g, u)
    nu, dt, n = 0.02, 1e-2, 5
    for form in ("conservative", "rotational"):
        cfg = R.FluidConfig(g, nu=nu, dt=dt, dealias_mode=R.DEALIAS_TWO_THIRDS, nlin_form=form)
        W = V.copy()
        for _ in range(n):
            W = R.rk4_step(cfg, W)
        assert np.max(np.abs(W - V * math.exp(-nu * n * dt))) < 1e-13


def test_nonlinear_term_conserves_energy_two_thirds():
    """For a two-thirds-dealiased field the projected nonlinear term does no work:
    sum_w Re(U* . RHS(U)) = 0 (inviscid, unforced), in both forms."""
    g = R.Grid((32, 32, 32))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 3.0), 5, 0.5)
    V = R.dealias(g, V, R.DEALIAS_TWO_THIRDS)
    for form in ("conservative", "rotational"):
        cfg = R.FluidConfig(g, nu=0.0, dt=1e-3, dealias_mode=R.DEALIAS_TWO_THIRDS, nlin_form=form)
        rhs, _ = R.fluid_rhs(cfg, V, g.modes_in_shell())
        work = sum(R.cross_energy(g, rhs[i], V[i]) for i in range(3))
        scale = sum(R.cross_energy(g, np.abs(rhs[i]), np.abs(V[i])) for i in range(3))
        assert abs(work) < 1e-14 * scale


def test_conservative_and_rotational_agree_on_kept_modes():
    g = R.Grid((16, 16, 16))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 2, 0.5)
    Vd = R.dealias(g, V, R.DEALIAS_TWO_THIRDS)
    Nc = R.project_rhs(g, R.nlin_conservative(g, Vd))
    Nr = R.project_rhs(g, R.nlin_rotational(g, Vd))
    keep = ~R.dealias_mask(g, R.DEALIAS_TWO_THIRDS)
    assert np.max(np.abs((Nc - Nr)[:, keep])) < 1e-14


def test_flux_one_pass_equals_per_sphere():
    g = R.Grid((16, 16, 16))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 3.0), 7, 0.5)
    radii = [0.0, 1.5, 2.0, 3.0, 4.0]
    a = R.flux_per_sphere(g, V, radii, R.DEALIAS_TWO_THIRDS)
    b = R.flux_one_pass(g, V, radii, R.DEALIAS_TWO_THIRDS)
    assert np.max(np.abs(a - b)) < 1e-15


def test_flux_one_pass_equals_per_sphere_on_ssf():
    """On the SSF basis too the two flux forms agree under two-thirds dealiasing (the
    per-sphere restatement goes through the sin/cos parities of every product)."""
    kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    g = R.Grid((16, 32, 16), kf, "SSF")
    rng = np.random.default_rng(3)
    U = np.stack([R.forward(g, rng.standard_normal(g.rshape), R.SSF_PARITY[v]) for v in ("Vx", "Vy", "Vz")])
    U = -0.3 * R.project_rhs(g, U)
    radii = [1.0, 2.0, 4.0, 6.0]
    a = R.flux_per_sphere(g, U, radii, R.DEALIAS_TWO_THIRDS)
    b = R.flux_one_pass(g, U, radii, R.DEALIAS_TWO_THIRDS)
    assert np.max(np.abs(a - b)) < 1e-12 * np.max(np.abs(a))
    # and under the corner box they differ, as on FFF
    a = R.flux_per_sphere(g, U, radii, R.DEALIAS_REFERENCE_CORNER)
    b = R.flux_one_pass(g, U, radii, R.DEALIAS_REFERENCE_CORNER)
    assert np.max(np.abs(a - b)) > 0.1 * np.max(np.abs(a))


def test_flux_one_pass_equals_per_sphere_on_sff():
    """On the SFF basis (sin/cos along x, Fourier along y and z; the RBC basis) the two flux
    forms agree under two-thirds dealiasing, in three and in two dimensions."""
    kf = (math.pi, 2 * math.pi, 2 * math.pi)
    for N in ((16, 16, 16), (32, 1, 32)):
        g = R.Grid(N, kf, "SFF")
        rng = np.random.default_rng(5)
        U = np.stack([R.reality_fix(g, R.forward(g, rng.standard_normal(g.rshape), R.SFF_PARITY[v]))
                      for v in ("Vx", "Vy", "Vz")])
        if N[1] == 1:
            U[1] = 0
        U = -0.3 * R.project_rhs(g, U)
        radii = [1.0, 3.0, 6.0, 10.0]
        a = R.flux_per_sphere(g, U, radii, R.DEALIAS_TWO_THIRDS)
        b = R.flux_one_pass(g, U, radii, R.DEALIAS_TWO_THIRDS)
        assert np.max(np.abs(a)) > 0
        assert np.max(np.abs(a - b)) < 1e-12 * np.max(np.abs(a)), (N, a, b)


def test_flux_forms_differ_under_the_corner_box():
    """Under the reference's corner-box dealiasing (and none) the products alias onto modes the
    field holds, so the one-pass form is not the reference's per-sphere Pi(R): at 32^3 with
    k0 = 8 they differ by about 8 % of max|Pi|.  The library therefore runs the per-sphere
    algorithm in those modes and keeps the one-pass form for two-thirds dealiasing only."""
    g = R.Grid((32, 32, 32))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 8.0), 0, 0.5)
    radii = [2.0, 4.0, 8.0, 12.0]
    for mode in (R.DEALIAS_REFERENCE_CORNER, 0):
        a = R.flux_per_sphere(g, V, radii, mode)
        b = R.flux_one_pass(g, V, radii, mode)
        assert np.max(np.abs(a - b)) > 0.05 * np.max(np.abs(a))
    # the per-sphere flux out of a sphere holding every mode is zero
    assert abs(R.flux_per_sphere(g, V, [1e9], R.DEALIAS_REFERENCE_CORNER)[0]) == 0.0


def test_ic_shell_energies_and_divergence():
    """Per shell s < N/2-1 the Tarang-weighted energy equals c E_ic(s) exactly; div = 0."""
    g = R.Grid((32, 32, 32))
    E = R.spectrum_k4_gauss(g.n_shells(), 4.0)
    V = R.init_energy_spectrum(g, E, 11, None)
    assert R.max_abs_div(g, V) < 1e-15 * 16 * np.abs(V).max()
    idx = np.ceil(g.Kmag()).astype(int)
    w = np.where(np.arange(g.shape[2])[None, None, :] == 0, 0.5, 1.0) * np.ones(g.shape)
    e = (np.abs(V) ** 2).sum(0) * w
    shells = np.bincount(idx.ravel(), weights=e.ravel())
    s = np.arange(1, 15)
    np.testing.assert_allclose(shells[s], E[s], rtol=1e-12)
    V2 = R.init_energy_spectrum(g, E, 11, 0.5)
    assert abs(R.total_energy(g, V2) - 0.5) < 1e-14


def test_rng_is_counter_based_splitmix64():
    u = R.uniform01(0, np.arange(4, dtype=np.uint64))
    assert np.all((u >= 0) & (u < 1))
    # fixed values of this project's generator (shared with csrc/ts_misc.cuh)
    assert abs(u[0] - R.uniform01(0, np.array([0], np.uint64))[0]) == 0
    assert R.uniform01(1, np.arange(4, dtype=np.uint64))[0] != u[0]


def test_reality_fix_makes_kz0_plane_hermitian():
    g = R.Grid((8, 8, 8))
    rng = np.random.default_rng(4)
    A = rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)
    B = R.reality_fix(g, A)
    assert np.all(B[:, :, 4] == 0)
    for lx in range(5, 8):
        for ly in range(8):
            if g.ky[ly] != 4:
                assert B[lx, ly, 0] == np.conj(B[(-g.kx[lx]) % 8, (-g.ky[ly]) % 8, 0])


def test_rbc_linear_stability():
    """Free-slip RBC, kfactor (pi, 2pi, 2pi): the lowest mode (m=1, k_perp=2pi) has critical
    Ra = (pi^2 + 4 pi^2)^3 / (4 pi^2) ~ 3044; a small perturbation decays at Ra=1000 and grows at Ra=1e5."""
    g = R.Grid((16, 8, 8), (math.pi, 2 * math.pi, 2 * math.pi), "SFF")
    T0 = R.rbc_temperature_ic(g, 1e-6, 1.5, 3)
    U0 = np.zeros((3,) + g.shape, complex)
    out = {}
    for Ra in (1e3, 1e5):
        cfg = R.RBCConfig(g, Ra=Ra, Pr=1.0, dt=2e-2)
        U, T = U0.copy(), T0.copy()
        E0 = R.total_energy_scalar(g, T)
        for _ in range(60):
            U, T = R.rbc_rk4_step(cfg, U, T)
        out[Ra] = R.total_energy_scalar(g, T) / E0
    assert out[1e3] < 0.9
    assert out[1e5] > 1.1


# ---------------------------------------------------------------------------
# discrete adjoint: <Phi'(U) d, lam> = <d, Phi'(U)^T lam> with Phi' from central
# differences of the oracle step (16^3, both reality-fix settings)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("reality", [False, True])
def test_adjoint_dot_product(reality):
    g = R.Grid((16, 16, 16))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=0.01, dt=5e-2, dealias_mode=2, nlin_form="rotational", reality_fix=reality)
    rng = np.random.default_rng(7)
    rnd = lambda: rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
    ip = lambda a, b: float(np.real(np.sum(a * np.conj(b))))
    d, lam, eps = rnd(), rnd(), 1e-6
    jd = (R.rk4_step(cfg, V + eps * d) - R.rk4_step(cfg, V - eps * d)) / (2 * eps)
    lhs, rhs = ip(jd, lam), ip(d, R.rk4_step_adjoint(cfg, V, lam))
    assert abs(lhs - rhs) < 1e-8 * abs(lhs)


def test_reality_fix_adjoint_is_transpose():
    g = R.Grid((16, 32, 16))
    rng = np.random.default_rng(3)
    A = rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
    B = rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
    ip = lambda a, b: float(np.real(np.sum(a * np.conj(b))))
    assert abs(ip(R.reality_fix_vec(g, A), B) - ip(A, R.reality_fix_vec_adjoint(g, B))) < 1e-12 * abs(ip(A, B)) + 1e-9


# ---------------------------------------------------------------------------
# passive scalar and MHD (FFF)
# ---------------------------------------------------------------------------
def test_scalar_pure_diffusion_is_exact():
    """u = 0: the passive scalar only diffuses, and the integrating factor makes that exact."""
    g = R.Grid((16, 16, 16))
    rng = np.random.default_rng(3)
    T0 = R.reality_fix(g, R.forward(g, rng.standard_normal(g.rshape)))
    cfg = R.ScalarConfig(g, nu=0.01, kappa=0.05, dt=1e-2, dealias_mode=0)
    U, T = np.zeros((3,) + g.shape, complex), T0.copy()
    for _ in range(5):
        U, T = R.rbc_rk4_step(cfg, U, T)
    expect = R.reality_fix(g, T0 * np.exp(-cfg.kappa * g.Ksqr() * 5 * cfg.dt))
    assert np.max(np.abs(T - expect)) < 1e-14
    assert np.max(np.abs(U)) == 0


def test_scalar_mean_kept_and_variance_decays():
    g = R.Grid((16, 16, 16))
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 2.0), 0, 0.5)
    rng = np.random.default_rng(4)
    T = R.reality_fix(g, R.forward(g, rng.standard_normal(g.rshape)))
    T[0, 0, 0] = 0.3
    cfg = R.ScalarConfig(g, nu=0.01, kappa=0.05, dt=2e-3, dealias_mode=2)
    v0 = R.total_energy_scalar(g, T)
    for _ in range(5):
        U, T = R.rbc_rk4_step(cfg, U, T)
    assert abs(T[0, 0, 0] - 0.3) < 1e-15
    assert R.total_energy_scalar(g, T) < v0


def test_mhd_without_field_is_the_fluid_step():
    """B = 0: the Elsasser nonlinear terms reduce to the conservative fluid term and B stays 0."""
    g = R.Grid((16, 16, 16))
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 3.0), 1, 0.5)
    fl = R.FluidConfig(g, nu=0.01, dt=1e-3, dealias_mode=2, nlin_form="conservative")
    mh = R.MHDConfig(g, nu=0.01, eta=0.02, dt=1e-3, dealias_mode=2)
    Uf = R.rk4_step(fl, U.copy())
    Um, Bm = R.mhd_rk4_step(mh, U.copy(), np.zeros_like(U))
    assert np.max(np.abs(Bm)) == 0
    assert np.linalg.norm(Um - Uf) <= 1e-13 * np.linalg.norm(Uf)


def test_ideal_mhd_invariants():
    """nu = eta = 0: total energy and cross helicity conserved to the RK4 error, fields solenoidal."""
    g = R.Grid((16, 16, 16))
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 2.0), 0, 0.5)
    B = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 2.0), 1, 0.3)
    cfg = R.MHDConfig(g, nu=0.0, eta=0.0, dt=1e-3, dealias_mode=2)
    E0 = R.total_energy(g, U) + R.total_energy(g, B)
    H0 = sum(R.cross_energy(g, U[i], B[i]) for i in range(3))
    for _ in range(10):
        U, B = R.mhd_rk4_step(cfg, U, B)
    E1 = R.total_energy(g, U) + R.total_energy(g, B)
    H1 = sum(R.cross_energy(g, U[i], B[i]) for i in range(3))
    assert abs(E1 - E0) < 1e-6 * E0
    assert abs(H1 - H0) < 1e-6 * E0
    assert R.max_abs_div(g, B) < 1e-14 and R.max_abs_div(g, U) < 1e-14


def test_ssf_taylor_green_step_is_exact_decay():
    """SSF basis: u = sin x cos y, v = -cos x sin y has a gradient nonlinear term, so the
    projected right-hand side vanishes and the step is exp(-2 nu t)."""
    g = R.Grid((16, 16, 16), (1.0, 1.0, 1.0), "SSF")
    x = (np.arange(16) + 0.5) * np.pi / 16
    z = 2 * np.pi * np.arange(16) / 16
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    U0 = np.stack([R.forward(g, np.sin(X) * np.cos(Y), "SCF"), R.forward(g, -np.cos(X) * np.sin(Y), "CSF"),
                   R.forward(g, np.zeros_like(X), "CCF")])
    assert abs(U0[0, 1, 1, 0] - 0.25) < 1e-15  # 2 sin x . 2 cos y / 4
    cfg = R.FluidConfig(g, nu=0.05, dt=1e-2, dealias_mode=1, nlin_form="conservative")
    U = U0.copy()
    for _ in range(5):
        U = R.rk4_step(cfg, U)
    assert np.max(np.abs(U - U0 * np.exp(-0.05 * 2 * 5e-2))) < 1e-15


def test_sss_transforms_and_taylor_green():
    """SSS basis: synthesis then analysis returns representable coefficients for every
    parity, and the 2-D Taylor-Green field decays exactly."""
    g = R.Grid((16, 16, 16), (1.0, 1.0, 1.0), "SSS")
    rng = np.random.default_rng(0)
    for par in ("SCC", "CSC", "CCS", "CCC", "SSC", "SCS", "CSS", "SSS"):
        A = rng.standard_normal(g.shape)
        for ax in range(3):
            if par[ax] == "S":
                idx = [slice(None)] * 3
                idx[ax] = 0
                A[tuple(idx)] = 0
        assert np.max(np.abs(R.forward(g, R.inverse(g, A, par), par) - A)) < 1e-13
    x = (np.arange(16) + 0.5) * np.pi / 16
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    U0 = np.stack([R.forward(g, np.sin(X) * np.cos(Y), "SCC"), R.forward(g, -np.cos(X) * np.sin(Y), "CSC"),
                   R.forward(g, np.zeros_like(X), "CCS")])
    cfg = R.FluidConfig(g, nu=0.05, dt=1e-2, dealias_mode=1, nlin_form="conservative")
    U = U0.copy()
    for _ in range(5):
        U = R.rk4_step(cfg, U)
    assert np.max(np.abs(U - U0 * np.exp(-0.05 * 2 * 5e-2))) < 1e-15


@pytest.mark.parametrize("basis", ["SSF", "SSS"])
def test_rbc_single_roll_follows_linear_theory(basis):
    """RBC on SSF / SSS (PRLARGE, ULARGE; the temperature takes the Vx parity): one small
    roll u_x = a sin(kx x) cos(ky y), u_y = c cos(kx x) sin(ky y), theta = b sin(kx x) cos(ky y)
    obeys da/dt = (1 - kx^2/K^2) b - nu K^2 a, db/dt = a - kappa K^2 b to O(amplitude):
    compared with the matrix exponential of that system over 20 steps."""
    from scipy.linalg import expm
    kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    g = R.Grid((16, 16, 8), kf, basis)
    eps = 1e-9
    U0 = np.zeros((3,) + g.shape, np.float64 if basis == "SSS" else complex)
    T0 = np.zeros(g.shape, U0.dtype)
    kx, ky = kf[0], kf[1]
    U0[0, 1, 1, 0] = eps
    U0[1, 1, 1, 0] = -kx * eps / ky   # kx a + ky c = 0
    T0[1, 1, 0] = 0.5 * eps
    cfg = R.RBCConfig(g, Ra=3e4, Pr=0.7, dt=2e-3)
    U, T = U0.copy(), T0.copy()
    for _ in range(20):
        U, T = R.rbc_rk4_step(cfg, U, T)
    K2 = kx * kx + ky * ky
    M = np.array([[-cfg.nu * K2, 1 - kx * kx / K2], [1.0, -cfg.kappa * K2]])
    a, b = expm(M * 20 * cfg.dt) @ np.array([eps, 0.5 * eps])
    assert abs(U[0, 1, 1, 0] - a) < 1e-7 * eps and abs(T[1, 1, 0] - b) < 1e-7 * eps
    assert abs(U[0, 1, 1, 0] / U0[0, 1, 1, 0] - 1) > 1e-3   # the buoyancy did act
    # the roll stays in its mode: kx a + ky c = 0, and nothing else grows at first order
    assert abs(kx * U[0, 1, 1, 0] + ky * U[1, 1, 1, 0]) < 1e-7 * eps
    U[:, 1, 1, 0] = 0
    T[1, 1, 0] = 0
    assert np.max(np.abs(U)) < 1e-6 * eps and np.max(np.abs(T)) < 1e-6 * eps


@pytest.mark.parametrize("basis,parity", [("SSF", "SCF"), ("SSF", "CCF"), ("SSF", "SSF"), ("SSS", "SCC"),
                                          ("SSS", "CCC"), ("SSS", "SSS"), ("SSS", "CSS")])
def test_sincos_energy_weights_are_parseval(basis, parity):
    """The SSF / SSS energy weights (4 / 2 / 1 / 1/2 by the number of zero indices) give
    <u^2>/2 of the real field; on SSF with the kz = Nz/2 plane empty, which the reference
    weights like an interior plane."""
    g = R.Grid((16, 8, 16), (1.0, 1.0, 1.0), basis)
    A = R.forward(g, np.random.default_rng(2).standard_normal(g.rshape), parity)
    if basis == "SSF":
        A[:, :, -1] = 0
    u = R.inverse(g, A, parity)
    assert abs(R.total_energy_scalar(g, A) / (0.5 * np.mean(u ** 2)) - 1) < 1e-13
    assert abs(R.cross_energy(g, A, A) - R.total_energy_scalar(g, A)) < 1e-13


SCALINGS = [("PRLARGE", "ULARGE"), ("PRLARGE", "USMALL"), ("PRSMALL", "ULARGE"), ("PRSMALL", "USMALL")]


@pytest.mark.parametrize("pr,us", SCALINGS)
def test_rbc_scalings_are_one_physics(pr, us):
    """Every scaling of compute_force_RBC.cc / Iscalar_main.cc describes the same Boussinesq
    system in other units: cu cT / (nu kappa) = Ra and nu / kappa = Pr."""
    Ra, Pr = 3.7e5, 0.3
    c = R.rbc_coefficients(pr, us, Ra, Pr)
    assert abs(c["cu"] * c["cT"] / (c["nu"] * c["kappa"]) / Ra - 1) < 1e-14
    assert abs(c["nu"] / c["kappa"] / Pr - 1) < 1e-14
    with pytest.raises(ValueError):
        R.rbc_coefficients("PRHALF", us, Ra, Pr)


@pytest.mark.parametrize("pr,us", SCALINGS)
def test_rbc_roll_follows_the_linear_system_every_scaling(pr, us):
    """One small free-slip roll on SFF under each scaling follows the exact linear system
    da/dt = cu (1 - kx^2/K^2) b - nu K^2 a, db/dt = cT a - kappa K^2 b to 1e-7 of its amplitude
    over 20 steps, and the Nusselt number is nu0 + nuc <u1, T>."""
    from scipy.linalg import expm
    kf = (math.pi, 2 * math.pi, 2 * math.pi)
    g = R.Grid((16, 8, 8), kf, "SFF")
    eps = 1e-9
    U0 = np.zeros((3,) + g.shape, complex)
    T0 = np.zeros(g.shape, complex)
    kx, kz = kf[0], kf[2]
    # mode m = 1, kz = 1: u1 sine, u3 cosine with kx a + kz c = 0 (divergence Kx U1 + i Kz U3 = 0)
    U0[0, 1, 0, 1] = eps
    U0[2, 1, 0, 1] = 1j * kx * eps / kz
    T0[1, 0, 1] = 0.5 * eps
    cfg = R.RBCConfig(g, Ra=2e4, Pr=0.7, dt=5e-5 if us == "USMALL" else 2e-3, pr_option=pr, uscaling=us)
    co = cfg.coeffs
    U, T = U0.copy(), T0.copy()
    for _ in range(20):
        U, T = R.rbc_rk4_step(cfg, U, T)
    K2 = kx * kx + kz * kz
    M = np.array([[-cfg.nu * K2, co["cu"] * (1 - kx * kx / K2)], [co["cT"], -cfg.kappa * K2]])
    a, b = expm(M * 20 * cfg.dt) @ np.array([eps, 0.5 * eps])
    assert abs(U[0, 1, 0, 1] - a) < 1e-7 * eps and abs(T[1, 0, 1] - b) < 1e-7 * eps
    assert abs(U[0, 1, 0, 1] / eps - 1) > 1e-5   # the state moved
    nu = R.nusselt(cfg, U, T)
    assert nu == co["nu0"] + co["nuc"] * R.cross_energy(g, U[0], T)


@pytest.mark.parametrize("pr,us", [("PRZERO", "USMALL"), ("PRZERO", "ULARGE"), ("PRINFTY", "USMALL"),
                                   ("PRINFTY", "ULARGE")])
def test_rbc_slaved_roll_follows_its_growth_rate(pr, us):
    """PRZERO (T = U.V1 / K^2) and PRINFTY (U = vs P(T x) / K^2) reduce one small free-slip
    roll to one linear equation: da/dt = (cu kz^2 / K^4 - nu K^2) a for PRZERO and
    db/dt = (cT vs kz^2 / K^4 - kappa K^2) b for PRINFTY.  Over 20 steps the advanced field
    follows it to 1e-7 of its amplitude, the slaved field equals its formula exactly, and
    the slaved velocity is divergence-free."""
    kf = (math.pi, 2 * math.pi, 2 * math.pi)
    g = R.Grid((16, 8, 8), kf, "SFF")
    eps = 1e-9
    kx, kz = kf[0], kf[2]
    K2 = kx * kx + kz * kz
    Ra = 2e3 if us == "USMALL" else 2e4
    cfg = R.RBCConfig(g, Ra=Ra, Pr=0.7, dt=2e-4 if us == "USMALL" else 2e-3, pr_option=pr, uscaling=us)
    co = cfg.coeffs
    U0 = np.zeros((3,) + g.shape, complex)
    T0 = np.zeros(g.shape, complex)
    if pr == "PRZERO":
        U0[0, 1, 0, 1] = eps
        U0[2, 1, 0, 1] = 1j * kx * eps / kz
        T0 = R.rbc_slave_temperature(g, U0)
        sigma = co["cu"] * kz * kz / K2 ** 2 - co["nu"] * K2
    else:
        T0[1, 0, 1] = eps
        U0 = R.rbc_slave_velocity(g, T0, co["vs"])
        sigma = co["cT"] * co["vs"] * kz * kz / K2 ** 2 - co["kappa"] * K2
        # the slaved roll: U1 = vs kz^2 / K^4 T, U3 = i kx U1 / kz, divergence Kx U1 + i Kz U3 = 0
        assert abs(U0[0, 1, 0, 1] - co["vs"] * kz * kz / K2 ** 2 * eps) < 1e-15 * abs(U0[0, 1, 0, 1])
        assert abs(kx * U0[0, 1, 0, 1] + 1j * kz * U0[2, 1, 0, 1]) < 1e-12 * abs(U0[0, 1, 0, 1])
    U, T = U0.copy(), T0.copy()
    for _ in range(20):
        U, T = R.rbc_rk4_step(cfg, U, T)
    growth = math.exp(sigma * 20 * cfg.dt)
    assert abs(growth - 1) > 1e-4   # the state moved
    if pr == "PRZERO":
        assert abs(U[0, 1, 0, 1] - growth * eps) < 1e-7 * eps
        assert np.array_equal(T, R.reality_fix(g, R.rbc_slave_temperature(g, U)))
    else:
        assert abs(T[1, 0, 1] - growth * eps) < 1e-7 * eps
        assert np.array_equal(U, R.reality_fix_vec(g, R.rbc_slave_velocity(g, T, co["vs"])))
    assert R.nusselt(cfg, U, T) == co["nu0"] + co["nuc"] * R.cross_energy(g, U[0], T)


def test_rbc_slaved_critical_rayleigh_number():
    """Free-slip Rayleigh-Benard onset at infinite and zero Prandtl number (USMALL units):
    growth rate Ra kperp^2 / K^4 - K^2 changes sign at Ra_c = K^6 / kperp^2 = 27 pi^4 / 4 for the
    roll kx = pi, kperp = pi / sqrt(2).  Below Ra_c the oracle's roll decays, above it grows."""
    kp = math.pi / math.sqrt(2)
    kf = (math.pi, kp, kp)
    g = R.Grid((16, 8, 8), kf, "SFF")
    Rac = 27 * math.pi ** 4 / 4
    for pr in ("PRZERO", "PRINFTY"):
        for Ra, grows in ((0.95 * Rac, False), (1.05 * Rac, True)):
            cfg = R.RBCConfig(g, Ra=Ra, Pr=1.0, dt=1e-4, pr_option=pr, uscaling="USMALL")
            T0 = np.zeros(g.shape, complex)
            T0[1, 0, 1] = 1e-9
            U0 = R.rbc_slave_velocity(g, T0, cfg.coeffs["vs"]) if pr == "PRINFTY" else None
            if pr == "PRZERO":
                U0 = np.zeros((3,) + g.shape, complex)
                U0[0, 1, 0, 1] = 1e-9
                U0[2, 1, 0, 1] = 1j * math.pi * 1e-9 / kp
                T0 = R.rbc_slave_temperature(g, U0)
            U, T = U0, T0
            for _ in range(5):
                U, T = R.rbc_rk4_step(cfg, U, T)
            a = abs(U[0, 1, 0, 1] / U0[0, 1, 0, 1]) if pr == "PRZERO" else abs(T[1, 0, 1] / T0[1, 0, 1])
            assert (a > 1) == grows, (pr, Ra, a)
