"""Reading reference-format run inputs (para.yaml, forcing.txt) and writing the
reference's text outputs (spectrum.d, flux.d, glob.d).  The gpu-marked tests step
runs built from a para.yaml (the fluid on FFF, SSF and SSS, MHD, the passive
scalar) and write outputs on the GPU against the oracle."""
import io
import math
import os

import numpy as np
import pytest

from tarang_b200 import para

HERE = os.path.dirname(os.path.abspath(__file__))
FFF_DIR = os.path.join(HERE, "golden", "para_fff")
RBC_DIR = os.path.join(HERE, "golden", "para_rbc")
KIND_DIRS = {k: os.path.join(HERE, "golden", f"para_{k}") for k in ("mhd", "scalar", "ssf", "sss", "rbc_sss", "rbc_2d")}


def test_read_para_fff_forced():
    rp = para.read_para(os.path.join(FFF_DIR, "in", "para.yaml"))
    assert (rp.kind, rp.basis, rp.N, rp.kfactor) == ("FLUID_INCOMPRESS", "FFF", (32, 32, 32), (1.0, 1.0, 1.0))
    assert rp.dealias == "reference" and rp.reality_fix
    assert rp.nu == 0.01 and rp.dt == 0.001 and rp.nsteps == 4
    assert rp.force_on and (rp.force_inner, rp.force_outer) == (2.0, 3.0) and not rp.force_global_alpha_beta
    # no radii given: the reference's default spheres for 8 spheres and max radius 16
    assert rp.flux_radii == [0.0, 2.0, 4.0, 8.0, 8.0, 8.0, 8.0, 16.0, para.INF_RADIUS]


def test_read_para_rbc_from_L():
    rp = para.read_para(os.path.join(RBC_DIR, "in", "para.yaml"))
    assert rp.kind == "RBC" and rp.basis == "SFF" and rp.N == (32, 16, 16)
    # L = (1, 2, 2): pi / L along the sin/cos direction, 2 pi / L along the Fourier ones
    assert np.allclose(rp.kfactor, (math.pi, math.pi, math.pi))
    assert rp.Ra == 1e5 and rp.Pr == 2.0
    assert math.isclose(rp.nu, math.sqrt(2.0 / 1e5)) and math.isclose(rp.kappa, 1.0 / math.sqrt(2e5))
    assert rp.nsteps == 100 and not rp.force_on


def test_read_para_other_kinds():
    """MHD and the passive scalar on FFF take [nu, eta] / [nu, kappa]; decay (field_procedure 0,
    or a procedure with every switch off) is unforced; SSF / SSS fluids default kfactor to 1."""
    rp = para.read_para(os.path.join(KIND_DIRS["mhd"], "in", "para.yaml"))
    assert (rp.kind, rp.basis, rp.N) == ("MHD_INCOMPRESS", "FFF", (32, 16, 32))
    assert (rp.nu, rp.kappa, rp.nsteps, rp.force_on, rp.reality_fix) == (0.01, 0.02, 3, False, True)
    rp = para.read_para(os.path.join(KIND_DIRS["scalar"], "in", "para.yaml"))
    assert (rp.kind, rp.N, rp.nu, rp.kappa, rp.nsteps) == ("SCALAR_INCOMPRESS", (32, 32, 16), 0.01, 0.03, 3)
    assert np.allclose(rp.kfactor, (1.0, 2.0, 1.0)) and rp.t_init == 0.5 and not rp.force_on
    rp = para.read_para(os.path.join(KIND_DIRS["ssf"], "in", "para.yaml"))
    assert (rp.kind, rp.basis, rp.kfactor, rp.nu, rp.nsteps) == ("FLUID_INCOMPRESS", "SSF", (1.0, 1.0, 1.0), 0.02, 3)
    rp = para.read_para(os.path.join(KIND_DIRS["sss"], "in", "para.yaml"))
    assert (rp.basis, rp.N, rp.kfactor, rp.dealias) == ("SSS", (16, 32, 16), (1.0, 1.0, 1.0), "reference")
    rp = para.read_para(os.path.join(KIND_DIRS["rbc_2d"], "in", "para.yaml"))
    assert (rp.kind, rp.basis, rp.N) == ("RBC", "SFF", (32, 1, 32))
    rp = para.read_para(os.path.join(KIND_DIRS["rbc_sss"], "in", "para.yaml"))
    assert (rp.kind, rp.basis, rp.Ra, rp.Pr, rp.nsteps, rp.force_on) == ("RBC", "SSS", 2e4, 0.7, 3, False)
    assert np.allclose(rp.kfactor, (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0)))
    assert math.isclose(rp.nu, math.sqrt(0.7 / 2e4)) and math.isclose(rp.kappa, 1 / math.sqrt(0.7 * 2e4))
    assert [para.n_fields(k) for k in ("FLUID_INCOMPRESS", "RBC", "SCALAR_INCOMPRESS", "MHD_INCOMPRESS")] == [1, 2, 2, 2]
    with pytest.raises(ValueError):
        para.advance(None, "MHD_INCOMPRESS", (None,), 1)


@pytest.mark.parametrize("kind,basis,force", [("FLUID_INCOMPRESS", "SSF", "U_switch: true\n  field_procedure: [1]"),
                                              ("MHD_INCOMPRESS", "FFF", "W_switch: true\n  field_procedure: 2"),
                                              ("FLUID_INCOMPRESS", "FFF", "T_switch: true\n  field_procedure: [1]"),
                                              ("SCALAR_INCOMPRESS", "SFF", "U_switch: false")])
def test_read_para_refuses_forcings_and_bases(tmp_path, kind, basis, force):
    f = tmp_path / "para.yaml"
    f.write_text(f"program:\n  kind: {kind}\n  basis_type: {basis}\nfield:\n  N: [8,8,8]\n"
                 f"time:\n  dt_fixed: 0.1\n  final: 1\nforce:\n  {force}\n")
    with pytest.raises(NotImplementedError):
        para.read_para(str(f))


def test_default_flux_radii_geometric():
    r = para.default_flux_radii(10, 64)
    assert r[:4] == [0.0, 2.0, 4.0, 8.0]
    assert r[8] == 32.0 and r[9] == 64.0 and r[10] == para.INF_RADIUS
    s = math.log2(64 / 16.0) / 5
    assert np.allclose(r[4:8], [8 * 2 ** (s * (i - 3)) for i in range(4, 8)])
    assert all(r[i] <= r[i + 1] for i in range(10))


def test_blitz_arrays_and_unsupported(tmp_path):
    arrs = para.read_blitz_arrays(os.path.join(FFF_DIR, "in", "forcing.txt"))
    assert len(arrs) == 2 and arrs[0].shape == (7,) and arrs[0][3] == 0.1 and not arrs[1].any()
    bad = tmp_path / "para.yaml"
    bad.write_text("program:\n  kind: MHD_INCOMPRESS\n  basis_type: SFF\nfield:\n  N: [8,8,8]\ntime:\n  dt_fixed: 0.1\n  final: 1\n")
    with pytest.raises(NotImplementedError):
        para.read_para(str(bad))
    (tmp_path / "b").write_text("(0,2)\n[ 1 2 ]\n")
    with pytest.raises(ValueError):
        para.read_blitz_arrays(str(tmp_path / "b"))


def test_output_layouts():
    f = io.StringIO()
    ek = [np.arange(4.0), np.arange(4.0) + 1, np.arange(4.0) + 2]
    para.write_spectrum(f, 0.5, ek, [2 * e for e in ek], [3 * e for e in ek])
    lines = f.getvalue().split("\n")
    # 14 lines per time block (+ the empty string after the last newline), as the reference writes them
    assert len(lines) == 15 and lines[-1] == ""
    assert lines[0] == "%% Time = 0.5" and lines[1] == " " and lines[2] == "%%Uek" and lines[6] == "%%UDk"
    assert lines[10] == "%%(Fv.v)(k)"
    assert lines[3] == "0\t1\t2\t3\t" and [float(x) for x in lines[13].split("\t")[:-1]] == [6, 9, 12, 15]
    g = io.StringIO()
    para.write_flux(g, 1.25, [0.0, 0.1, 0.25])
    assert g.getvalue() == "\n%% Time = 1.25\n%%flux: U2U \n0\t0.1\t0.25\t\n"
    h = io.StringIO()
    para.write_glob_row(h, [0.1, 0.5, 2e-3, 1e-3])
    assert h.getvalue() == "0.1\t0.5\t0.002\t0.001\t\n"


@pytest.mark.gpu
def test_plan_from_para_steps_like_the_oracle(cuda):
    """A forced FFF run set up from para.yaml + forcing.txt matches the oracle over its 4 steps."""
    import torch
    from oracle import tarang_ref as R
    plan, rp = para.plan_from_dir(FFF_DIR, precision="f64")
    g = R.Grid(rp.N, rp.kfactor)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    es = para.read_blitz_arrays(os.path.join(FFF_DIR, "in", "forcing.txt"))[0]
    cfg = R.FluidConfig(g, nu=rp.nu, dt=rp.dt, dealias_mode=1, forcing=R.CaratiForcing(rp.force_inner, rp.force_outer, es))
    W = V.copy()
    for _ in range(rp.nsteps):
        W = R.rk4_step(cfg, W)
    u = torch.from_numpy(V.copy()).to(cuda)
    plan.rk4_step(u, rp.nsteps)
    torch.cuda.synchronize()
    d = u.cpu().numpy() - W
    assert np.linalg.norm(d) / np.linalg.norm(W) < 1e-12


def _kind_state(g, kind, basis):
    """a seeded oracle state for a run of this kind: (U,), (U, T) or (U, B)"""
    from oracle import tarang_ref as R
    rng = np.random.default_rng(11)
    if basis in ("SSF", "SSS"):
        par = R.SSF_PARITY if basis == "SSF" else R.SSS_PARITY
        U = np.stack([R.forward(g, rng.standard_normal(g.rshape), par[v]) for v in ("Vx", "Vy", "Vz")])
        U = -0.3 * R.project_rhs(g, U)
        if kind == "RBC":
            return U, 0.3 * R.forward(g, rng.standard_normal(g.rshape), par["F"])
        return (U,)
    if basis == "SFF":
        # sin/cos parities along x (u1, T sine; u2, u3 cosine); u2 = 0 in a two-dimensional run
        U = np.stack([R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), p)) for p in "SCC"])
        if g.N[1] == 1:
            U[1] = 0
        return U, R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), "S"))
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    if kind == "MHD_INCOMPRESS":
        return U, R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 3.0), 1, 0.3)
    return U, R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape)))


def _kind_oracle(g, rp, state):
    from oracle import tarang_ref as R
    out = [s.copy() for s in state]
    for _ in range(rp.nsteps):
        if rp.kind == "FLUID_INCOMPRESS":
            out = [R.rk4_step(R.FluidConfig(g, nu=rp.nu, dt=rp.dt, dealias_mode=1, nlin_form="conservative"), out[0])]
        elif rp.kind == "RBC":
            out = list(R.rbc_rk4_step(R.RBCConfig(g, Ra=rp.Ra, Pr=rp.Pr, dt=rp.dt, dealias_mode=1), *out))
        elif rp.kind == "MHD_INCOMPRESS":
            out = list(R.mhd_rk4_step(R.MHDConfig(g, nu=rp.nu, eta=rp.kappa, dt=rp.dt, dealias_mode=1), *out))
        else:
            out = list(R.rbc_rk4_step(R.ScalarConfig(g, nu=rp.nu, kappa=rp.kappa, dt=rp.dt, dealias_mode=1), *out))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mhd", "scalar", "ssf", "sss", "rbc_sss", "rbc_2d"])
def test_plan_from_para_other_kinds_step_like_the_oracle(cuda, name):
    """MHD, passive-scalar, SSF and SSS fluid, SSS RBC and two-dimensional SFF RBC
    (Ny = 1) runs set up from a para.yaml,
    stepped through para.advance, match the FP64 oracle over the run's 3 steps
    (relative L2 <= 1e-12)."""
    import torch
    from oracle import tarang_ref as R
    plan, rp = para.plan_from_dir(KIND_DIRS[name], precision="f64")
    g = R.Grid(rp.N, rp.kfactor, rp.basis)
    state = _kind_state(g, rp.kind, rp.basis)
    want = _kind_oracle(g, rp, state)
    Nz = rp.N[2]
    if rp.basis == "SSS":
        # real coefficients in the padded real layout (Nx, Ny, Nz + 2), viewed as complex
        fields = []
        for s in state:
            pad = np.zeros(s.shape[:-1] + (Nz + 2,))
            pad[..., :Nz] = s
            fields.append(torch.from_numpy(pad.view(np.complex128)).to(cuda))
    else:
        fields = [torch.from_numpy(s.copy()).to(cuda) for s in state]
    para.advance(plan, rp.kind, fields, rp.nsteps)
    plan.status()
    for f, w in zip(fields, want):
        got = f.cpu().numpy()
        if rp.basis == "SSS":
            got = got.view(np.float64)[..., :Nz]
        assert np.linalg.norm(got - w) / np.linalg.norm(w) < 1e-12


def _read_blocks(path, label):
    """Rows under %%label in every time block of a reference text output."""
    rows, cur = [], None
    for line in open(path).read().split("\n"):
        if line.startswith("%%"):
            cur = line[2:] == label
            if cur:
                rows.append([])
            continue
        if cur and line.strip():
            rows[-1].append(np.array([float(x) for x in line.split("\t")[:-1]]))
    return rows


@pytest.mark.gpu
def test_output_spectrum_and_flux_match_oracle(cuda, tmp_path):
    """spectrum.d / flux.d written from a forced 32^3 state against the oracle's quantities."""
    import torch
    from oracle import tarang_ref as R
    plan, rp = para.plan_from_dir(FFF_DIR, precision="f64")
    g = R.Grid(rp.N, rp.kfactor)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    u = torch.from_numpy(V.copy()).to(cuda)
    out = para.Output(plan, str(tmp_path), radii=rp.flux_radii)
    out.spectrum(u, 0.0)
    out.flux(u, 0.0)
    # oracle quantities
    Kmag = g.Kmag()
    idx = np.ceil(Kmag).astype(int)
    mult = g.multiplicity()
    nsh = g.n_shells()
    ok = idx < nsh
    cnt = np.bincount(idx[ok], weights=2 * mult[ok], minlength=nsh)
    kin = para.max_radius_inside(rp.N, rp.kfactor)
    sh = np.arange(nsh)
    es = para.read_blitz_arrays(os.path.join(FFF_DIR, "in", "forcing.txt"))[0]
    F = R.carati_force(g, V, R.CaratiForcing(rp.force_inner, rp.force_outer, es), g.modes_in_shell())
    ek = _read_blocks(tmp_path / "spectrum.d", "Uek")[0]
    ud = _read_blocks(tmp_path / "spectrum.d", "UDk")[0]
    fv = _read_blocks(tmp_path / "spectrum.d", "(Fv.v)(k)")[0]
    for i in range(3):
        ref = R.shell_spectrum(g, V[i:i + 1])
        assert np.allclose(ek[i], ref, rtol=2e-5, atol=1e-6 * ref.max())
        raw = np.bincount(idx[ok], weights=(mult * Kmag ** 2 * np.abs(V[i]) ** 2)[ok], minlength=nsh)
        beyond = (sh > kin) & (cnt >= 1)
        raw[beyond] *= (4 * np.pi * sh[beyond] ** 2) / cnt[beyond]
        assert np.allclose(ud[i], 2 * raw, rtol=2e-5, atol=1e-6 * raw.max())
        cr = np.bincount(idx[ok], weights=(mult * Kmag ** 2 * (V[i] * np.conj(F[i])).real)[ok], minlength=nsh)
        ref_f = 2 * np.where(cnt > 0, cr * 4 * np.pi / np.where(cnt > 0, cnt, 1), 0.0)
        assert np.allclose(fv[i], ref_f, rtol=2e-5, atol=1e-6 * np.abs(ref_f).max())
    flux = _read_blocks(tmp_path / "flux.d", "flux: U2U ")[0][0]
    # the reference's per-sphere algorithm (corner-box dealiasing), with radii[0] never computed
    ref_pi = R.flux_per_sphere(g, V, rp.flux_radii, 1)
    ref_pi[0] = 0.0
    # flux.d holds %g values (six significant digits, Print_array)
    assert np.allclose(flux, ref_pi, rtol=2e-5, atol=1e-9)
    # Compute_flux dealiases U in place, and so does the output
    assert np.array_equal(u.cpu().numpy(), R.dealias(g, V, 1))
    power = _read_blocks(tmp_path / "flux.d", "sum(Fv.v)")[0][0]
    dot = 2 * mult * np.sum((F * np.conj(V)).real, axis=0)
    ins = Kmag <= kin
    b = np.searchsorted(np.asarray(rp.flux_radii), Kmag[ins], side="left")
    ref_p = np.zeros(len(rp.flux_radii))
    np.add.at(ref_p, b, dot[ins])
    assert np.allclose(power, ref_p, rtol=2e-5, atol=1e-9)
    # the total power equals the energy injection 2 sum mult Re(F.u*) = epsilon (0.1) up to 6 digits
    assert abs(power.sum() - 0.1) < 1e-5


@pytest.mark.gpu
def test_output_glob_matches_oracle(cuda, tmp_path):
    """glob.d row (FluidIO::Output_global) from a 32^3 state against numpy sums of the oracle field."""
    import torch
    from oracle import tarang_ref as R
    plan, rp = para.plan_from_dir(FFF_DIR, precision="f64")
    g = R.Grid(rp.N, rp.kfactor)
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    u = torch.from_numpy(V.copy()).to(cuda)
    out = para.Output(plan, str(tmp_path), radii=rp.flux_radii)
    row = out.glob(u, 0.25, 5e-4, helicity=True)
    text = open(tmp_path / "glob.d").read().split("\n")[0].split("\t")[:-1]
    assert len(text) == 15
    mult = g.multiplicity()
    Kx, Ky, Kz = g.K()
    K2 = g.Ksqr()
    E = [float(np.sum(mult * np.abs(V[i]) ** 2)) for i in range(3)]
    Et = E[0] + E[1] + E[2]
    k2 = 2 * float(np.sum(mult * K2 * np.sum(np.abs(V) ** 2, axis=0)))
    nu = plan.cfg.nu
    eps = nu * k2
    cr = np.cross(V.real, V.imag, axis=0)
    h = 2 * mult * (Kx * cr[0] + Ky * cr[1] + Kz * cr[2])
    H1 = float(h.sum())
    H2 = float(np.where(K2 > 1e-15, h / np.where(K2 > 1e-15, K2, 1), 0).sum())
    modal = mult * np.sum(np.abs(V) ** 2, axis=0)
    p = modal / Et
    ent = float(np.where(p > 1e-15, -p * np.log2(np.where(p > 1e-15, p, 1)), 0).sum())
    kin = para.max_radius_inside(rp.N, rp.kfactor)
    ref = [0.25, Et, eps, H1, H2, 2 * float((K2 * h).sum()), 2 * H1, ent, kin * (nu ** 3 / eps) ** 0.25, nu,
           2 * Et * math.sqrt(15 / eps), 5e-4, E[0], E[1], E[2]]
    for a, b in zip(row, ref):
        assert abs(a - b) <= 1e-10 * max(1.0, abs(b))
    for a, b in zip(text, ref):
        assert abs(float(a) - b) <= 1e-5 * max(1e-12, abs(b))


@pytest.mark.gpu
def test_output_glob_rbc_matches_oracle(cuda, tmp_path):
    """glob.d for an RBC run on SFF (Output_global_RBC's 21 columns) against numpy sums of
    the oracle fields: energies, k^2 energies (SFF multiplicity), Nusselt, entropies,
    kmax eta_1 / eta_2, R_lambda and the component energies (relative 1e-10, FP64)."""
    import torch
    import tarang_b200 as tb
    from oracle import tarang_ref as R
    N, kf, Ra, Pr = (32, 16, 16), (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0)), 2e5, 0.7
    g = R.Grid(N, kf, "SFF")
    rng = np.random.default_rng(21)
    U = np.stack([R.reality_fix(g, 0.3 * R.forward(g, rng.standard_normal(g.rshape), p)) for p in ("S", "C", "C")])
    T = R.reality_fix(g, 0.2 * R.forward(g, rng.standard_normal(g.rshape), "S"))
    cfg = R.RBCConfig(g, Ra=Ra, Pr=Pr, dt=1e-3)
    plan = tb.Plan(N, basis="SFF", kfactor=kf, nu=cfg.nu, kappa=cfg.kappa, Ra=Ra, Pr=Pr, dt=1e-3)
    out = para.Output(plan, str(tmp_path))
    row = out.glob_rbc(torch.from_numpy(U).to(cuda), torch.from_numpy(T[None]).to(cuda), 0.25, 1e-3)
    # numpy restatement
    lx = np.arange(N[0])[:, None, None]
    ky = np.fft.fftfreq(N[1], 1.0 / N[1])[None, :, None]
    lz = np.arange(N[2] // 2 + 1)[None, None, :]
    mult = np.where(lz > 0, np.where(lx > 0, 2.0, 1.0), np.where(lx > 0, 1.0, 0.5))
    mult = mult * np.where(np.abs(ky) == N[1] // 2, 2.0, 1.0)
    K2 = (lx * kf[0]) ** 2 + (ky * kf[1]) ** 2 + (lz * kf[2]) ** 2
    Eu, ET = R.total_energy(g, U), R.total_energy_scalar(g, T)
    eps = cfg.nu * 2 * (mult * K2 * (np.abs(U) ** 2).sum(0)).sum()
    epsT = cfg.kappa * 2 * (mult * K2 * np.abs(T) ** 2).sum()

    def ent(a2, e):
        pr = mult * a2 / e
        pr = pr[pr > 1e-15]
        return float((-pr * np.log(pr) / np.log(2.0)).sum())

    kmax = int(min((N[0] - 1) * kf[0], (N[1] // 2) * kf[1], (N[2] // 2) * kf[2]))
    k1 = kmax * (cfg.nu ** 3 / eps) ** 0.25
    r = cfg.nu / cfg.kappa
    want = [0.25, Eu, ET, eps, epsT, R.nusselt(cfg, U, T), 0, 0, 0, 0, ent((np.abs(U) ** 2).sum(0), Eu),
            ent(np.abs(T) ** 2, ET), k1, k1 * r ** 0.25 / r, cfg.nu, cfg.kappa, 2 * Eu * math.sqrt(15 / eps), 1e-3,
            R.total_energy(g, U[:1]), R.total_energy(g, U[1:2]), R.total_energy(g, U[2:])]
    assert len(row) == 21
    for i, (a, b) in enumerate(zip(row, want)):
        assert abs(a - b) <= max(1e-10 * abs(b), 1e-12), (i, a, b)
    line = open(tmp_path / "glob.d").read()
    assert line.endswith("\t\n") and len(line.split("\t")) == 22


@pytest.mark.gpu
@pytest.mark.parametrize("basis", ["SSF", "SSS"])
def test_output_glob_rbc_ssf_sss_matches_oracle(cuda, tmp_path, basis):
    """glob.d for RBC runs on SSF and SSS (the same 21 columns): the k^2 sums and entropies
    over the complex array shape with the sin/cos multiplicity (on SSS the real pair of a z
    slot with Kz = lz kfactor_z, as the reference's universal loops take it), Max_radius_inside
    of the basis, energies and Nusselt from the oracle (relative 1e-10, FP64)."""
    import torch
    import tarang_b200 as tb
    from oracle import tarang_ref as R
    N, kf, Ra, Pr = (16, 32, 16), (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0)), 3e4, 0.7
    g = R.Grid(N, kf, basis)
    par = R.SSF_PARITY if basis == "SSF" else R.SSS_PARITY
    rng = np.random.default_rng(23)
    U = np.stack([0.3 * R.forward(g, rng.standard_normal(g.rshape), par[v]) for v in ("Vx", "Vy", "Vz")])
    T = 0.2 * R.forward(g, rng.standard_normal(g.rshape), par["F"])
    cfg = R.RBCConfig(g, Ra=Ra, Pr=Pr, dt=1e-3)
    plan = tb.Plan(N, basis=basis, kfactor=kf, nu=cfg.nu, kappa=cfg.kappa, Ra=Ra, Pr=Pr, dt=1e-3)
    if basis == "SSS":
        def dev(a):
            pad = np.zeros(a.shape[:-1] + (N[2] + 2,))
            pad[..., :N[2]] = a
            return torch.from_numpy(pad.view(np.complex128)).to(cuda)
        Uc = np.stack([R.sss_complex_view(g, U[i])[0] for i in range(3)])
        Tc, gc = R.sss_complex_view(g, T)
        mult, K2 = R._sss_mult(gc), gc.Ksqr()
    else:
        def dev(a):
            return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
        Uc, Tc, mult, K2 = U, T, g.multiplicity(), g.Ksqr()
    out = para.Output(plan, str(tmp_path))
    row = out.glob_rbc(dev(U), dev(T[None]), 0.5, 1e-3)
    Eu, ET = R.total_energy(g, U), R.total_energy_scalar(g, T)
    eps = cfg.nu * 2 * (mult * K2 * (np.abs(Uc) ** 2).sum(0)).sum()
    epsT = cfg.kappa * 2 * (mult * K2 * np.abs(Tc) ** 2).sum()

    def ent(a2, e):
        pr = mult * a2 / e
        pr = pr[pr > 1e-15]
        return float((-pr * np.log(pr) / np.log(2.0)).sum())

    third = (N[2] // 2) * kf[2] if basis == "SSF" else (N[1] - 1) * kf[2]
    kmax = int(min((N[0] - 1) * kf[0], (N[1] - 1) * kf[1], third))
    k1 = kmax * (cfg.nu ** 3 / eps) ** 0.25
    r = cfg.nu / cfg.kappa
    want = [0.5, Eu, ET, eps, epsT, R.nusselt(cfg, U, T), 0, 0, 0, 0, ent((np.abs(Uc) ** 2).sum(0), Eu),
            ent(np.abs(Tc) ** 2, ET), k1, k1 * r ** 0.25 / r, cfg.nu, cfg.kappa, 2 * Eu * math.sqrt(15 / eps), 1e-3,
            R.total_energy(g, U[:1]), R.total_energy(g, U[1:2]), R.total_energy(g, U[2:])]
    assert len(row) == 21
    for i, (a, b) in enumerate(zip(row, want)):
        assert abs(a - b) <= max(1e-10 * abs(b), 1e-12), (i, a, b)


@pytest.mark.gpu
def test_output_flux_ssf_matches_oracle(cuda, tmp_path):
    """flux.d of an SSF fluid run (the reference's per-sphere flux on the SSF basis, the
    default radii from SSF's Max_radius_inside, radii[0] never computed) against the oracle,
    and U dealiased in place as Compute_nlin(U, Giver) leaves it."""
    import torch
    from oracle import tarang_ref as R
    plan, rp = para.plan_from_dir(KIND_DIRS["ssf"], precision="f64")
    g = R.Grid(rp.N, rp.kfactor, rp.basis)
    (U,) = _kind_state(g, rp.kind, rp.basis)
    u = torch.from_numpy(U.copy()).to(cuda)
    out = para.Output(plan, str(tmp_path))
    out.flux(u, 0.0)
    flux = _read_blocks(tmp_path / "flux.d", "flux: U2U ")[0][0]
    ref = R.flux_per_sphere(g, U, out.radii, 1)
    ref[0] = 0.0
    assert len(out.radii) == len(flux)
    assert np.allclose(flux, ref, rtol=2e-5, atol=1e-9 * np.abs(ref).max())
    assert np.array_equal(u.cpu().numpy(), R.dealias(g, U, 1))


def _helicity_np(V, kx, ky, kz, mult):
    """H1, H2, k2H1, k2H2 on FFF with kfactor 1: h = 2 mult K . (Vr x Vi)"""
    cr = np.cross(V.real, V.imag, axis=0)
    h = 2 * mult * (kx * cr[0] + ky * cr[1] + kz * cr[2])
    K2 = kx ** 2 + ky ** 2 + kz ** 2
    H1 = float(h.sum())
    return [H1, float(np.where(K2 > 1e-15, h / np.where(K2 > 1e-15, K2, 1.0), 0.0).sum()),
            2 * float((K2 * h).sum()), 2 * H1]


@pytest.mark.gpu
def test_output_glob_scalar_matches_oracle(cuda, tmp_path):
    """glob.d for a passive-scalar run on FFF (Output_global_scalar's 20 columns: the RBC row
    without Nusselt) with the FFF multiplicity, against numpy sums of the oracle fields."""
    import torch
    import tarang_b200 as tb
    from oracle import tarang_ref as R
    N, nu, kappa = (32, 16, 32), 0.01, 0.03
    g = R.Grid(N)
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 2, 0.5)
    T = R.reality_fix(g, 0.2 * R.forward(g, np.random.default_rng(22).standard_normal(g.rshape)))
    plan = tb.Plan(N, nu=nu, kappa=kappa, dt=1e-3)
    out = para.Output(plan, str(tmp_path))
    row = out.glob_scalar(torch.from_numpy(U).to(cuda), torch.from_numpy(T[None]).to(cuda), 1.5, 1e-3, helicity=True)
    kx = np.fft.fftfreq(N[0], 1.0 / N[0])[:, None, None]
    ky = np.fft.fftfreq(N[1], 1.0 / N[1])[None, :, None]
    kz = np.arange(N[2] // 2 + 1)[None, None, :]
    mult = np.where(kz > 0, 1.0, 0.5) * np.where((np.abs(kx) == N[0] // 2) | (np.abs(ky) == N[1] // 2), 2.0, 1.0)
    K2 = kx ** 2 + ky ** 2 + kz ** 2
    Eu, ET = R.total_energy(g, U), R.total_energy_scalar(g, T)
    eps = nu * 2 * (mult * K2 * (np.abs(U) ** 2).sum(0)).sum()
    epsT = kappa * 2 * (mult * K2 * np.abs(T) ** 2).sum()

    def ent(a2, e):
        pr = mult * a2 / e
        pr = pr[pr > 1e-15]
        return float((-pr * np.log(pr) / np.log(2.0)).sum())

    kmax = para.max_radius_inside(N, (1.0, 1.0, 1.0))
    k1 = kmax * (nu ** 3 / eps) ** 0.25
    r = nu / kappa
    want = [1.5, Eu, ET, eps, epsT] + _helicity_np(U, kx, ky, kz, mult) + [ent((np.abs(U) ** 2).sum(0), Eu),
                                                                         ent(np.abs(T) ** 2, ET), k1,
            k1 * r ** 0.25 / r, nu, kappa, 2 * Eu * math.sqrt(15 / eps), 1e-3,
            R.total_energy(g, U[:1]), R.total_energy(g, U[1:2]), R.total_energy(g, U[2:])]
    assert len(row) == 20
    for i, (a, b) in enumerate(zip(row, want)):
        assert abs(a - b) <= max(1e-10 * abs(b), 1e-12), (i, a, b)


@pytest.mark.gpu
def test_output_glob_mhd_matches_oracle(cuda, tmp_path):
    """glob.d for an MHD run on FFF (Output_global(U, W)'s 29 columns: energies,
    dissipations, cross helicity and its dissipation, entropies, kmax eta_1 / eta_2,
    R_lambda, component energies) against numpy sums of the oracle fields."""
    import torch
    import tarang_b200 as tb
    from oracle import tarang_ref as R
    N, nu, eta = (32, 32, 16), 0.01, 0.02
    g = R.Grid(N)
    U = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 3, 0.5)
    B = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 3.0), 4, 0.3)
    plan = tb.Plan(N, nu=nu, kappa=eta, dt=1e-3)
    out = para.Output(plan, str(tmp_path))
    row = out.glob_mhd(torch.from_numpy(U).to(cuda), torch.from_numpy(B).to(cuda), 2.0, 1e-3, helicity=True)
    kx = np.fft.fftfreq(N[0], 1.0 / N[0])[:, None, None]
    ky = np.fft.fftfreq(N[1], 1.0 / N[1])[None, :, None]
    kz = np.arange(N[2] // 2 + 1)[None, None, :]
    mult = np.where(kz > 0, 1.0, 0.5) * np.where((np.abs(kx) == N[0] // 2) | (np.abs(ky) == N[1] // 2), 2.0, 1.0)
    K2 = kx ** 2 + ky ** 2 + kz ** 2
    Eu, Eb = R.total_energy(g, U), R.total_energy(g, B)
    Hc = sum(R.cross_energy(g, U[i], B[i]) for i in range(3))
    eps = nu * 2 * (mult * K2 * (np.abs(U) ** 2).sum(0)).sum()
    epsb = eta * 2 * (mult * K2 * (np.abs(B) ** 2).sum(0)).sum()
    k2Hc = 2 * (mult * K2 * (U * B.conj()).real.sum(0)).sum()

    def ent(a2, e):
        pr = mult * a2 / e
        pr = pr[pr > 1e-15]
        return float((-pr * np.log(pr) / np.log(2.0)).sum())

    kmax = para.max_radius_inside(N, (1.0, 1.0, 1.0))
    k1 = kmax * (nu ** 3 / eps) ** 0.25
    r = nu / eta
    hu, hb = _helicity_np(U, kx, ky, kz, mult), _helicity_np(B, kx, ky, kz, mult)
    want = ([2.0, Eu, Eb, eps, epsb, Hc, 0.5 * (nu + eta) * k2Hc] + hu[:2] + hb[:2] + hu[2:] + hb[2:] +
            [ent((np.abs(U) ** 2).sum(0), Eu), ent((np.abs(B) ** 2).sum(0), Eb), k1, k1 * r ** 0.25 / r, nu, eta,
             2 * Eu * math.sqrt(15 / eps), 1e-3] +
            [R.total_energy(g, U[i:i + 1]) for i in range(3)] + [R.total_energy(g, B[i:i + 1]) for i in range(3)])
    assert len(row) == 29
    for i, (a, b) in enumerate(zip(row, want)):
        assert abs(a - b) <= max(1e-10 * abs(b), 1e-12), (i, a, b)


# ---------------------------------------------------------------------------
# restart: complex-field checkpoints (Cvf.cc:494-528) and input_field_procedure 1
# ---------------------------------------------------------------------------
def _fake_plan(N=(16, 8, 12), basis="FFF", precision="f64", kf=(1.0, 2.0, 1.0)):
    from types import SimpleNamespace
    return SimpleNamespace(N=N, basis=basis, precision=precision,
                           cfg=SimpleNamespace(kfactor=list(kf), dt=1e-3))


@pytest.mark.parametrize("kind", ["FLUID_INCOMPRESS", "RBC", "MHD_INCOMPRESS"])
def test_state_round_trip_bit_exact(tmp_path, kind):
    """save_state -> load_state returns the same bits; one raw file per component named as the
    reference's datasets (U.V1 ... T.F, W.V1 ...), plus the JSON header."""
    import json
    import torch
    plan = _fake_plan()
    g = torch.Generator().manual_seed(5)
    shape = (16, 8, 7)
    fields = [torch.complex(torch.randn((len(c),) + shape, generator=g, dtype=torch.float64),
                            torch.randn((len(c),) + shape, generator=g, dtype=torch.float64))
              for _, c in para.field_layout(kind)]
    para.save_state(str(tmp_path / "s"), plan, kind, fields, 0.25, 250)
    head = json.load(open(tmp_path / "s" / "state.json"))
    assert head["t"] == 0.25 and head["step"] == 250 and head["N"] == [16, 8, 12] and head["precision"] == "f64"
    names = sorted(f["file"] for f in head["files"])
    want = {"FLUID_INCOMPRESS": ["U.V1.bin", "U.V2.bin", "U.V3.bin"],
            "RBC": ["T.F.bin", "U.V1.bin", "U.V2.bin", "U.V3.bin"],
            "MHD_INCOMPRESS": ["U.V1.bin", "U.V2.bin", "U.V3.bin", "W.V1.bin", "W.V2.bin", "W.V3.bin"]}[kind]
    assert names == want
    # component files hold the component's C-order array, little endian
    raw = np.fromfile(tmp_path / "s" / "U.V2.bin", dtype="<c16").reshape(shape)
    assert np.array_equal(raw, fields[0][1].numpy())
    back, t, step = para.load_state(str(tmp_path / "s"), plan, kind, device="cpu")
    assert (t, step) == (0.25, 250)
    for a, b in zip(back, fields):
        assert torch.equal(a, b)
    # an FP64 state into an FP32 run is rounded once
    back32, _, _ = para.load_state(str(tmp_path / "s"), _fake_plan(precision="f32"), kind, device="cpu")
    assert torch.equal(back32[0], fields[0].to(torch.complex64))


def test_state_refuses_other_geometry_and_kind(tmp_path):
    import torch
    plan = _fake_plan()
    u = torch.zeros((3, 16, 8, 7), dtype=torch.complex128)
    para.save_state(str(tmp_path / "s"), plan, "FLUID_INCOMPRESS", [u], 0.0)
    with pytest.raises(ValueError):
        para.load_state(str(tmp_path / "s"), _fake_plan(N=(16, 8, 16)), "FLUID_INCOMPRESS", device="cpu")
    with pytest.raises(ValueError):
        para.load_state(str(tmp_path / "s"), plan, "RBC", device="cpu")
    with pytest.raises(ValueError):
        para.load_state(str(tmp_path / "s"), _fake_plan(kf=(1.0, 1.0, 1.0)), "FLUID_INCOMPRESS", device="cpu")
    with pytest.raises(ValueError):
        para.save_state(str(tmp_path / "t"), plan, "RBC", [u], 0.0)


def test_read_para_input_field_procedure(tmp_path):
    text = open(os.path.join(FFF_DIR, "in", "para.yaml")).read()
    assert para.read_para(os.path.join(FFF_DIR, "in", "para.yaml")).input_field_procedure == 5
    (tmp_path / "in").mkdir()
    (tmp_path / "in" / "para.yaml").write_text(text.replace("io:\n", "io:\n    input_field_procedure: 1\n"))
    rp = para.read_para(str(tmp_path / "in" / "para.yaml"))
    assert rp.input_field_procedure == 1
    rp.input_field_procedure = 6
    with pytest.raises(NotImplementedError):
        para.read_init_cond(str(tmp_path), None, rp)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("name", ["fff", "rbc", "rbc_przero", "rbc_prinfty"])
def test_restart_continues_bit_for_bit(cuda, tmp_path, name, precision):
    """Save after 2 steps into out/time_<t>/, restart a second run from it through
    input_field_procedure 1 (the saved folder as the new run's in/), step 2 more: the state equals
    4 unbroken steps bit for bit (under PRZERO / PRINFTY the slaved field is recomputed from
    the read one, as Init_cond_RBC_complex_field does)."""
    import shutil
    import torch
    from oracle import tarang_ref as R
    src = FFF_DIR if name == "fff" else RBC_DIR
    if name in ("rbc_przero", "rbc_prinfty"):
        pr = "PRZERO" if name == "rbc_przero" else "PRINFTY"
        os.makedirs(tmp_path / "src" / "in")
        (tmp_path / "src" / "in" / "para.yaml").write_text(
            open(os.path.join(RBC_DIR, "in", "para.yaml")).read().replace("Pr_option: PRLARGE", f"Pr_option: {pr}"))
        src = str(tmp_path / "src")
    plan, rp = para.plan_from_dir(src, precision=precision)
    if name == "fff":
        g = R.Grid(rp.N, rp.kfactor)
        V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
        fields = [torch.from_numpy(V).to(cuda).to(plan.torch_dtype())]
    else:
        u, T = plan.field(3), plan.field(1)
        plan.init_temperature_perturbation(1e-2, 4.0, 3, u[0:1] if name == "rbc_przero" else T)
        if name != "rbc":
            plan.rbc_slave(u, T)
            assert float(torch.linalg.vector_norm(u if name == "rbc_prinfty" else T)) > 0
        fields = [u, T]
    ref = [f.clone() for f in fields]
    if name in ("rbc_przero", "rbc_prinfty"):
        # the restart recomputes the slaved field from the read one, as the reference does;
        # the reality fix at the end of a step conjugates the self-conjugate modes, which
        # does not commute with the slave map, so the unbroken reference run takes the same
        # recomputation after step 2
        para.advance(plan, rp.kind, ref, 2)
        plan.rbc_slave(ref[0], ref[1])
        para.advance(plan, rp.kind, ref, 2)
    else:
        para.advance(plan, rp.kind, ref, 4)
    para.advance(plan, rp.kind, fields, 2)
    out = para.Output(plan, str(tmp_path / "run1" / "out"))
    folder = out.save(rp.kind, fields, rp.t_init + 2 * rp.dt, 2)
    assert os.path.basename(folder) == f"time_{rp.t_init + 2 * rp.dt:g}"
    # the second run: its in/ holds the para.yaml (input_field_procedure 1) and the saved fields
    run2 = tmp_path / "run2"
    shutil.copytree(folder, run2 / "in")
    text = open(os.path.join(src, "in", "para.yaml")).read()
    if "io:\n" in text:
        text = text.replace("io:\n", "io:\n    input_field_procedure: 1\n")
    else:
        text += "\nio:\n    input_field_procedure: 1\n"
    (run2 / "in" / "para.yaml").write_text(text)
    for extra in ("forcing.txt",):
        if os.path.exists(os.path.join(src, "in", extra)):
            shutil.copy(os.path.join(src, "in", extra), run2 / "in" / extra)
    plan2, rp2 = para.plan_from_dir(str(run2), precision=precision)
    assert rp2.input_field_procedure == 1
    fields2, t, step = para.read_init_cond(str(run2), plan2, rp2)
    assert step == 2 and abs(t - (rp.t_init + 2 * rp.dt)) < 1e-15
    para.advance(plan2, rp2.kind, fields2, 2)
    torch.cuda.synchronize()
    for a, b in zip(fields2, ref):
        assert torch.equal(a, b)


@pytest.mark.parametrize("pr,us", [("PRSMALL", "USMALL"), ("PRLARGE", "USMALL"), ("PRSMALL", "ULARGE"),
                                   ("PRZERO", "USMALL"), ("PRINFTY", "ULARGE")])
def test_read_para_rbc_scalings(tmp_path, pr, us):
    """Every Pr_option with Uscaling ULARGE / USMALL sets nu and kappa as Iscalar_main.cc:52-92
    (PRZERO: 1 and 0); an unknown option is refused by name, and so are the slaved scalings
    on SSF."""
    from tarang_b200.solver import rbc_diss_coefficients
    text = open(os.path.join(RBC_DIR, "in", "para.yaml")).read()
    (tmp_path / "in").mkdir()
    (tmp_path / "in" / "para.yaml").write_text(text.replace("Pr_option: PRLARGE", f"Pr_option: {pr}")
                                                .replace("Uscaling: ULARGE", f"Uscaling: {us}"))
    rp = para.read_para(str(tmp_path / "in" / "para.yaml"))
    assert (rp.pr_option, rp.uscaling) == (pr, us)
    assert (rp.nu, rp.kappa) == rbc_diss_coefficients(pr, us, rp.Ra, rp.Pr)
    if us == "USMALL":
        assert rp.nu == (rp.Pr if pr == "PRLARGE" else 1.0)
    if pr == "PRZERO":
        assert (rp.nu, rp.kappa) == (1.0, 0.0)
    (tmp_path / "in" / "para.yaml").write_text(text.replace("Pr_option: PRLARGE", "Pr_option: PRHALF"))
    with pytest.raises(NotImplementedError):
        para.read_para(str(tmp_path / "in" / "para.yaml"))
    (tmp_path / "in" / "para.yaml").write_text(text.replace("Pr_option: PRLARGE", "Pr_option: PRZERO")
                                                .replace("basis_type: SFF", "basis_type: SSF"))
    with pytest.raises(NotImplementedError):
        para.read_para(str(tmp_path / "in" / "para.yaml"))


@pytest.mark.gpu
@pytest.mark.parametrize("sign", [1, -1])
def test_glob_helicity_of_a_beltrami_mode(cuda, tmp_path, sign):
    """Known answer for the helicity columns, with a non-unit kfactor: one Beltrami mode stored
    as V = a (1, sign i, 0) at (kx, ky, kz) = (0, 0, 3), i.e. u = 2a (cos Kz z, -sign sin Kz z, 0),
    whose vorticity is sign Kz u; the reference's helicity 1/2 <u . omega> (FFF_pencil_energy.cc:
    99-139) is then H1 = sign Kz E and H2 = H1 / Kz^2 = sign E / Kz, E the Tarang energy,
    Kz = 3 kfactor_z; then an oblique mode (ky = 2, kz = 1) with |K| from both kfactors."""
    import torch
    import tarang_b200 as tb
    kf = (1.0, 2.0, 1.5)
    plan = tb.Plan((16, 16, 16), precision="f64", kfactor=kf, dealias="none")
    u = plan.field(3)
    a = 0.3
    u[0, 0, 0, 3] = a
    u[1, 0, 0, 3] = sign * 1j * a
    out = para.Output(plan, str(tmp_path))
    row = out.glob(u, 0.0, 1e-3, helicity=True)
    E = plan.energy(u)
    Kz = 3 * kf[2]
    assert abs(E - 2 * a * a) < 1e-15
    assert abs(row[1] - E) < 1e-15
    assert abs(row[3] - sign * Kz * E) < 1e-14
    assert abs(row[4] - sign * E / Kz) < 1e-14
    # a mode along y (ky = 2, kz = 1): K = (0, 2 kf_y, kf_z); a Beltrami vector e1 + sign i e2 with
    # e1, e2 unit vectors perpendicular to K and e1 x e2 = K / |K|
    u.zero_()
    K = np.array([0.0, 2 * kf[1], 1 * kf[2]])
    Km = np.linalg.norm(K)
    e1 = np.array([1.0, 0.0, 0.0])
    e2 = np.cross(K / Km, e1)
    V = a * (e1 + sign * 1j * e2)
    for i in range(3):
        u[i, 0, 2, 1] = complex(V[i])
    row = out.glob(u, 0.0, 1e-3, helicity=True)
    E = plan.energy(u)
    assert abs(row[3] - sign * Km * E) < 1e-13 * Km * E
    assert abs(row[4] - sign * E / Km) < 1e-13 * E / Km


MODES_RBC_2D = """io:
    input_field_procedure: 4
    init_cond_modes:
            - coord: [1,0,1]
              mode: [ (0.01,0), (0,0), (0,0) ]
            - coord: [2,0,0]
              mode: [ (0,0), (0,0), (-0.16,0) ]
            - coord: [3,0,40]
              mode: [ (1,0), (0,0), (1,0) ]
"""


def _modes_para(tmp_path, src_dir, modes_text, edit=None):
    text = open(os.path.join(src_dir, "in", "para.yaml")).read()
    text = "\n".join(line for line in text.split("\n") if not line.startswith("io:")) + "\n" + modes_text
    if edit:
        text = edit(text)
    (tmp_path / "in").mkdir(exist_ok=True)
    (tmp_path / "in" / "para.yaml").write_text(text)
    return para.read_para(str(tmp_path / "in" / "para.yaml"))


def test_init_cond_modes_rbc_two_dimensional(tmp_path):
    """io.input_field_procedure 4 on the reference's RBC/2d layout (SFF, 32 x 1 x 32): the
    "(re,im)" values parse, Vz follows from incompressibility (SFF: d_x of the sine series
    Vx is +Kx Vx), the scalar takes its value, a mode outside the array (kz = 40) is
    skipped, and nothing else is set."""
    rp = _modes_para(tmp_path, KIND_DIRS["rbc_2d"], MODES_RBC_2D)
    assert rp.input_field_procedure == 4 and len(rp.init_cond_modes) == 3
    assert rp.init_cond_modes[0] == ((1, 0, 1), [0.01 + 0j, 0j, 0j])
    U, T = para.init_cond_modes(rp)
    Kx, Kz = 1 * rp.kfactor[0], 1 * rp.kfactor[2]
    want_U = np.zeros_like(U)
    want_U[0, 1, 0, 1] = 0.01
    want_U[2, 1, 0, 1] = Kx * 0.01 / (-1j * Kz)
    want_T = np.zeros_like(T)
    want_T[0, 2, 0, 0] = -0.16
    assert np.array_equal(U, want_U) and np.array_equal(T, want_T)
    # divergence of the set mode: Kx Vx + i Kz Vz = 0
    assert abs(Kx * U[0, 1, 0, 1] + 1j * Kz * U[2, 1, 0, 1]) < 1e-18


def test_init_cond_modes_fff_fluid_conjugates_and_divergence(tmp_path):
    """FFF fluid modes: Vz from incompressibility off the kz = 0 plane; on it the pair read
    is (Vx, Vz) with Vy computed (ky != 0), or (Vy, Vz) with Vx = 0 (ky = 0); the mirror
    (-kx, -ky, 0) holds the conjugate; every set mode is solenoidal."""
    modes = """io:
    input_field_procedure: 4
    init_cond_modes:
            - coord: [1,2,3]
              mode: [ (0.1,0.2), (0.3,-0.1) ]
            - coord: [2,-1,0]
              mode: [ (0.5,0.1), (0.2,0.0) ]
            - coord: [3,0,0]
              mode: [ (0.4,0.0), (0.0,0.7) ]
"""
    rp = _modes_para(tmp_path, FFF_DIR, modes)
    (U,) = para.init_cond_modes(rp)
    Nx, Ny, Nz = rp.N
    kf = rp.kfactor
    set_modes = np.argwhere(np.abs(U).sum(axis=0) > 0)
    for lx, ly, lz in set_modes:
        kx = lx if lx <= Nx // 2 else lx - Nx
        ky = ly if ly <= Ny // 2 else ly - Ny
        div = 1j * (kx * kf[0] * U[0, lx, ly, lz] + ky * kf[1] * U[1, lx, ly, lz] + lz * kf[2] * U[2, lx, ly, lz])
        assert abs(div) < 1e-15
    assert np.allclose(U[:, 1, 2, 3], [0.1 + 0.2j, 0.3 - 0.1j, U[2, 1, 2, 3]])
    # kz = 0, ky != 0: the pair is (Vx, Vz), the mirror is the conjugate
    assert U[0, 2, Ny - 1, 0] == 0.5 + 0.1j and U[2, 2, Ny - 1, 0] == 0.2
    assert np.array_equal(U[:, Nx - 2, 1, 0], np.conj(U[:, 2, Ny - 1, 0]))
    # kz = 0, ky = 0: the pair is (Vy, Vz) and Vx = 0
    assert U[0, 3, 0, 0] == 0 and U[1, 3, 0, 0] == 0.4 and U[2, 3, 0, 0] == 0.7j
    assert np.array_equal(U[:, Nx - 3, 0, 0], np.conj(U[:, 3, 0, 0]))


def test_init_cond_modes_refused_off_fff_sff(tmp_path):
    rp = _modes_para(tmp_path, KIND_DIRS["sss"], "io:\n    input_field_procedure: 4\n    init_cond_modes:\n"
                     "            - coord: [1,0,1]\n              mode: [ 1, 0 ]\n")
    with pytest.raises(NotImplementedError):
        para.init_cond_modes(rp)
    rp = _modes_para(tmp_path, KIND_DIRS["mhd"], MODES_RBC_2D)
    with pytest.raises(NotImplementedError):
        para.init_cond_modes(rp)


@pytest.mark.gpu
@pytest.mark.parametrize("pr", ["PRLARGE", "PRZERO"])
def test_init_cond_modes_rbc_steps_like_the_oracle(cuda, tmp_path, pr):
    """A two-dimensional RBC run started from io.input_field_procedure 4 (the reference's
    RBC/2d modes; PRZERO also slaves T = U1 / K^2 on the device) steps like the oracle
    from the same modes: FP64 relative L2 <= 1e-12 after 3 steps."""
    from oracle import tarang_ref as R
    rp = _modes_para(tmp_path, KIND_DIRS["rbc_2d"], MODES_RBC_2D,
                     edit=lambda t: t.replace("Pr_option: PRLARGE", f"Pr_option: {pr}"))
    plan, rp2 = para.plan_from_dir(str(tmp_path), precision="f64")
    fields, t, step = para.read_init_cond(str(tmp_path), plan, rp2)
    U0, T0 = para.init_cond_modes(rp2)
    g = R.Grid(rp2.N, rp2.kfactor, "SFF")
    cfg = R.RBCConfig(g, Ra=rp2.Ra, Pr=rp2.Pr, dt=rp2.dt, dealias_mode=1, reality_fix=rp2.reality_fix,
                      pr_option=pr, uscaling=rp2.uscaling)
    if pr == "PRZERO":
        T0 = R.rbc_slave_temperature(g, U0)[None]
    assert np.abs(fields[1][0].cpu().numpy() - T0[0]).max() <= 1e-15 * max(1.0, np.abs(T0).max())
    Uo, To = U0, T0[0]
    for _ in range(3):
        Uo, To = R.rbc_rk4_step(cfg, Uo, To)
    para.advance(plan, rp2.kind, fields, 3)
    u, T = fields
    assert np.linalg.norm(u.cpu().numpy() - Uo) <= 1e-12 * np.linalg.norm(Uo)
    assert np.linalg.norm(T[0].cpu().numpy() - To) <= 1e-12 * max(np.linalg.norm(To), 1e-300)
    plan.close()


def _write_initial(tmp_path, E, H=None):
    def arr(a):
        return f"({0},{len(a) - 1})\n[ " + " ".join(f"{x:.17g}" for x in a) + " ]\n"
    (tmp_path / "in").mkdir(exist_ok=True)
    (tmp_path / "in" / "initial.txt").write_text(arr(E) + arr(np.zeros(len(E)) if H is None else H))


def test_init_cond_energy_spectrum_refusals(tmp_path):
    """io.input_field_procedure 5 is taken for the FFF fluid with a zero helicity spectrum;
    other kinds and a helical spectrum are refused by name."""
    rp = _modes_para(tmp_path, KIND_DIRS["rbc_2d"], "io:\n    input_field_procedure: 5\n")
    assert rp.input_field_procedure == 5
    with pytest.raises(NotImplementedError):
        para.read_init_cond(str(tmp_path), None, rp)
    rp = _modes_para(tmp_path, FFF_DIR, "io:\n    input_field_procedure: 5\n")
    _write_initial(tmp_path, np.linspace(0, 1, 8), np.full(8, 0.1))
    with pytest.raises(NotImplementedError):
        para.read_init_cond(str(tmp_path), None, rp)


@pytest.mark.gpu
def test_init_cond_energy_spectrum_matches_oracle(cuda, tmp_path):
    """io.input_field_procedure 5 on an FFF fluid run: E(k) from in/initial.txt, the
    random-phase construction of init_cond_energy.cc:67-120 with the splitmix64 phases of
    seed 0, no rescaling: the oracle's field to 1e-13, and the run steps."""
    from oracle import tarang_ref as R
    rp = _modes_para(tmp_path, FFF_DIR, "io:\n    input_field_procedure: 5\n")
    g = R.Grid(rp.N, rp.kfactor)
    E = R.spectrum_k4_gauss(g.n_shells(), 3.0) * 0.7
    _write_initial(tmp_path, E)
    (tmp_path / "in" / "forcing.txt").write_text(open(os.path.join(FFF_DIR, "in", "forcing.txt")).read())
    plan, rp2 = para.plan_from_dir(str(tmp_path), precision="f64")
    fields, t, step = para.read_init_cond(str(tmp_path), plan, rp2)
    want = R.init_energy_spectrum(g, E, 0, None)
    u = fields[0].cpu().numpy()
    assert np.abs(u - want).max() <= 1e-13 * np.abs(want).max()
    para.advance(plan, rp2.kind, fields, 2)
    assert np.isfinite(fields[0].cpu().numpy()).all()
    plan.close()
