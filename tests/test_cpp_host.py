"""The C++ host mirror (include/tarang_b200.hpp) compiles against the C ABI (CPU) and, on a GPU,
gives the same numbers as the Python binding of the same library."""
import json
import math
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def build_driver(tmp_path):
    lib = ROOT / "tarang_b200" / "libtarang_b200.so"
    if not lib.exists():
        pytest.skip("library not built")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = tmp_path / "host_mirror"
    cmd = [gxx, "-std=c++17", "-O2", str(ROOT / "tests" / "cpp" / "host_mirror_main.cpp"), "-I", str(ROOT / "include"),
           "-I", str(CUDA / "include"), str(lib), f"-Wl,-rpath,{lib.parent}", "-L", str(CUDA / "lib64"), "-lcudart",
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_host_mirror_compiles_and_links(tmp_path):
    build_driver(tmp_path)


@pytest.mark.gpu
def test_host_mirror_matches_python_binding(cuda, tmp_path):
    import torch
    import tarang_b200 as tb
    exe = build_driver(tmp_path)
    r = subprocess.run([str(exe), "fff", "32", "5"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    plan = tb.Plan(32, nu=0.01, dt=1e-3)
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    e0 = plan.energy(u)
    plan.rk4_step(u, 5)
    torch.cuda.synchronize()
    assert abs(out["e0"] - e0) < 1e-14
    assert abs(out["e1"] - plan.energy(u)) < 1e-14
    assert np.max(np.abs(np.array(out["Ek"]) - plan.shell_spectrum(u))) < 1e-13
    assert out["div"] < 1e-12
    assert np.max(np.abs(np.array(out["Pi"]) - plan.flux(u, [2.0, 4.0, 8.0]))) < 1e-14


@pytest.mark.gpu
def test_host_mirror_mhd_matches_python_binding(cuda, tmp_path):
    import tarang_b200 as tb
    out = run_driver(build_driver(tmp_path), "mhd", 32, 4)
    plan = tb.Plan(32, nu=0.01, kappa=0.02, dt=1e-3, dealias="two_thirds")
    u, b = plan.field(3), plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 3.0), 1, 0.3, b)
    plan.rk4_step_mhd(u, b, 4)
    # the drivers build the initial spectra with different pow/exp (last-bit differences)
    assert abs(out["eu"] - plan.energy(u)) < 1e-13 * out["eu"]
    assert abs(out["eb"] - plan.energy(b)) < 1e-13 * out["eb"]
    assert out["divb"] < 1e-12


@pytest.mark.gpu
def test_host_mirror_autotuned_matches_rule(cuda, tmp_path):
    exe = build_driver(tmp_path)
    a = run_driver(exe, "fff", 64, 3)
    b = run_driver(exe, "fff_tuned", 64, 3)
    assert abs(a["e1"] - b["e1"]) < 1e-13 * a["e1"]  # FP64: candidates differ in rounding only
    assert np.max(np.abs(np.array(a["Ek"]) - np.array(b["Ek"]))) < 1e-13 * a["e1"]


def run_driver(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


@pytest.mark.gpu
def test_host_mirror_rbc_matches_python_binding(cuda, tmp_path):
    import torch
    import tarang_b200 as tb
    out = run_driver(build_driver(tmp_path), "rbc", 32, 5)
    Ra, Pr = 1e5, 1.0
    plan = tb.Plan(32, basis="SFF", precision="f32", kfactor=(math.pi, 2 * math.pi, 2 * math.pi),
                   nu=math.sqrt(Pr / Ra), kappa=1 / math.sqrt(Pr * Ra), dt=1e-3, Ra=Ra, Pr=Pr)
    u, T = plan.field(3), plan.field(1)
    plan.init_temperature_perturbation(0.01, 4.0, 3, T)
    plan.rk4_step_rbc(u, T, 5)
    torch.cuda.synchronize()
    # same library, same launches: bitwise equal
    assert out["eu"] == plan.energy(u)
    assert out["eT"] == plan.energy(T)
    assert out["Nu"] == plan.nusselt(u, T)
    assert out["eu"] > 0 and out["Nu"] != 1.0


@pytest.mark.gpu
def test_host_mirror_rbc_sss_matches_python_binding(cuda, tmp_path):
    """RBC on SSS through SSS_PENCIL, FluidVF, FluidSF and Time_advance_incompress::RK4(U, T)
    gives the Python binding's energies and Nusselt number bit for bit."""
    import torch
    import tarang_b200 as tb
    N, steps = 32, 4
    out = run_driver(build_driver(tmp_path), "rbc_sss", N, steps)
    Ra, Pr = 1e5, 1.0
    kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    plan = tb.Plan(N, basis="SSS", precision="f64", kfactor=kf, nu=math.sqrt(Pr / Ra), kappa=1 / math.sqrt(Pr * Ra),
                   dt=1e-3, Ra=Ra, Pr=Pr)
    u = np.zeros((3, N, N, N + 2))
    t = np.zeros((1, N, N, N + 2))
    u[0, 1, 1, 1] = 0.1
    u[1, 1, 1, 1] = -0.1 * kf[0] / kf[1]
    t[0, 1, 1, 1] = 0.05
    t[0, 2, 1, 0] = 0.02
    ud = torch.from_numpy(u.view(np.complex128)).to(cuda)
    td = torch.from_numpy(t.view(np.complex128)).to(cuda)
    plan.rk4_step_rbc(ud, td, steps)
    torch.cuda.synchronize()
    assert out["eu"] == plan.energy(ud) and out["eT"] == plan.energy(td)
    assert out["Nu"] == plan.nusselt(ud, td)
    assert out["eu"] > 0 and out["Nu"] != 1.0


@pytest.mark.gpu
def test_host_mirror_ensemble_matches_python_binding(cuda, tmp_path):
    import tarang_b200 as tb
    out = run_driver(build_driver(tmp_path), "ensemble", 32, 4)
    ens = tb.Ensemble([(32, 1e5, 1.0), (48, 1e6, 1.0)], dt=1e-4, precision="f32")
    ens.init_temperature(0.01, 4.0, 7)
    ens.run(4)
    assert out["Nu"] == list(ens.nusselt())


@pytest.mark.gpu
def test_host_mirror_adjoint_matches_python_binding(cuda, tmp_path):
    import torch
    import tarang_b200 as tb
    out = run_driver(build_driver(tmp_path), "adjoint", 32, 3)
    plan = tb.Plan(32, nlin_form="rotational", dealias="two_thirds", nu=0.01, dt=1e-3)
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    lam = u.clone()
    work = torch.empty(plan.adjoint_work_bytes(3), dtype=torch.uint8, device=cuda)
    plan.adjoint_window(u, 3, lam, work)
    plan.status()
    # the two drivers build the initial spectrum with different pow/exp (last-bit differences)
    assert abs(out["elam"] - plan.energy(lam)) < 1e-13 * out["elam"]
    assert np.max(np.abs(np.array(out["Ek"]) - plan.shell_spectrum(lam))) < 1e-13 * out["elam"]
    assert out["elam"] > 0
