"""The C++ host mirror (include/tarang_b200.hpp) compiles against the C ABI (CPU) and, on a GPU,
gives the same numbers as the Python binding of the same library."""
import json
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
    r = subprocess.run([str(exe), "32", "5"], capture_output=True, text=True, timeout=300)
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
