"""The allocation-free shell spectrum, through the C ABI.

ts_shell_spectrum_noalloc serves callers that cannot allocate device memory
when they need E(k): a stepping loop that has reserved nearly all of the GPU's
memory for its fields, or one that must not let cudaMalloc / cudaFree
synchronize the device.  Its accumulators are a file-scope __device__ array
that every call shares, so this test makes two calls in a row (the second one
must not see the first one's sums) and compares both with the planned entry
point ts_shell_spectrum.  It lives in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, basis, prec, N, kf, a, ncomp, out, stream):
    Na = (ctypes.c_int * 3)(*N)
    Ka = (ctypes.c_double * 3)(*kf)
    return lib.ts_shell_spectrum_noalloc(basis, prec, Na, Ka, ctypes.c_void_p(a.data_ptr()), ncomp,
                                         ctypes.c_void_p(out.data_ptr()), out.numel(), ctypes.c_void_p(stream))


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_noalloc_shell_spectrum_matches_planned(cuda, precision):
    import torch
    import tarang_b200 as tb
    from tarang_b200 import _lib as L

    lib = L.load()
    N = (32, 32, 32)
    plan = tb.Plan(N, precision=precision)
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    v = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 8.0), 1, 2.0, v)
    stream = torch.cuda.current_stream().cuda_stream
    prec = L.TS_F64 if precision == "f64" else L.TS_F32
    tol = 1e-12 if precision == "f64" else 1e-6
    for field in (u, v):  # two calls in a row on different fields
        ref = plan.shell_spectrum(field)
        out = torch.full((plan.n_shells,), float("nan"), dtype=torch.float64, device=cuda)
        rc = _noalloc(lib, L.TS_BASIS_FFF, prec, N, (1.0, 1.0, 1.0), field, 3, out, stream)
        assert rc == L.TS_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    plan.close()


def test_noalloc_rejects_too_many_shells(cuda):
    import torch
    from tarang_b200 import _lib as L

    lib = L.load()
    # a correctly sized 16^3 field whose kfactor 600 gives ceil(sqrt(3)*8*600)+1 = 8315 shells (> 4096):
    # the call must refuse before launching anything
    a = torch.zeros((1, 16, 16, 9), dtype=torch.complex128, device=cuda)
    out = torch.zeros(8, dtype=torch.float64, device=cuda)
    rc = _noalloc(lib, L.TS_BASIS_FFF, L.TS_F64, (16, 16, 16), (600.0, 600.0, 600.0), a, 1, out, 0)
    assert rc == L.TS_ERR_ARG
    assert torch.all(out == 0)
