"""The C ABI library loads and exports every function include/tarang_b200.h declares (CPU only:
no compute call is made without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "tarang_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s+(ts_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = header_functions()
    for n in ["ts_plan_create", "ts_rk4_step", "ts_nlin", "ts_fft_forward", "ts_fft_inverse", "ts_shell_spectrum",
              "ts_flux", "ts_energy", "ts_max_div", "ts_rk4_step_rbc", "ts_nusselt", "ts_shell_spectrum_noalloc"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from tarang_b200 import _lib as L
    lib = L.load()
    for n in header_functions():
        assert hasattr(lib, n), n
        assert n in L.SIGNATURES, f"{n} has no ctypes signature"


def test_config_default_without_gpu():
    from tarang_b200 import _lib as L
    lib = L.load()
    c = L.TsConfig()
    lib.ts_config_default(ctypes.byref(c))
    assert c.basis == L.TS_BASIS_FFF and tuple(c.N) == (64, 64, 64)
    assert c.dealias_mode == L.TS_DEALIAS_REFERENCE_CORNER and c.reality_fix == 1
    assert abs(c.nu - 0.01) < 1e-15 and abs(c.dt - 1e-3) < 1e-15


def test_invalid_config_is_rejected_without_touching_the_gpu():
    from tarang_b200 import _lib as L
    lib = L.load()
    c = L.TsConfig()
    lib.ts_config_default(ctypes.byref(c))
    c.N[0] = 100  # not a supported power of two: rejected before any CUDA call
    h = ctypes.c_void_p()
    assert lib.ts_plan_create(ctypes.byref(c), ctypes.byref(h)) == L.TS_ERR_ARG
    assert not h.value


def test_struct_layout_matches_header_field_order():
    from tarang_b200 import _lib as L
    text = (ROOT / "include" / "tarang_b200.h").read_text()
    body = text[text.index("typedef struct {"):text.index("} ts_config;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        for part in decl.replace("typedef struct {", "").split(","):
            m = re.findall(r"\**\s*([A-Za-z_][A-Za-z_0-9]*)\s*(?:\[\d+\])?\s*$", part.strip())
            if m:
                fields.append(m[-1])
    assert fields == [f for f, _ in L.TsConfig._fields_]
