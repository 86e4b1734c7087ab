"""Host-side API over the C ABI, with the reference's names.

``Plan`` owns a ``ts_plan`` (the basis object + FFTK plan + RK work arrays of
the reference).  Fields are torch tensors on the GPU (complex64 / complex128,
shape (ncomp, Nx, Ny, Nz//2+1), the reference's spectral layout) or numpy
arrays on the host; host arrays are staged by the library inside the call.

Reference-named wrappers (paths inside anandogc/tarang ``trunk/lib``):
  FluidVF                     fluid/fluid_base/FluidVF.h:73-180
  Nlin_incompress.Compute_nlin fluid/incompressible/nlin/compute_nlin.cc:58-109
  Time_advance_incompress.RK4  fluid/incompressible/time_advance/RK.cc:91-170
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from dataclasses import dataclass

import numpy as np

from . import _lib as L

_DEALIAS = {"none": L.TS_DEALIAS_NONE, "reference": L.TS_DEALIAS_REFERENCE_CORNER,
            "two_thirds": L.TS_DEALIAS_TWO_THIRDS}
_FORM = {"conservative": L.TS_NLIN_CONSERVATIVE, "rotational": L.TS_NLIN_ROTATIONAL}


@dataclass
class Forcing:
    """Carati constant energy supply, non-global alpha/beta (force.field_procedure 1)."""
    inner_radius: float
    outer_radius: float
    energy_supply: np.ndarray
    helicity_supply: np.ndarray | None = None


def _tuning_struct(tuning: dict) -> L.TsTuning:
    t = L.TsTuning()
    for i in range(5):
        t.variant[i] = int(tuning["variant"][i])
        t.blocks_per_sm[i] = int(tuning["blocks_per_sm"][i])
    return t


def _cache_put(path: str, key: str, tuning: dict):
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[key] = tuning
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _ptr(a) -> int:
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("field must be contiguous")
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("field must be C contiguous")
        return a.ctypes.data
    raise TypeError(type(a))


# PHYSICS.Pr_option / PHYSICS.Uscaling of an RBC run
_PR_OPTION = {"PRLARGE": 0, "PRSMALL": 1, "PRZERO": 2, "PRINFTY": 3}
_USCALING = {"ULARGE": 0, "USMALL": 1}


def rbc_diss_coefficients(pr_option: str, uscaling: str, Ra: float, Pr: float) -> tuple:
    """(nu, kappa) of an RBC run (Iscalar_main.cc:52-92)."""
    small = uscaling == "USMALL"
    if pr_option == "PRLARGE":
        return (Pr, 1.0) if small else (math.sqrt(Pr / Ra), 1.0 / math.sqrt(Pr * Ra))
    if pr_option == "PRSMALL":
        return (1.0, 1.0 / Pr) if small else (math.sqrt(Pr / Ra), 1.0 / math.sqrt(Pr * Ra))
    if pr_option == "PRZERO":
        return (1.0, 0.0)
    if pr_option == "PRINFTY":
        return (Pr, 1.0) if small else (1.0 / math.sqrt(Ra), 1.0 / math.sqrt(Ra))
    raise ValueError(f"Pr_option {pr_option}")


class Plan:
    def __init__(self, N, basis: str = "FFF", precision: str = "f64", nlin_form: str = "conservative",
                 dealias: str = "reference", nu: float = 0.01, dt: float = 1e-3, kfactor=(1.0, 1.0, 1.0),
                 reality_fix: bool = True, forcing: Forcing | None = None, kappa: float = 0.01,
                 Ra: float = 1e5, Pr: float = 1.0, Pr_option: str = "PRLARGE", Uscaling: str = "ULARGE"):
        self.lib = L.load()
        if isinstance(N, int):
            N = (N, N, N)
        self.N = tuple(int(n) for n in N)
        c = L.TsConfig()
        self.lib.ts_config_default(ctypes.byref(c))
        c.basis = {"FFF": L.TS_BASIS_FFF, "SFF": L.TS_BASIS_SFF, "SSF": L.TS_BASIS_SSF, "SSS": L.TS_BASIS_SSS}[basis]
        for i in range(3):
            c.N[i] = self.N[i]
            c.kfactor[i] = float(kfactor[i])
        c.precision = L.TS_F64 if precision == "f64" else L.TS_F32
        c.nlin_form = _FORM[nlin_form]
        c.dealias_mode = _DEALIAS[dealias]
        c.reality_fix = int(bool(reality_fix))
        c.nu, c.kappa, c.dt, c.Ra, c.Pr = nu, kappa, dt, Ra, Pr
        c.Pr_option = _PR_OPTION[Pr_option]
        c.Uscaling = _USCALING[Uscaling]
        self._keep = []
        if forcing is not None:
            es = np.ascontiguousarray(forcing.energy_supply, dtype=np.float64)
            self._keep.append(es)
            c.force_type = L.TS_FORCE_CARATI_ENERGY_SUPPLY
            c.force_inner_radius = forcing.inner_radius
            c.force_outer_radius = forcing.outer_radius
            c.energy_supply = es.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            c.n_supply = len(es)
            if forcing.helicity_supply is not None:
                hs = np.ascontiguousarray(forcing.helicity_supply, dtype=np.float64)
                self._keep.append(hs)
                c.helicity_supply = hs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self.cfg = c
        self.basis = basis
        self.precision = precision
        h = ctypes.c_void_p()
        L.check(self.lib.ts_plan_create(ctypes.byref(c), ctypes.byref(h)), "ts_plan_create")
        self.h = h
        n = ctypes.c_int()
        L.check(self.lib.ts_plan_num_shells(self.h, ctypes.byref(n)), "ts_plan_num_shells")
        self.n_shells = n.value

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.ts_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def spec_shape(self):
        Nx, Ny, Nz = self.N
        return (Nx, Ny, Nz // 2 + 1)

    def torch_dtype(self):
        import torch
        return torch.complex64 if self.precision == "f32" else torch.complex128

    def numpy_dtype(self):
        return np.complex64 if self.precision == "f32" else np.complex128

    def field(self, ncomp: int = 3, device: str = "cuda"):
        import torch
        return torch.zeros((ncomp,) + self.spec_shape, dtype=self.torch_dtype(), device=device)

    def set_stream(self, stream=None):
        """Use a torch.cuda.Stream (default: torch's current stream) for every later call."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        L.check(self.lib.ts_plan_set_stream(self.h, ctypes.c_void_p(s.cuda_stream)), "ts_plan_set_stream")

    def status(self):
        """Synchronise the plan's stream; raise TsError (status TS_ERR_TIMEOUT or TS_ERR_NAN) if a
        bounded device wait gave up or a step wrote a NaN / Inf into the state earlier."""
        L.check(self.lib.ts_plan_status(self.h), "ts_plan_status")

    def status_code(self) -> int:
        """ts_plan_status without raising: TS_OK, TS_ERR_TIMEOUT or TS_ERR_NAN."""
        return int(self.lib.ts_plan_status(self.h))

    def clear_status(self):
        L.check(self.lib.ts_plan_clear_status(self.h), "ts_plan_clear_status")

    # ------------------------------------------------------------------
    # launch tuning (candidate kernels per pass class; see ts_plan_autotune)
    def tuning(self) -> dict:
        t = L.TsTuning()
        L.check(self.lib.ts_plan_get_tuning(self.h, ctypes.byref(t)), "ts_plan_get_tuning")
        return {"variant": list(t.variant), "blocks_per_sm": list(t.blocks_per_sm)}

    def set_tuning(self, tuning: dict):
        L.check(self.lib.ts_plan_set_tuning(self.h, ctypes.byref(_tuning_struct(tuning))), "ts_plan_set_tuning")

    def tuning_candidates(self) -> dict:
        """{class: {"variants": [candidate indices], "blocks": takes a blocks-per-SM count}}"""
        out = {}
        for c, name in enumerate(L.TUNE_CLASSES):
            m, b = ctypes.c_int(), ctypes.c_int()
            L.check(self.lib.ts_tuning_candidates(self.h, c, ctypes.byref(m), ctypes.byref(b)), "ts_tuning_candidates")
            out[name] = {"variants": [v for v in range(8) if m.value >> v & 1], "blocks": bool(b.value)}
        return out

    def tuning_key(self) -> str:
        import torch
        dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
        c = self.cfg
        return (f"{dev}|{self.basis}|{'x'.join(map(str, self.N))}|{self.precision}|form{c.nlin_form}"
                f"|dealias{c.dealias_mode}|force{c.force_type}")

    def autotune(self, reps: int = 3, cache: str | None = None) -> dict:
        """Pick the fastest kernel candidate of every pass class on this GPU (ts_plan_autotune) and
        return the timing report.  cache: a JSON file of earlier results keyed by device and plan
        configuration; a hit applies the stored tuning without timing anything."""
        key = self.tuning_key()
        if cache and os.path.exists(cache):
            with open(cache) as f:
                hit = json.load(f).get(key)
            if hit is not None:
                self.set_tuning(hit)
                return {"cached": True, "tuning": hit}
        buf = ctypes.create_string_buffer(1 << 16)
        L.check(self.lib.ts_plan_autotune(self.h, reps, buf, len(buf)), "ts_plan_autotune")
        report = json.loads(buf.value.decode())
        report["tuning"] = self.tuning()
        if cache:
            _cache_put(cache, key, report["tuning"])
        return report

    # ------------------------------------------------------------------
    def rk4_step(self, u, nsteps: int = 1):
        L.check(self.lib.ts_rk4_step(self.h, _ptr(u), nsteps), "ts_rk4_step")

    def rk4_step_keep(self, u, u_next, stages):
        """One step u -> u_next (may be u) keeping the stage fields U1, U2, U3 in stages (9 components)."""
        L.check(self.lib.ts_rk4_step_keep(self.h, _ptr(u), _ptr(u_next), _ptr(stages)), "ts_rk4_step_keep")

    def adjoint_step(self, u, stages, lam):
        """lam <- (d step / d u)^T lam for the step from u whose stage fields are `stages`."""
        L.check(self.lib.ts_adjoint_step(self.h, _ptr(u), _ptr(stages), _ptr(lam)), "ts_adjoint_step")
        return lam

    def adjoint_work_bytes(self, nsteps: int) -> int:
        b = ctypes.c_size_t()
        L.check(self.lib.ts_adjoint_work_bytes(self.h, nsteps, ctypes.byref(b)), "ts_adjoint_work_bytes")
        return b.value

    def adjoint_window(self, u_start, nsteps: int, lam, work):
        """Recompute nsteps steps from u_start (states and stages kept in `work`), then map lam, the
        cotangent of the state after nsteps, to the cotangent of u_start (in place)."""
        nbytes = work.numel() * work.element_size()
        L.check(self.lib.ts_adjoint_window(self.h, _ptr(u_start), nsteps, _ptr(lam), _ptr(work), nbytes),
                "ts_adjoint_window")
        return lam

    def rk4_step_rbc(self, u, T, nsteps: int = 1):
        L.check(self.lib.ts_rk4_step_rbc(self.h, _ptr(u), _ptr(T), nsteps), "ts_rk4_step_rbc")

    def rk4_step_mhd(self, u, b, nsteps: int = 1):
        """RK4(U, W, P, F) for incompressible MHD (FFF, unforced): u with nu, b with eta = the plan's kappa."""
        L.check(self.lib.ts_rk4_step_mhd(self.h, _ptr(u), _ptr(b), nsteps), "ts_rk4_step_mhd")

    def rk4_step_scalar(self, u, T, nsteps: int = 1):
        """RK4(U,T,P,F) with a passive scalar T (FFF, conservative form, unforced; kappa of the plan)."""
        L.check(self.lib.ts_rk4_step_scalar(self.h, _ptr(u), _ptr(T), nsteps), "ts_rk4_step_scalar")

    def nlin(self, u, out):
        L.check(self.lib.ts_nlin(self.h, _ptr(u), _ptr(out)), "ts_nlin")
        return out

    def energy(self, a, ncomp: int | None = None) -> float:
        n = a.shape[0] if ncomp is None else ncomp
        e = ctypes.c_double()
        L.check(self.lib.ts_energy(self.h, _ptr(a), n, ctypes.byref(e)), "ts_energy")
        return e.value

    def max_div(self, u) -> float:
        e = ctypes.c_double()
        L.check(self.lib.ts_max_div(self.h, _ptr(u), ctypes.byref(e)), "ts_max_div")
        return e.value

    def shell_spectrum(self, a, ncomp: int | None = None) -> np.ndarray:
        n = a.shape[0] if ncomp is None else ncomp
        out = np.zeros(self.n_shells)
        L.check(self.lib.ts_shell_spectrum(self.h, _ptr(a), n, out.ctypes.data_as(L._D), self.n_shells),
                "ts_shell_spectrum")
        return out

    def shell_sums(self, a, b=None, ncomp: int | None = None):
        """Raw shell sums (sum mult K^2 Re(a . conj(b)), or |a|^2) and counts (sum 2 mult) per shell."""
        n = a.shape[0] if ncomp is None else ncomp
        sums, counts = np.zeros(self.n_shells), np.zeros(self.n_shells)
        L.check(self.lib.ts_shell_sums(self.h, _ptr(a), _ptr(b) if b is not None else None, n,
                                       sums.ctypes.data_as(L._D), counts.ctypes.data_as(L._D), self.n_shells),
                "ts_shell_sums")
        return sums, counts

    def force_field(self, u, out):
        """The Carati force of state u as a full spectral field (zero outside the band)."""
        L.check(self.lib.ts_force_field(self.h, _ptr(u), _ptr(out)), "ts_force_field")
        return out

    def dealias(self, a, ncomp: int | None = None):
        """Universal::Dealias in place (the plan's dealias mode)."""
        n = a.shape[0] if ncomp is None else ncomp
        L.check(self.lib.ts_dealias_field(self.h, _ptr(a), n), "ts_dealias_field")
        return a

    def flux(self, u, radii) -> np.ndarray:
        r = np.ascontiguousarray(radii, dtype=np.float64)
        out = np.zeros(len(r))
        L.check(self.lib.ts_flux(self.h, _ptr(u), r.ctypes.data_as(L._D), len(r), out.ctypes.data_as(L._D)),
                "ts_flux")
        return out

    def init_temperature_perturbation(self, amp: float, kmax: float, seed: int, out):
        L.check(self.lib.ts_init_temperature_perturbation(self.h, amp, kmax, seed, _ptr(out)),
                "ts_init_temperature_perturbation")
        return out

    def nusselt(self, u, T) -> float:
        e = ctypes.c_double()
        L.check(self.lib.ts_nusselt(self.h, _ptr(u), _ptr(T), ctypes.byref(e)), "ts_nusselt")
        return e.value

    def rbc_slave(self, u, T):
        """PRZERO: T = U.V1 / K^2; PRINFTY: u = vs P(T x) / K^2 (in place; SFF plans)."""
        L.check(self.lib.ts_rbc_slave(self.h, _ptr(u), _ptr(T)), "ts_rbc_slave")
        return u, T

    def init_energy_spectrum(self, E_ic, seed: int, target_energy: float, out):
        e = np.ascontiguousarray(E_ic, dtype=np.float64)
        L.check(self.lib.ts_init_energy_spectrum(self.h, e.ctypes.data_as(L._D), len(e), seed, target_energy,
                                                 _ptr(out)), "ts_init_energy_spectrum")
        return out

    def forward(self, real, spec, parity: str = "FFF", ncomp: int | None = None):
        n = real.shape[0] if ncomp is None else ncomp
        L.check(self.lib.ts_fft_forward(self.h, parity.encode(), _ptr(real), _ptr(spec), n), "ts_fft_forward")
        return spec

    def inverse(self, spec, real, parity: str = "FFF", ncomp: int | None = None):
        n = spec.shape[0] if ncomp is None else ncomp
        L.check(self.lib.ts_fft_inverse(self.h, parity.encode(), _ptr(spec), _ptr(real), n), "ts_fft_inverse")
        return real


def kernel_launch_count() -> int:
    return int(L.load().ts_kernel_launch_count())


def spectrum_k4_gauss(nsh: int, k0: float) -> np.ndarray:
    """E_IC(s) = s^4 exp(-2 (s/k0)^2) for shell s >= 1 (the benchmark initial spectrum)."""
    s = np.arange(nsh, dtype=np.float64)
    E = s ** 4 * np.exp(-2.0 * (s / k0) ** 2)
    E[0] = 0
    return E


# ---------------------------------------------------------------------------
# reference-named wrappers
# ---------------------------------------------------------------------------
class FluidVF:
    """Velocity field container: ``cvf`` (3 spectral components) and ``nlin``."""

    def __init__(self, plan: Plan, device: str = "cuda"):
        self.plan = plan
        self.cvf = plan.field(3, device)
        self.nlin = plan.field(3, device)

    def Compute_total_energy(self) -> float:
        return self.plan.energy(self.cvf)

    def Compute_divergence_field(self) -> float:
        return self.plan.max_div(self.cvf)


class Nlin_incompress:
    @staticmethod
    def Compute_nlin(U: FluidVF):
        """Dealias U.cvf in place, then U.nlin = F[(u.grad)u] (compute_nlin.cc:58-109)."""
        U.plan.nlin(U.cvf, U.nlin)


class Time_advance_incompress:
    @staticmethod
    def RK4(U: FluidVF, nsteps: int = 1):
        """IF-RK4 step(s) + strong reality condition (RK.cc:91-170, Time_advance.cc:59-60)."""
        U.plan.rk4_step(U.cvf, nsteps)


class Ensemble:
    """Independent RBC runs (SFF; Pr_option PRLARGE / PRSMALL, Uscaling ULARGE / USMALL) of
    uneven sizes advanced together: one CUDA graph launch per group of ensemble steps, with
    one parallel branch per grid size."""

    def __init__(self, members, kfactor=(math.pi, 2 * math.pi, 2 * math.pi), dt: float = 1e-4,
                 precision: str = "f32", dealias: str = "reference", reality_fix: bool = True,
                 Pr_option: str = "PRLARGE", Uscaling: str = "ULARGE"):
        self.lib = L.load()
        c = L.TsConfig()
        self.lib.ts_config_default(ctypes.byref(c))
        c.basis = L.TS_BASIS_SFF
        for i in range(3):
            c.kfactor[i] = float(kfactor[i])
        c.precision = L.TS_F64 if precision == "f64" else L.TS_F32
        c.dealias_mode = _DEALIAS[dealias]
        c.reality_fix = int(bool(reality_fix))
        c.dt = dt
        c.force_type = L.TS_FORCE_RBC
        c.Pr_option = _PR_OPTION[Pr_option]
        c.Uscaling = _USCALING[Uscaling]
        arr = (L.TsMember * len(members))()
        for m, (N, Ra, Pr) in enumerate(members):
            N = (N, N, N) if isinstance(N, int) else N
            for i in range(3):
                arr[m].N[i] = int(N[i])
            arr[m].Ra, arr[m].Pr = float(Ra), float(Pr)
        self.members = [((N, N, N) if isinstance(N, int) else tuple(N), Ra, Pr) for N, Ra, Pr in members]
        self.precision = precision
        h = ctypes.c_void_p()
        L.check(self.lib.ts_ensemble_create(ctypes.byref(c), arr, len(members), ctypes.byref(h)), "ts_ensemble_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ts_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def member(self, m):
        """(plan handle, u_hat pointer, T_hat pointer) of member m (device memory owned by the ensemble)."""
        p, u, t = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        L.check(self.lib.ts_ensemble_member(self.h, m, ctypes.byref(p), ctypes.byref(u), ctypes.byref(t)),
                "ts_ensemble_member")
        return p, u, t

    def init_temperature(self, amp: float, kmax: float, seed: int):
        L.check(self.lib.ts_ensemble_init_temperature(self.h, amp, kmax, seed), "ts_ensemble_init_temperature")

    def run(self, nsteps: int):
        L.check(self.lib.ts_ensemble_run(self.h, nsteps), "ts_ensemble_run")

    def synchronize(self):
        L.check(self.lib.ts_ensemble_synchronize(self.h), "ts_ensemble_synchronize")

    def nusselt(self) -> np.ndarray:
        out = np.zeros(len(self.members))
        L.check(self.lib.ts_ensemble_nusselt(self.h, out.ctypes.data_as(L._D)), "ts_ensemble_nusselt")
        return out

    def health(self, clear: bool = False) -> np.ndarray:
        """Per-member status after the steps so far: TS_OK, TS_ERR_NAN or TS_ERR_TIMEOUT."""
        out = np.zeros(len(self.members), dtype=np.int32)
        L.check(self.lib.ts_ensemble_health(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(clear)),
                "ts_ensemble_health")
        return out

    def tuning(self, m: int) -> dict:
        """launch tuning of the size group of member m"""
        t = L.TsTuning()
        L.check(self.lib.ts_ensemble_get_tuning(self.h, m, ctypes.byref(t)), "ts_ensemble_get_tuning")
        return {"variant": list(t.variant), "blocks_per_sm": list(t.blocks_per_sm)}

    def set_tuning(self, m: int, tuning: dict):
        L.check(self.lib.ts_ensemble_set_tuning(self.h, m, ctypes.byref(_tuning_struct(tuning))),
                "ts_ensemble_set_tuning")

    def autotune(self, reps: int = 3) -> dict:
        """Tune every size group on whole ensemble steps (ts_ensemble_autotune); states are kept."""
        buf = ctypes.create_string_buffer(1 << 18)
        L.check(self.lib.ts_ensemble_autotune(self.h, reps, buf, len(buf)), "ts_ensemble_autotune")
        return json.loads(buf.value.decode())

    def view(self, m: int, which: str = "T"):
        """A torch tensor viewing member m's device state in place: U (3, Nx, Ny, Nz/2+1) or
        T (1, Nx, Ny, Nz/2+1), complex64 / complex128 by the ensemble's precision.  Call
        synchronize() before reading it after run()."""
        import torch
        p, u, t = self.member(m)
        Nx, Ny, Nz = self.members[m][0]
        ncomp = 3 if which == "U" else 1
        f64 = self.precision == "f64"

        class _Dev:
            pass
        d = _Dev()
        d.__cuda_array_interface__ = {"shape": (ncomp, Nx, Ny, Nz // 2 + 1), "typestr": "<c16" if f64 else "<c8",
                                      "data": ((t if which == "T" else u).value, False), "version": 3}
        return torch.as_tensor(d, device="cuda")

    def energy(self, m: int, which: str = "T") -> float:
        self.synchronize()  # ensemble steps run on the ensemble's own stream
        p, u, t = self.member(m)
        e = ctypes.c_double()
        L.check(self.lib.ts_energy(p, t if which == "T" else u, 1 if which == "T" else 3, ctypes.byref(e)), "ts_energy")
        return e.value


def ensemble_members(count: int = 64, sizes=(32, 48, 64, 96, 128), ra_range=(1e5, 1e7), Pr: float = 1.0,
                     size_seed: int = 1, ra_seed: int = 2):
    """The benchmark ensemble: sizes drawn uniformly (seed 1) and Ra log-uniform (seed 2) with this
    project's counter-based generator (splitmix64, as the initial conditions)."""
    def u01(seed, n):
        def sm(x):
            x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
            x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
            x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
            return x ^ (x >> 31)
        key = sm(seed)
        return [(sm(key ^ i) >> 11) * (1.0 / 9007199254740992.0) for i in range(n)]
    su, ru = u01(size_seed, count), u01(ra_seed, count)
    lo, hi = math.log(ra_range[0]), math.log(ra_range[1])
    return [(sizes[min(int(a * len(sizes)), len(sizes) - 1)], math.exp(lo + b * (hi - lo)), Pr) for a, b in zip(su, ru)]


def shard_members(members, rank: int, world: int):
    """Indices of the ensemble members that rank `rank` of `world` advances: greedy bin packing
    on the per-member cost N^3 (largest first, onto the least-loaded rank).  Members are
    independent, so ranks exchange nothing while stepping; only diagnostics are gathered."""
    cost = [int(np.prod((m[0],) * 3 if isinstance(m[0], int) else m[0])) for m in members]
    order = sorted(range(len(members)), key=lambda i: (-cost[i], i))
    load = [0] * world
    owner = [0] * len(members)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += cost[i]
        owner[i] = r
    return [i for i in range(len(members)) if owner[i] == rank]
