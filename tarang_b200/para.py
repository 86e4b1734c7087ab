"""Run inputs and text outputs in the reference's formats, for the hot-path subset.

Inputs (a reference data directory ``<dir>/in/``):

* ``para.yaml`` — the keys the IF-RK4 step reads (``Global::Read``,
  global/Global_read.cc:319-450): ``program.kind``, ``program.basis_type``,
  ``program.alias_option``, ``program.apply_strong_realitycond_alltime_switch``,
  ``field.N``, ``field.kfactor`` / ``field.L``, ``field.diss_coefficients``,
  ``time.init / final / dt_fixed``, ``force.U_switch / W_switch / T_switch /
  field_procedure / parameters``, ``PHYSICS.Pr_option / Uscaling / Rayleigh / Prandtl`` and
  ``energy_transfer.flux.no_spheres / radii``, ``io.input_field_procedure`` (1: complex
  fields, 4: ``io.init_cond_modes``).  Kinds and bases: FLUID_INCOMPRESS on
  FFF, SSF and SSS; RBC on SFF, SSF and SSS; SCALAR_INCOMPRESS and MHD_INCOMPRESS on
  FFF (``diss_coefficients`` = [nu, kappa] or [nu, eta]).  Any other kind or basis is
  refused by name (NotImplementedError), never silently changed.
* ``initial.txt`` / ``forcing.txt`` — Blitz++ 1-D arrays as text,
  ``(lb,ub)`` then ``[ v0 v1 ... ]`` (``Global::Read_IC_energy_supply_arrays``,
  Global_read.cc:822-850): E(k), H(k) of the initial condition and the energy /
  helicity supply per shell.

Outputs (``<dir>/out/``), in the layouts the reference writes and its
post-processors read:

* ``spectrum.d`` — per time ``%% Time = t``, a line with one space, then
  ``%%<label>`` and one tab-separated row per component
  (``FluidIO::Output_shell_spectrum``, fluid_base/io/output/output_energy.cc:844-868,
  ``Print_array`` fluid_base/io/FluidIO.h:327-418);
* ``flux.d`` — per time an empty line, ``%% Time = t``, ``%%flux: U2U `` and the
  Pi(R) row (``Output_flux``, incompressible/incio/output/output_ET.cc:46-86);
* ``glob.d`` — one tab-separated row per time (``Global::io::Dump_buffer``,
  global/Global.cc:447-459) with time, total energy, total dissipation and dt.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

INF_RADIUS = 1e9   # the last flux sphere encloses every mode

# (program.kind, basis_type) pairs this library steps (solvers/main.cc:113-130 picks the
# solver by kind): the fluid on FFF, SSF and SSS, RBC on SFF, SSF and SSS, the passive scalar
# and MHD on FFF
STEPPED = (("FLUID_INCOMPRESS", "FFF"), ("FLUID_INCOMPRESS", "SSF"), ("FLUID_INCOMPRESS", "SSS"),
           ("RBC", "SFF"), ("RBC", "SSF"), ("RBC", "SSS"), ("SCALAR_INCOMPRESS", "FFF"), ("MHD_INCOMPRESS", "FFF"))


@dataclass
class RunParams:
    kind: str
    basis: str
    N: tuple
    kfactor: tuple
    dealias: str                 # "reference" (alias_option DEALIAS) or "none"
    reality_fix: bool
    nu: float
    kappa: float
    dt: float
    t_init: float
    t_final: float
    Ra: float | None = None
    Pr: float | None = None
    force_on: bool = False
    force_inner: float | None = None
    force_outer: float | None = None
    force_global_alpha_beta: bool = False
    flux_radii: list = field(default_factory=list)
    input_field_procedure: int = 5   # io.input_field_procedure (1: read complex fields from in/)
    pr_option: str = "PRLARGE"       # PHYSICS.Pr_option (RBC)
    uscaling: str = "ULARGE"         # PHYSICS.Uscaling (RBC)
    init_cond_modes: list = field(default_factory=list)   # io.init_cond_modes: ((kx, ky, kz), values)

    @property
    def nsteps(self) -> int:
        return int(round((self.t_final - self.t_init) / self.dt))


def _flag(v) -> bool:
    if isinstance(v, bool):
        return v
    return str(v).strip().lower() in ("1", "true", "yes", "on")


def read_blitz_arrays(path: str) -> list:
    """All ``(lb,ub) [ ... ]`` 1-D arrays of a Blitz++ text file, in order."""
    text = open(path).read()
    out = []
    for m in re.finditer(r"\(\s*(-?\d+)\s*,\s*(-?\d+)\s*\)\s*\[([^\]]*)\]", text):
        lb, ub = int(m.group(1)), int(m.group(2))
        vals = np.array([float(x) for x in m.group(3).split()], dtype=np.float64)
        if vals.size != ub - lb + 1:
            raise ValueError(f"{path}: array ({lb},{ub}) holds {vals.size} values")
        out.append(vals)
    return out


def max_radius_inside(N, kfactor) -> int:
    """``Max_radius_inside`` for the FFF basis with waveno_switch (FFF_pencil_inline.h:509-539)."""
    Nx, Ny, Nz = N
    if Ny > 1:
        return int(min((Nx // 2) * kfactor[0], (Ny // 2) * kfactor[1], (Nz // 2) * kfactor[2]))
    return int(min((Nx // 2) * kfactor[0], (Nz // 2) * kfactor[2]))


def default_flux_radii(no_spheres: int, rmax: float) -> list:
    """The sphere radii the reference builds when none are given
    (Global_process_advanced_vars.cc:133-154): 0, 2, 4, 8, then geometric up to
    rmax/2, rmax and INF_RADIUS; no_spheres + 1 values."""
    r = [0.0] * (no_spheres + 1)
    fixed = [0.0, 2.0, 4.0, 8.0]
    for i, v in enumerate(fixed):
        if i <= no_spheres:
            r[i] = v
    r[no_spheres - 2] = rmax / 2.0
    r[no_spheres - 1] = float(rmax)
    r[no_spheres] = INF_RADIUS
    if no_spheres > 6:
        s = math.log2(rmax / 16.0) / (no_spheres - 5)
        for i in range(4, no_spheres - 2):
            r[i] = 8 * 2 ** (s * (i - 3))
    return r


def read_para(path: str) -> RunParams:
    """The hot-path subset of a reference ``para.yaml``."""
    import yaml
    with open(path) as f:
        # yaml-cpp accepts trailing tabs and tab-only lines, which PyYAML rejects; strip them
        p = yaml.safe_load("\n".join(line.rstrip() for line in f.read().split("\n")))
    prog, fld, tim = p["program"], p["field"], p["time"]
    kind = str(prog["kind"]).strip()
    basis = str(prog["basis_type"]).strip()
    if (kind, basis) not in STEPPED:
        raise NotImplementedError(f"program.kind {kind} with basis_type {basis}: this library steps "
                                  + ", ".join(f"{k} on {b}" for k, b in STEPPED))
    N = tuple(int(n) for n in fld["N"])
    # kfactor, else from L, else the basis defaults (FFF_pencil.cc:34-66, SFF_pencil.cc:40-80,
    # SSF_pencil.cc:40-80, SSS_pencil.cc:40-80: RBC (pi, pi/sqrt2, pi/sqrt2), otherwise 1)
    if fld.get("kfactor") and len(fld["kfactor"]) == 3:
        kf = tuple(float(k) for k in fld["kfactor"])
    elif fld.get("L") and len(fld["L"]) == 3:
        # Fourier directions: 2 pi / L; the sin/cos direction: pi / L
        L = [float(x) for x in fld["L"]]
        kf = tuple((math.pi if (basis[i] in "SC") else 2 * math.pi) / L[i] for i in range(3))
    elif kind == "RBC":
        kf = (math.pi, math.pi / math.sqrt(2.0), math.pi / math.sqrt(2.0))
    else:
        kf = (1.0, 1.0, 1.0)
    alias = str(prog.get("alias_option", "DEALIAS")).strip()
    diss = [float(x) for x in (fld.get("diss_coefficients") or [0.0])]
    rp = RunParams(kind=kind, basis=basis, N=N, kfactor=kf,
                   dealias="reference" if alias == "DEALIAS" else "none",
                   reality_fix=_flag(prog.get("apply_strong_realitycond_alltime_switch", False)),
                   nu=diss[0], kappa=diss[1] if len(diss) > 1 else 0.0,
                   dt=float(tim["dt_fixed"]), t_init=float(tim.get("init") or 0.0), t_final=float(tim["final"]))
    if kind == "RBC":
        ph = p.get("PHYSICS") or {}
        pr_opt = str(ph.get("Pr_option", "PRLARGE")).strip()
        usc = str(ph.get("Uscaling", "USMALL")).strip()
        if pr_opt not in ("PRLARGE", "PRSMALL", "PRZERO", "PRINFTY") or usc not in ("ULARGE", "USMALL"):
            raise NotImplementedError(f"PHYSICS Pr_option {pr_opt} / Uscaling {usc}")
        if pr_opt in ("PRZERO", "PRINFTY") and basis != "SFF":
            raise NotImplementedError(f"PHYSICS Pr_option {pr_opt} on {basis}: the slaved scalings step on SFF")
        rp.pr_option, rp.uscaling = pr_opt, usc
        rp.Ra = float(ph.get("Rayleigh", 2000.0))
        rp.Pr = float(ph.get("Prandtl", 1.0))
        # diss_coefficients of the scaling (Iscalar_main.cc:52-92; ULARGE: sqrt(Pr/Ra), 1/sqrt(Pr Ra))
        from .solver import rbc_diss_coefficients
        rp.nu, rp.kappa = rbc_diss_coefficients(pr_opt, usc, rp.Ra, rp.Pr)
    force = p.get("force") or {}
    procs = force.get("field_procedure")
    procs = [int(x) for x in (procs if isinstance(procs, list) else [procs]) if x is not None]
    # field_procedure 0 is decay (no force); RBC's buoyancy (51) is part of the RBC step
    switches = [_flag(force.get(s, False)) for s in ("U_switch", "W_switch", "T_switch")]
    if kind != "RBC" and any(switches) and procs and any(x != 0 for x in procs):
        if (kind, basis) != ("FLUID_INCOMPRESS", "FFF") or switches[1] or switches[2]:
            raise NotImplementedError(f"force.field_procedure {procs} for {kind} on {basis}: "
                                      "decay (0) only; the forced step is the FFF fluid one")
        if switches[0]:
            if procs != [1]:
                raise NotImplementedError(f"force.field_procedure {procs}: Carati energy supply (1) only")
            params = force.get("parameters") or []
            words = str(params[0] if isinstance(params, list) and params else params or "").split()
            if not words or words[0] != "ENERGY_SUPPLY" or len(words) < 4:
                raise NotImplementedError(f"force.parameters {params}: 'ENERGY_SUPPLY global inner outer' only")
            rp.force_on = True
            rp.force_global_alpha_beta = _flag(words[1])
            rp.force_inner, rp.force_outer = float(words[2]), float(words[3])
            if rp.force_global_alpha_beta:
                raise NotImplementedError("ENERGY_SUPPLY with global_alpha_beta = 1: the non-global branch only")
    io = p.get("io") or {}
    if io.get("input_field_procedure") is not None:
        rp.input_field_procedure = int(io["input_field_procedure"])
    if rp.input_field_procedure == 4:
        # Global_read.cc:506-540: coord [kx, ky, kz] and the mode's values, complex
        # "(re,im)" entries (real numbers on SSS)
        for m in io.get("init_cond_modes") or []:
            rp.init_cond_modes.append((tuple(int(k) for k in m["coord"]), _mode_values(m["mode"])))
    et = p.get("energy_transfer") or {}
    fl = et.get("flux") or {}
    if _flag(et.get("turnon", False)) and _flag(fl.get("turnon", False)):
        ns = int(fl.get("no_spheres") or 0)
        radii = fl.get("radii")
        if radii and len(radii) == ns + 1:
            rp.flux_radii = [float(x) for x in radii]
        elif ns > 0:
            rp.flux_radii = default_flux_radii(ns, max_radius_inside(N, kf))
    return rp


def plan_from_dir(data_dir: str, precision: str = "f64", nlin_form: str = "conservative"):
    """(Plan, RunParams) for a reference data directory (``in/para.yaml`` and, for a
    forced run, ``in/forcing.txt``)."""
    from .solver import Forcing, Plan
    rp = read_para(os.path.join(data_dir, "in", "para.yaml"))
    forcing = None
    if rp.force_on:
        arrs = read_blitz_arrays(os.path.join(data_dir, "in", "forcing.txt"))
        forcing = Forcing(rp.force_inner, rp.force_outer, arrs[0], arrs[1] if len(arrs) > 1 else None)
    kw = dict(precision=precision, dealias=rp.dealias, kfactor=rp.kfactor, reality_fix=rp.reality_fix, dt=rp.dt)
    if rp.kind == "RBC":
        plan = Plan(rp.N, basis=rp.basis, nu=rp.nu, kappa=rp.kappa, Ra=rp.Ra, Pr=rp.Pr, Pr_option=rp.pr_option,
                    Uscaling=rp.uscaling, **kw)
    elif rp.kind in ("SCALAR_INCOMPRESS", "MHD_INCOMPRESS"):
        # the second dissipation coefficient: kappa of T, or eta of B (stored as the plan's kappa)
        plan = Plan(rp.N, nlin_form="conservative", nu=rp.nu, kappa=rp.kappa, **kw)
    elif rp.basis in ("SSF", "SSS"):
        plan = Plan(rp.N, basis=rp.basis, nlin_form="conservative", nu=rp.nu, **kw)
    else:
        plan = Plan(rp.N, nlin_form=nlin_form, nu=rp.nu, forcing=forcing, **kw)
    return plan, rp


def n_fields(kind: str) -> int:
    """How many fields one step advances: U alone, or U with T (RBC, passive scalar) or B (MHD)."""
    return 1 if kind == "FLUID_INCOMPRESS" else 2


def advance(plan, kind: str, fields, nsteps: int = 1):
    """nsteps IF-RK4 steps of the fields of a run of this kind, the RK4 the reference's
    solver for the kind calls (RK_VF.cc, RK_SF.cc, RK_VF_MHD.cc): ``fields`` is (u,) for
    FLUID_INCOMPRESS, (u, T) for RBC and SCALAR_INCOMPRESS, (u, b) for MHD_INCOMPRESS."""
    if len(fields) != n_fields(kind):
        raise ValueError(f"{kind} advances {n_fields(kind)} field(s), got {len(fields)}")
    if kind == "FLUID_INCOMPRESS":
        plan.rk4_step(fields[0], nsteps)
    elif kind == "RBC":
        plan.rk4_step_rbc(fields[0], fields[1], nsteps)
    elif kind == "SCALAR_INCOMPRESS":
        plan.rk4_step_scalar(fields[0], fields[1], nsteps)
    elif kind == "MHD_INCOMPRESS":
        plan.rk4_step_mhd(fields[0], fields[1], nsteps)
    else:
        raise NotImplementedError(f"program.kind {kind}")


# ----------------------------------------------------------------------------
# complex-field checkpoints (restart)
# ----------------------------------------------------------------------------
STATE_FORMAT = "tarang_b200 spectral state 1"


def field_layout(kind: str) -> list:
    """(field name, component names) of the fields a run of this kind advances, named as the
    reference names its complex-field datasets (CVF::Write_complex_field Cvf.cc:494-508:
    U.V1, U.V2, U.V3; a scalar field's F: T.F; the second vector field of MHD: W.V1..V3)."""
    if kind == "FLUID_INCOMPRESS":
        return [("U", ("V1", "V2", "V3"))]
    if kind in ("RBC", "SCALAR_INCOMPRESS"):
        return [("U", ("V1", "V2", "V3")), ("T", ("F",))]
    if kind == "MHD_INCOMPRESS":
        return [("U", ("V1", "V2", "V3")), ("W", ("V1", "V2", "V3"))]
    raise NotImplementedError(f"program.kind {kind}")


def save_state(folder: str, plan, kind: str, fields, t: float, step: int = 0) -> str:
    """Write the state of a run (the fields of ``advance``) as one raw little-endian file per
    component, ``<name>.<comp>.bin`` (the component's spectral array, C order, the plan's
    precision: complex (Nx, Ny, Nz/2+1), or on SSS the real coefficients in the padded
    (Nx, Ny, Nz+2) layout), plus ``state.json`` (format, kind, basis, N, kfactor, precision,
    dt, t, step, files).  The reference writes the same components as HDF5 datasets into
    out/time_<t>/ (Cvf.cc:494-508); no HDF5 library is used here."""
    import json
    os.makedirs(folder, exist_ok=True)
    layout = field_layout(kind)
    if len(fields) != len(layout):
        raise ValueError(f"{kind} has {len(layout)} field(s), got {len(fields)}")
    files = []
    for (name, comps), f in zip(layout, fields):
        if f.shape[0] != len(comps):
            raise ValueError(f"field {name}: {len(comps)} components expected, got {f.shape[0]}")
        host = f.detach().to("cpu").contiguous().numpy()
        for c, cn in enumerate(comps):
            fn = f"{name}.{cn}.bin"
            np.ascontiguousarray(host[c]).astype(host.dtype.newbyteorder("<"), copy=False).tofile(
                os.path.join(folder, fn))
            files.append({"field": name, "component": cn, "file": fn, "shape": list(host.shape[1:]),
                          "dtype": str(host.dtype)})
    cfg = plan.cfg
    head = {"format": STATE_FORMAT, "kind": kind, "basis": plan.basis, "N": list(plan.N),
            "kfactor": [float(cfg.kfactor[i]) for i in range(3)],
            "precision": "f64" if fields[0].dtype.itemsize == 16 else "f32",
            "dt": float(cfg.dt), "t": float(t), "step": int(step), "files": files}
    with open(os.path.join(folder, "state.json"), "w") as fh:
        json.dump(head, fh, indent=1)
    return folder


def load_state(folder: str, plan, kind: str, device: str = "cuda"):
    """(fields, t, step) from a folder written by ``save_state``: device tensors in the plan's
    precision (an FP64 state is rounded once for an FP32 plan).  The geometry, basis and kind
    must match the plan's, else ValueError (Read_complex_field reads into the run's own
    arrays, which fixes their shape)."""
    import json
    import torch
    with open(os.path.join(folder, "state.json")) as fh:
        head = json.load(fh)
    if head.get("format") != STATE_FORMAT:
        raise ValueError(f"{folder}: not a {STATE_FORMAT!r} folder")
    if head["kind"] != kind or head["basis"] != plan.basis or tuple(head["N"]) != tuple(plan.N):
        raise ValueError(f"{folder}: state of {head['kind']} on {head['basis']} {head['N']}, "
                         f"run is {kind} on {plan.basis} {list(plan.N)}")
    kf = [float(plan.cfg.kfactor[i]) for i in range(3)]
    if any(abs(a - b) > 1e-12 * max(1.0, abs(b)) for a, b in zip(head["kfactor"], kf)):
        raise ValueError(f"{folder}: kfactor {head['kfactor']} differs from the run's {kf}")
    by = {(f["field"], f["component"]): f for f in head["files"]}
    want = torch.complex64 if plan.precision == "f32" else torch.complex128
    out = []
    for name, comps in field_layout(kind):
        arrs = []
        for cn in comps:
            f = by.get((name, cn))
            if f is None:
                raise ValueError(f"{folder}: {name}.{cn} missing")
            a = np.fromfile(os.path.join(folder, f["file"]), dtype=np.dtype(f["dtype"]).newbyteorder("<"))
            arrs.append(a.reshape(f["shape"]))
        t = torch.from_numpy(np.stack(arrs)).to(want).to(device)
        out.append(t.contiguous())
    return out, float(head["t"]), int(head["step"])


def _mode_values(items) -> list:
    """The values of one ``init_cond_modes`` entry: numbers, or complex numbers written
    "(re,im)" as yaml-cpp reads them (PyYAML splits a flow list at every comma, so the
    items are joined back before the pairs are read)."""
    import re
    text = ",".join(str(v) for v in (items if isinstance(items, list) else [items]))
    out = []
    for pair_re, pair_im, num in re.findall(r"\(\s*([^,()\s]+)\s*,\s*([^,()\s]+)\s*\)|([^,()\s]+)", text):
        out.append(complex(float(pair_re), float(pair_im)) if pair_re else complex(float(num), 0.0))
    return out


def _last_component(rp: RunParams, kx: int, ky: int, kz: int, Vx: complex, Vy: complex):
    """Universal::Last_component: the third component from incompressibility, or the input
    pair reinterpreted on the kz = 0 plane (FFF_pencil_basic.cc:51-73; SFF_pencil_basic.cc:
    51-83 with Vx a sine series, sincostr_switch "SFF": d_x Vx = +Kx Vx)."""
    Kx, Ky, Kz = kx * rp.kfactor[0], ky * rp.kfactor[1], kz * rp.kfactor[2]
    dvx = 1j * Kx * Vx if rp.basis == "FFF" else Kx * Vx
    if kz != 0:
        return Vx, Vy, (dvx + 1j * Ky * Vy) / (-1j * Kz)
    if ky != 0:
        return Vx, dvx / (-1j * Ky), Vy
    if rp.basis == "FFF":
        return 0j, Vx, Vy
    return 0j, complex(Vx.real, 0.0), complex(Vy.real, 0.0)


def init_cond_modes(rp: RunParams) -> list:
    """FluidIO::Init_cond_modes for ``io.input_field_procedure: 4`` (init_cond_modes.cc:
    56-100 fluid, 153-221 scalar / RBC, 224-275 RBC PRZERO / PRINFTY) on FFF and SFF:
    host arrays (complex128, the spectral layout) of the run's fields with every listed
    mode set.  Per mode (kx, ky, kz): the fluid reads Vx and, for Ny > 1, Vy; the scalar
    and RBC (PRLARGE, PRSMALL) read Vx, Vy and the scalar G; PRINFTY reads G only and
    PRZERO the fluid's values (their slaved field comes from ``Plan.rbc_slave``).  The last
    velocity component is ``_last_component``; Assign_field_and_comp_conj (FluidVF.cc:
    407-433, FluidSF.cc:265-292) also sets, on the kz = 0 plane, the mirror mode
    (FFF (-kx, -ky), SFF (kx, -ky)) of the velocity to its conjugate, and, on the kz = 0
    and kz = Nz/2 planes, the scalar's mirror to the same value G (the reference assigns
    G there, not its conjugate).  Modes outside the array are skipped (Assign_spectral_field
    range check).  Then Read_init_cond's preprocessing (init_cond_main.cc:80-88, 138-150):
    the strong reality condition (always for the fluid, with
    apply_strong_realitycond_alltime_switch for the scalar kinds) and, on SFF, Zero_modes
    (SFF_pencil_basic.cc:214-243: the sine components Vx and T at kx = 0).  Other kinds
    and bases are refused by name."""
    if rp.basis not in ("FFF", "SFF") or rp.kind not in ("FLUID_INCOMPRESS", "RBC", "SCALAR_INCOMPRESS"):
        raise NotImplementedError(f"io.input_field_procedure 4 for {rp.kind} on {rp.basis}: "
                                  "the fluid, scalar and RBC modes on FFF and SFF")
    Nx, Ny, Nz = rp.N
    H = Nz // 2 + 1
    U = np.zeros((3, Nx, Ny, H), np.complex128)
    scal = rp.kind != "FLUID_INCOMPRESS"
    T = np.zeros((1, Nx, Ny, H), np.complex128) if scal else None

    def index(kx, ky, kz):
        lx = kx if rp.basis == "SFF" else (kx + Nx if kx < 0 else kx)
        ly = ky + Ny if ky < 0 else ky
        ok = 0 <= lx < Nx and 0 <= ly < Ny and 0 <= kz < H
        return (lx, ly, kz) if ok else None

    def mirror(kx, ky):
        return (-kx, -ky) if rp.basis == "FFF" else (kx, -ky)

    def put_vector(kx, ky, kz, V):
        i = index(kx, ky, kz)
        if i is not None:
            U[(slice(None),) + i] = V
        if kz == 0:
            j = index(*mirror(kx, ky), kz)
            if j is not None:
                U[(slice(None),) + j] = np.conj(V)

    def put_scalar(kx, ky, kz, G):
        i = index(kx, ky, kz)
        if i is not None:
            T[(0,) + i] = G
        if kz == 0 or kz == Nz // 2:
            j = index(*mirror(kx, ky), kz)
            if j is not None:
                T[(0,) + j] = G

    prinfty = rp.kind == "RBC" and rp.pr_option == "PRINFTY"
    fluid_only = rp.kind == "FLUID_INCOMPRESS" or (rp.kind == "RBC" and rp.pr_option == "PRZERO")
    for (kx, ky, kz), vals in rp.init_cond_modes:
        vals = list(vals) + [0j] * 3
        if prinfty:
            put_scalar(kx, ky, kz, vals[0])
            continue
        Vy = vals[1] if (Ny > 1 or not fluid_only) else 0j
        put_vector(kx, ky, kz, np.array(_last_component(rp, kx, ky, kz, vals[0], Vy)))
        if not fluid_only:
            put_scalar(kx, ky, kz, vals[2])
    if not scal or rp.reality_fix:
        U = np.stack([_strong_reality(rp, U[c]) for c in range(3)])
        if scal:
            T = _strong_reality(rp, T[0])[None]
    if rp.basis == "SFF":
        U[0, 0] = 0
        if scal:
            T[0, 0] = 0
    return [U] if not scal else [U, T]


def _strong_reality(rp: RunParams, A: np.ndarray) -> np.ndarray:
    """Satisfy_strong_reality_condition_in_Array on one component: FFF (FFF_pencil_basic.cc:
    139-179) A(kx, ky, 0) = conj A(-kx, -ky, 0) for kx < 0 (ky != Ny/2) and for kx = 0,
    ky < 0; SFF (SFF_pencil_basic.cc:143-167) A(m, ky, 0) = conj A(m, -ky, 0) for ky < 0;
    then the kz = Nz/2 plane is zero."""
    Nx, Ny, Nz = rp.N
    B = A.copy()
    ky = np.where(np.arange(Ny) <= Ny // 2, np.arange(Ny), np.arange(Ny) - Ny)
    neg_y = (-ky) % Ny
    if rp.basis == "FFF":
        kx = np.where(np.arange(Nx) <= Nx // 2, np.arange(Nx), np.arange(Nx) - Nx)
        for lx in range(Nx):
            if kx[lx] < 0:
                src = (-kx[lx]) % Nx
                for ly in range(Ny):
                    if ky[ly] != Ny // 2 or Ny == 1:
                        B[lx, ly, 0] = np.conj(B[src, neg_y[ly], 0])
        for ly in range(Ny):
            if ky[ly] < 0:
                B[0, ly, 0] = np.conj(B[0, neg_y[ly], 0])
    else:
        for ly in range(Ny):
            if ky[ly] < 0:
                B[:, ly, 0] = np.conj(B[:, neg_y[ly], 0])
    if Nz // 2 < B.shape[2] and Nz > 1:
        B[:, :, Nz // 2] = 0
    return B


def init_cond_energy_spectrum(data_dir: str, plan, rp: RunParams, seed: int = 0):
    """FluidIO::Init_cond_energy_helicity_spectrum for ``io.input_field_procedure: 5`` on an
    FFF fluid run (init_cond_energy.cc:67-120): the shell energies E(k) of
    ``<data_dir>/in/initial.txt`` (its first Blitz array, Global::Read_IC_energy_supply_arrays,
    Global_read.cc:822-833), a solenoidal random-phase field with exactly that energy per
    shell, no rescaling, then the strong reality condition (init_cond_main.cc:80-84).  The
    reference seeds its phases from the clock; here they come from ``seed`` (splitmix64), so
    a run is repeatable.  A nonzero helicity spectrum (the second array), other kinds and
    other bases are refused by name."""
    if rp.kind != "FLUID_INCOMPRESS" or rp.basis != "FFF":
        raise NotImplementedError(f"io.input_field_procedure 5 for {rp.kind} on {rp.basis}: the FFF fluid only")
    arrs = read_blitz_arrays(os.path.join(data_dir, "in", "initial.txt"))
    if not arrs:
        raise ValueError(f"{data_dir}/in/initial.txt: no E(k) array")
    if len(arrs) > 1 and np.any(arrs[1] != 0):
        raise NotImplementedError("io.input_field_procedure 5 with a helicity spectrum: non-helical fields only")
    u = plan.field(3)
    plan.init_energy_spectrum(arrs[0], seed, 0.0, u)
    return u


def read_init_cond(data_dir: str, plan, rp: RunParams):
    """FluidIO::Read_init_cond (init_cond_main.cc:48-56): ``io.input_field_procedure: 1``
    (Init_cond_complex_field init_cond_field.cc:49-58) reads the run's complex fields from
    ``<data_dir>/in/`` as ``save_state`` writes them; ``4`` sets the listed modes
    (``init_cond_modes``); ``5`` builds an FFF fluid field from E(k)
    (``init_cond_energy_spectrum``).  Returns (fields, t, step); the run continues from
    time t.  Other procedures are refused by name."""
    if rp.input_field_procedure == 5:
        return [init_cond_energy_spectrum(data_dir, plan, rp)], rp.t_init, 0
    if rp.input_field_procedure == 4:
        import torch
        want = torch.complex64 if plan.precision == "f32" else torch.complex128
        fields = [torch.from_numpy(a).to(want).to("cuda").contiguous() for a in init_cond_modes(rp)]
        if rp.kind == "RBC" and rp.pr_option in ("PRZERO", "PRINFTY"):
            plan.rbc_slave(fields[0], fields[1])
        return fields, rp.t_init, 0
    if rp.input_field_procedure != 1:
        raise NotImplementedError(f"io.input_field_procedure {rp.input_field_procedure}: "
                                  "1 (complex fields from in/), 4 (modes) and 5 (E(k) of an FFF fluid) only")
    fields, t, step = load_state(os.path.join(data_dir, "in"), plan, rp.kind)
    if rp.kind == "RBC" and rp.pr_option in ("PRZERO", "PRINFTY"):
        # Init_cond_RBC_complex_field (init_cond_field.cc:176-190): the slaved field is
        # computed from the advanced one (T = U.V1 / K^2, or U from T)
        plan.rbc_slave(fields[0], fields[1])
    return fields, t, step


# ----------------------------------------------------------------------------
# text outputs
# ----------------------------------------------------------------------------
def _row(values) -> str:
    """One Print_array row: every value followed by a tab (ostream_iterator with "\\t")."""
    return "".join(f"{float(v):g}\t" for v in values) + "\n"


def write_spectrum(f, t: float, ek: list, dissk: list | None = None, force_k: list | None = None):
    """One time block of spectrum.d: %%Uek (one row per component), %%UDk, %%(Fv.v)(k)."""
    f.write(f"%% Time = {t:g}\n \n")
    for label, rows in (("Uek", ek), ("UDk", dissk), ("(Fv.v)(k)", force_k)):
        if rows is None:
            continue
        f.write(f"%%{label}\n")
        for r in rows:
            f.write(_row(r))


def write_flux(f, t: float, flux, power_in_sphere=None):
    """One time block of flux.d: %%flux: U2U  and optionally %%sum(Fv.v)."""
    f.write(f"\n%% Time = {t:g}\n")
    f.write("%%flux: U2U \n")
    f.write(_row(flux))
    if power_in_sphere is not None:
        f.write("%%sum(Fv.v)\n")
        f.write(_row(power_in_sphere))


def write_glob_row(f, values):
    """One glob.d row (Dump_buffer: tab-separated packet, newline)."""
    f.write(_row(values))


def sff_max_radius_inside(N, kfactor) -> int:
    """``Max_radius_inside`` for the SFF basis with waveno_switch (SFF_pencil_inline.h:436-452):
    min((Nx - 1) Kx, (Ny/2) Ky, (Nz/2) Kz), truncated."""
    Nx, Ny, Nz = N
    return int(min((Nx - 1) * kfactor[0], (Ny // 2) * kfactor[1], (Nz // 2) * kfactor[2]))


def ssf_max_radius_inside(N, kfactor) -> int:
    """``Max_radius_inside`` for the SSF basis with waveno_switch (SSF_pencil_inline.h:456-474):
    min((Nx - 1) Kx, (Ny - 1) Ky, (Nz/2) Kz), truncated."""
    Nx, Ny, Nz = N
    return int(min((Nx - 1) * kfactor[0], (Ny - 1) * kfactor[1], (Nz // 2) * kfactor[2]))


def sss_max_radius_inside(N, kfactor) -> int:
    """``Max_radius_inside`` for the SSS basis with waveno_switch (SSS_pencil_inline.h:481-499):
    min((Nx - 1) Kx, (Ny - 1) Ky, (Ny - 1) Kz) as the reference writes it (its third term
    takes Ny, not Nz), truncated."""
    Nx, Ny, Nz = N
    return int(min((Nx - 1) * kfactor[0], (Ny - 1) * kfactor[1], (Ny - 1) * kfactor[2]))


def _fff_multiplicity(kx, ky, kz, Nx, Ny):
    """Multiplicity_factor (FFF_pencil_inline.h:583-602): 1 (kz > 0) or 1/2 (kz = 0),
    doubled on the kx = Nx/2 and ky = Ny/2 planes."""
    f = np.where(kz > 0, 1.0, 0.5)
    return np.where((kx == Nx // 2) | ((ky == Ny // 2) & (Ny > 1)), 2 * f, f)


class Output:
    """Appends out/glob.d, out/spectrum.d and out/flux.d for an FFF plan in the reference's
    layouts.

    spectrum.d (FluidIO::Output_shell_spectrum): %%Uek = per-component shell
    spectra (Compute_shell_spectrum, n = 0); %%UDk = 2 x per-component raw sums of
    mult K^2 |A|^2, rescaled by Approx_number_modes_in_shell / count beyond the
    inscribed sphere (Compute_shell_spectrum_force with n = 2,
    universal_energy.cc:196-262); for a forced plan %%(Fv.v)(k) = 2 x the
    component cross spectra of u and the force (Compute_force_shell_spectrum,
    Correlation.cc:457-469).
    flux.d (Output_flux): %%flux: U2U = Pi(R_i) (ts_flux, after dealiasing u in place
    as the reference's Compute_flux does) and %%sum(Fv.v) = the
    power the force puts into the shells between consecutive radii, modes inside
    the inscribed sphere only (Shell_mult_all, universal_ET.cc:145-176).
    """

    def __init__(self, plan, out_dir: str, radii=None):
        os.makedirs(out_dir, exist_ok=True)
        self.plan = plan
        self.out_dir = out_dir
        self.kf = tuple(plan.cfg.kfactor[i] for i in range(3))
        self.kmax_inside = {"FFF": max_radius_inside, "SFF": sff_max_radius_inside, "SSF": ssf_max_radius_inside,
                            "SSS": sss_max_radius_inside}[plan.basis](plan.N, self.kf)
        self.radii = list(radii) if radii is not None else default_flux_radii(8, self.kmax_inside)
        self.forced = plan.cfg.force_type != 0

    def save(self, kind: str, fields, t: float, step: int = 0) -> str:
        """The run's complex fields into out/time_<t>/ (CVF::Write_complex_field, Cvf.cc:494-508,
        folder "time_" + time.now) in ``save_state``'s format; ``read_init_cond`` restarts from it."""
        return save_state(os.path.join(self.out_dir, f"time_{t:g}"), self.plan, kind, fields, t, step)

    def _force(self, u):
        return self.plan.force_field(u, self.plan.field(3)) if self.forced else None

    def spectrum(self, u, t: float):
        if self.plan.basis != "FFF":
            raise NotImplementedError("this output is written for FFF fluid runs")
        p = self.plan
        kfp = self.kf[0] * self.kf[1] * self.kf[2]
        idx = np.arange(p.n_shells, dtype=np.float64)
        approx = 4 * math.pi * idx ** 2 / kfp    # Approx_number_modes_in_shell (FFF_pencil_inline.h:558-565)
        ek, dissk, fvk = [], [], None
        for i in range(3):
            ui = u[i:i + 1]
            ek.append(p.shell_spectrum(ui, 1))
            s, c = p.shell_sums(ui, ncomp=1)
            d = s.copy()
            out = (idx > self.kmax_inside) & (c >= 1)
            d[out] = s[out] * approx[out] / c[out]
            dissk.append(2 * d)
        if self.forced:
            F = self._force(u)
            fvk = []
            for i in range(3):
                s, c = p.shell_sums(u[i:i + 1], F[i:i + 1], ncomp=1)
                fvk.append(2 * np.where(c > 0, s * 4 * math.pi / np.where(c > 0, c, 1) / kfp, 0.0))
        with open(os.path.join(self.out_dir, "spectrum.d"), "a") as f:
            write_spectrum(f, t, ek, dissk, fvk)

    def glob(self, u, t: float, dt: float, helicity: bool = False):
        """One row of out/glob.d (FluidIO::Output_global, output_energy.cc:69-117): time,
        total energy, dissipation nu * total_k2energy (total_k2energy = 2 sum mult K^2 |V|^2,
        Cvf.cc:224-227), helicity1, helicity2, k2H1, k2H2 (2 mult K.(Vr x Vi) summed, / K^2,
        and the K^2 moments; FFF_pencil_energy.cc:99-139; zero when helicity is off), the
        modal-energy entropy in bits (universal_energy.cc:449-473), kmax * Kolmogorov scale,
        nu, R_lambda = 2 E sqrt(15 / eps), dt, and the three component energies."""
        if self.plan.basis != "FFF":
            raise NotImplementedError("this output is written for FFF fluid runs")
        import torch
        p = self.plan
        nu = float(p.cfg.nu)
        E = [p.energy(u[i:i + 1], 1) for i in range(3)]
        Etot = E[0] + E[1] + E[2]
        k2 = 2 * sum(float(p.shell_sums(u[i:i + 1], ncomp=1)[0].sum()) for i in range(3))
        eps = nu * k2
        Nx, Ny, Nz = p.N
        dev = u.device
        lx = torch.arange(Nx, device=dev)
        ly = torch.arange(Ny, device=dev)
        kx = torch.where(lx <= Nx // 2, lx, lx - Nx).double()[:, None, None]
        ky = torch.where(ly <= Ny // 2, ly, ly - Ny).double()[None, :, None]
        kz = torch.arange(Nz // 2 + 1, device=dev).double()[None, None, :]
        mult = torch.where(kz > 0, 1.0, 0.5) * torch.where((kx == Nx // 2) | ((ky == Ny // 2) & (Ny > 1)), 2.0, 1.0)
        K = [kx * self.kf[0], ky * self.kf[1], kz * self.kf[2]]
        K2 = (K[0] ** 2 + K[1] ** 2) + K[2] ** 2
        v = u.to(torch.complex128)
        H1 = H2 = k2H1 = k2H2 = 0.0
        if helicity:
            vr, vi = v.real, v.imag
            cr = [vr[1] * vi[2] - vr[2] * vi[1], vr[2] * vi[0] - vr[0] * vi[2], vr[0] * vi[1] - vr[1] * vi[0]]
            h = 2 * mult * (K[0] * cr[0] + K[1] * cr[1] + K[2] * cr[2])
            H1 = float(h.sum())
            H2 = float(torch.where(K2 > 1e-15, h / torch.where(K2 > 1e-15, K2, 1.0), 0.0).sum())
            k2H1 = 2 * float((K2 * h).sum())
            k2H2 = 2 * H1
        modal = mult * (v.abs() ** 2).sum(0)
        prob = modal / Etot
        ent = float(torch.where(prob > 1e-15, -prob * torch.log(torch.where(prob > 1e-15, prob, 1.0)) / math.log(2.0),
                                0.0).sum())
        kmax_eta = self.kmax_inside * (nu ** 3 / eps) ** 0.25 if eps > 0 else float("inf")
        rlam = 2 * Etot * math.sqrt(15 / eps) if eps > 0 else float("inf")
        row = [t, Etot, eps, H1, H2, k2H1, k2H2, ent, kmax_eta, nu, rlam, dt, E[0], E[1], E[2]]
        with open(os.path.join(self.out_dir, "glob.d"), "a") as f:
            write_glob_row(f, row)
        return row

    def flux(self, u, t: float):
        if self.plan.basis not in ("FFF", "SSF", "SSS"):
            raise NotImplementedError("flux.d is written for fluid runs on FFF, SSF and SSS")
        p = self.plan
        # Compute_flux runs Compute_nlin(U, Giver), which dealiases U in place
        # (compute_nlin_ET_VF.cc:73-76): the run goes on from the dealiased state
        p.dealias(u)
        # spheres 1..no_spheres; the entry at radii[0] is never computed and stays 0
        # (flux_self = 0.0, compute_flux.cc:55-64)
        Pi = np.zeros(len(self.radii))
        if len(self.radii) > 1:
            Pi[1:] = p.flux(u, self.radii[1:])
        power = None
        if self.forced:
            F = self._force(u)
            Nx, Ny, Nz = p.N
            km = int(math.ceil(p.cfg.force_outer_radius / min(self.kf)))
            kx = np.arange(-km, km + 1)
            kz = np.arange(0, km + 1)
            import torch
            lx = torch.as_tensor(kx % Nx, device=u.device)
            ly = torch.as_tensor(kx % Ny, device=u.device)
            Fc = F[:, lx][:, :, ly][..., :km + 1].cpu().numpy()
            Uc = u[:, lx][:, :, ly][..., :km + 1].cpu().numpy()
            KX, KY, KZ = np.meshgrid(kx, kx, kz, indexing="ij")
            K = np.sqrt((KX * self.kf[0]) ** 2 + (KY * self.kf[1]) ** 2 + (KZ * self.kf[2]) ** 2)
            dot = np.sum((Fc * np.conj(Uc)).real, axis=0)
            w = 2 * _fff_multiplicity(KX, KY, KZ, Nx, Ny) * dot
            power = np.zeros(len(self.radii))
            ins = K <= self.kmax_inside
            b = np.searchsorted(np.asarray(self.radii), K[ins], side="left")   # first radius >= |K|
            np.add.at(power, np.minimum(b, len(self.radii) - 1), w[ins])
        with open(os.path.join(self.out_dir, "flux.d"), "a") as f:
            write_flux(f, t, Pi, power)

    def glob_rbc(self, u, T, t: float, dt: float):
        """One row of out/glob.d for an RBC run on SFF (FluidIO::Output_global_RBC,
        output_energy.cc:214-303; helicity_switch off, so the four helicity columns
        are 0): time, E_u, E_T, nu k2E_u, kappa k2E_T (k2E = 2 sum mult K^2 |A|^2,
        Get_total_Sn universal_energy.cc:106-141; no hyperviscosity), Nusselt
        (Correlation.cc:154-156), H1, H2, k2H1, k2H2, the modal entropies of u and T in
        bits (universal_energy.cc:449-537), kmax eta_1 = kmax (nu^3/eps)^(1/4),
        kmax eta_2 = kmax eta_1 (nu/kappa)^(1/4) / (nu/kappa), nu, kappa,
        R_lambda = 2 E_u sqrt(15/eps), dt, and the three component energies of u.
        kmax = Max_radius_inside of the basis; mult = its Multiplicity_factor
        (SFF_pencil_inline.h:492-515; on SSF and SSS 1/2 at the origin, 1, 2 or 4 with two,
        one or no zero indices, SSF_pencil_inline.h:512-532, SSS_pencil_inline.h:537-556).
        The sums run over the complex array shape as the reference's loops do
        (universal_energy.cc:106-141): on SSS each pair of real z coefficients is one
        complex slot lz with Kz = lz kfactor_z."""
        if self.plan.basis == "FFF":
            raise NotImplementedError("glob_rbc writes RBC runs on the SFF, SSF and SSS bases")
        return self._glob_uT(u, T, t, dt, nusselt=True)

    def glob_scalar(self, u, T, t: float, dt: float, helicity: bool = False):
        """One row of out/glob.d for a passive-scalar run on FFF (FluidIO::Output_global_scalar,
        output_energy.cc:134-205): the RBC row without the Nusselt column (20 columns),
        with the FFF multiplicity (FFF_pencil_inline.h:583-602) and Max_radius_inside.
        (The reference's Output_global(U, T) picks this row for program.kind INC_SCALAR,
        output_energy.cc:125, while its solver runs kind SCALAR_INCOMPRESS, main.cc:116.)
        With helicity (the reference's helicity_switch), columns 6-9 hold H1, H2, k2H1, k2H2
        of u."""
        if self.plan.basis != "FFF":
            raise NotImplementedError("glob_scalar writes passive-scalar runs on the FFF basis")
        return self._glob_uT(u, T, t, dt, nusselt=False, helicity=helicity)

    def glob_mhd(self, u, b, t: float, dt: float, helicity: bool = False):
        """One row of out/glob.d for an MHD run on FFF (FluidIO::Output_global(U, W),
        output_energy.cc:404-499; helicity_switch off, so the eight helicity columns are
        0): time, E_u, E_b, nu k2E_u, eta k2E_b, the cross helicity Hc = sum_i <u_i, b_i>
        (Correlation.cc:225-230), ((nu + eta)/2) k2Hc (k2Hc = 2 sum mult K^2 Re(u . b*),
        Cvf.cc:235-238), 8 helicity columns, the entropies of u and b, kmax eta_1,
        kmax eta_2 (with nu / eta), nu, eta, R_lambda, dt, and the component energies of
        u and of b: 29 columns.  eta is the plan's kappa.  With helicity (the reference's
        helicity_switch) the helicity columns hold H1_u, H2_u, H1_b, H2_b, k2H1_u, k2H2_u,
        k2H1_b, k2H2_b."""
        import torch
        p = self.plan
        if p.basis != "FFF":
            raise NotImplementedError("glob_mhd writes MHD runs on the FFF basis")
        nu, eta = float(p.cfg.nu), float(p.cfg.kappa)
        mult, K2 = self._mult_K2(u.device)
        v, w = u.to(torch.complex128), b.to(torch.complex128)
        Eu_c = [p.energy(u[i:i + 1], 1) for i in range(3)]
        Eb_c = [p.energy(b[i:i + 1], 1) for i in range(3)]
        Eu, Eb = sum(Eu_c), sum(Eb_c)
        d = (v * w.conj()).real.sum(0)
        Hc = float(d.sum() - 0.5 * d[:, :, 0].sum())   # FFF plane weights of Get_local_energy(A, B)
        k2u = 2 * float((mult * K2 * (v.abs() ** 2).sum(0)).sum())
        k2b = 2 * float((mult * K2 * (w.abs() ** 2).sum(0)).sum())
        k2Hc = 2 * float((mult * K2 * d).sum())
        eps, epsb = nu * k2u, eta * k2b
        kmax = self.kmax_inside
        keta1 = kmax * (nu ** 3 / eps) ** 0.25 if eps > 0 else float("inf")
        r = nu / eta
        keta2 = keta1 * r ** 0.25 / r
        rlam = 2 * Eu * math.sqrt(15 / eps) if eps > 0 else float("inf")
        hu = self._helicity(v) if helicity else [0.0] * 4
        hb = self._helicity(w) if helicity else [0.0] * 4
        row = ([t, Eu, Eb, eps, epsb, Hc, 0.5 * (nu + eta) * k2Hc] + hu[:2] + hb[:2] + hu[2:] + hb[2:] +
               [self._entropy(mult, v, Eu), self._entropy(mult, w, Eb), keta1, keta2, nu, eta, rlam, dt] +
               Eu_c + Eb_c)
        with open(os.path.join(self.out_dir, "glob.d"), "a") as f:
            write_glob_row(f, row)
        return row

    def _helicity(self, v):
        """H1, H2, k2H1, k2H2 of a spectral vector field on FFF (FFF_pencil_energy.cc:99-139):
        h = 2 mult K . (Vr x Vi) summed, / K^2, and the K^2 moments"""
        import torch
        p = self.plan
        if p.basis != "FFF":
            raise NotImplementedError("helicity columns are written for FFF runs")
        Nx, Ny, Nz = p.N
        dev = v.device
        lx, ly = torch.arange(Nx, device=dev), torch.arange(Ny, device=dev)
        K = [torch.where(lx <= Nx // 2, lx, lx - Nx).double()[:, None, None] * self.kf[0],
             torch.where(ly <= Ny // 2, ly, ly - Ny).double()[None, :, None] * self.kf[1],
             torch.arange(Nz // 2 + 1, device=dev).double()[None, None, :] * self.kf[2]]
        mult, K2 = self._mult_K2(dev)
        vr, vi = v.real, v.imag
        cr = [vr[1] * vi[2] - vr[2] * vi[1], vr[2] * vi[0] - vr[0] * vi[2], vr[0] * vi[1] - vr[1] * vi[0]]
        h = 2 * mult * (K[0] * cr[0] + K[1] * cr[1] + K[2] * cr[2])
        H1 = float(h.sum())
        H2 = float(torch.where(K2 > 1e-15, h / torch.where(K2 > 1e-15, K2, 1.0), 0.0).sum())
        return [H1, H2, 2 * float((K2 * h).sum()), 2 * H1]

    @staticmethod
    def _entropy(mult, a, etot):
        """modal-energy entropy in bits, mult |A|^2 / E as the probabilities (universal_energy.cc:449-537)"""
        import torch
        prob = mult * (a.abs() ** 2).sum(0) / etot
        return float(torch.where(prob > 1e-15, -prob * torch.log(torch.where(prob > 1e-15, prob, 1.0))
                                 / math.log(2.0), 0.0).sum())

    def _mult_K2(self, dev):
        """Multiplicity_factor (FFF_pencil_inline.h:583-602, SFF_pencil_inline.h:492-515) and K^2
        per stored mode of the plan's basis"""
        import torch
        p = self.plan
        Nx, Ny, Nz = p.N
        lxi = torch.arange(Nx, device=dev)
        ly = torch.arange(Ny, device=dev)
        ky = torch.where(ly <= Ny // 2, ly, ly - Ny).double()[None, :, None]
        lz = torch.arange(Nz // 2 + 1, device=dev).double()[None, None, :]
        if p.basis in ("SSF", "SSS"):
            # grid indices; the SSS z slot lz holds the real pair (2 lz, 2 lz + 1)
            lx = lxi.double()[:, None, None]
            ky = ly.double()[None, :, None]
            zeros = (lx == 0).double() + (ky == 0).double() + (lz == 0).double()
            mult = torch.where(zeros >= 3, 0.5, torch.where(zeros == 2, 1.0, torch.where(zeros == 1, 2.0, 4.0)))
        elif p.basis == "SFF":
            lx = lxi.double()[:, None, None]
            mult = torch.where(lz > 0, torch.where(lx > 0, 2.0, 1.0), torch.where(lx > 0, 1.0, 0.5))
            mult = mult * torch.where((ky == Ny // 2) & (Ny > 1), 2.0, 1.0)
        else:
            lx = torch.where(lxi <= Nx // 2, lxi, lxi - Nx).double()[:, None, None]
            mult = torch.where(lz > 0, 1.0, 0.5) * torch.where((lx == Nx // 2) | ((ky == Ny // 2) & (Ny > 1)), 2.0, 1.0)
        K2 = (lx * self.kf[0]) ** 2 + (ky * self.kf[1]) ** 2 + (lz * self.kf[2]) ** 2
        return mult, K2

    def _glob_uT(self, u, T, t: float, dt: float, nusselt: bool, helicity: bool = False):
        import torch
        p = self.plan
        nu, kappa = float(p.cfg.nu), float(p.cfg.kappa)
        Nx, Ny, Nz = p.N
        mult, K2 = self._mult_K2(u.device)
        v = u.to(torch.complex128)
        th = T.to(torch.complex128).reshape(1, Nx, Ny, Nz // 2 + 1)
        E = [p.energy(u[i:i + 1], 1) for i in range(3)]
        Eu = E[0] + E[1] + E[2]
        ET = p.energy(T, 1)
        k2u = 2 * float((mult * K2 * (v.abs() ** 2).sum(0)).sum())
        k2T = 2 * float((mult * K2 * (th.abs() ** 2).sum(0)).sum())
        eps, epsT = nu * k2u, kappa * k2T
        Nu = [p.nusselt(u, T)] if nusselt else []

        kmax = self.kmax_inside
        keta1 = kmax * (nu ** 3 / eps) ** 0.25 if eps > 0 else float("inf")
        r = nu / kappa
        keta2 = keta1 * r ** 0.25 / r
        rlam = 2 * Eu * math.sqrt(15 / eps) if eps > 0 else float("inf")
        hel = self._helicity(v) if helicity else [0.0] * 4
        row = [t, Eu, ET, eps, epsT] + Nu + hel + [self._entropy(mult, v, Eu),
                                            self._entropy(mult, th, ET), keta1, keta2, nu, kappa, rlam, dt,
                                            E[0], E[1], E[2]]
        with open(os.path.join(self.out_dir, "glob.d"), "a") as f:
            write_glob_row(f, row)
        return row
