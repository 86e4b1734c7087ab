#!/usr/bin/env python
"""Benchmark: IF-RK4 steps/s of the forced-turbulence workload on B200.

Workload (default): FFF 256^3, Carati constant energy supply on shell 3
(band 2 < |K| <= 3, epsilon = 0.1), nu = 1e-3, dt = 5e-4, initial E(k) ~
k^4 exp(-2 (k/4)^2) random phase (seed 0), total energy 0.5, two-thirds
dealiasing, rotational (u x omega) form, FP32 transforms with FP64 sums and
integrating factor.  One step = one full IF-RK4 step (4 right-hand sides).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tarang_b200|reference]

Multi-GPU (torchrun, one rank per GPU): the field does not shard (no pencil
decomposition), so ranks run independent replicas; value = steps of all ranks
/ max-over-ranks time ("scaling": "weak").  `--impl reference` times the FP64
CPU restatement of the reference algorithm (oracle/tarang_ref.py) on the host
cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 steps/s, FFF forced turbulence 256^3 (FP32 transforms, FP64 sums)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tarang_b200", choices=["tarang_b200", "reference"])
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--form", default="rotational", choices=["rotational", "conservative"])
    ap.add_argument("--no-extras", action="store_true", help="skip the FP64 comparison, e2e and CPU baseline legs")
    ap.add_argument("--workload", default="fff256",
                    choices=["fff256", "ensemble", "fff1024", "rbc", "adjoint", "scalar", "mhd", "ssf", "sss",
                             "rbc_ssf", "rbc_sss", "c1_trajectory", "c2_error"],
                    help="fff256: forced 256^3 (default headline); ensemble: 64 RBC members; fff1024: decaying "
                         "1024^3 (or --shape); rbc: one RBC run (SFF, --N, FP32); adjoint: adjoint/forward cost at 128^3")
    ap.add_argument("--tune", default="auto", choices=["auto", "off"],
                    help="auto: pick kernel candidates with the library's autotuner before warm-up "
                         "(untimed set-up); off: the fixed tile rules")
    ap.add_argument("--shape", default="1024,1024,1024",
                    help="grid of the fff1024 workload, Nx,Ny,Nz (smaller shapes exercise the same kernels)")
    return ap.parse_args()


TUNE = {"mode": "auto"}


def tune_plan(plan, reps: int = 3) -> dict | None:
    """Run the library autotuner on a plan (set-up, outside every timed region); returns the picks."""
    if TUNE["mode"] == "off":
        return None
    rep = plan.autotune(reps=reps)
    return {"tuning": rep["tuning"], "confirm": rep["confirm"]}


def ensemble_leg(rank: int, world: int, steps: int, warmup: int):
    """Config 3: 64 RBC members (SFF, N in {32,48,64,96,128}, Ra log-uniform [1e5,1e7], Pr=1, FP32,
    dt=1e-4), members greedily packed onto ranks by N^3; returns per-rank timing and model bytes."""
    import torch
    import tarang_b200 as tb
    allm = tb.ensemble_members()
    members = [allm[i] for i in tb.shard_members(allm, rank, world)]
    ens = tb.Ensemble(members, dt=1e-4, precision="f32", dealias="reference")
    ens.init_temperature(1e-3, 4.0, 3)
    tuned = None
    if TUNE["mode"] == "auto":
        rep = ens.autotune(reps=3)
        tuned = [{"N": gr["N"], "members": gr["members"], "confirm": gr["tuning"]["confirm"],
                  **gr["tuning"]["final"]} for gr in rep["groups"]]
        tuned.append({"schedule": rep.get("schedule"), "parallel_ms": rep.get("parallel_ms"),
                      "serial_ms": rep.get("serial_ms")})
    ens.run(warmup)
    ens.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.run(steps)
    ens.synchronize()
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    Nu = ens.nusselt()
    ens.close()
    model = sum(408.0 * m[0] ** 3 * 4 for m in members)   # SFF RBC byte model per member step, FP32
    return {"members": len(members), "seconds": wall, "steps": steps, "model_bytes_per_step": model,
            "nusselt_mean": float(np.mean(Nu)), "nusselt_finite": bool(np.all(np.isfinite(Nu))), "tuning": tuned}


def fff1024_leg(steps: int = 3, warmup: int = 2, shape=(1024, 1024, 1024), prec: str = "f32", tune: bool = True):
    """Config 2: FFF 1024^3 decaying turbulence, rotational, IC k^4 exp(-2(k/8)^2) E=0.5,
    nu=2e-4, dt=2e-4; steps/s and the per-kernel rates (FP32 by default; FP64 untuned is the
    plain FP64 GPU path the FP32 rate is compared with)."""
    import torch
    import ctypes
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = tb.Plan(tuple(shape), precision=prec, nlin_form="rotational", dealias="two_thirds", nu=2e-4, dt=2e-4)
    plan.set_stream(torch.cuda.current_stream())   # the timing events below go on this stream
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 8.0), 0, 0.5, u)
    tuned = tune_plan(plan, reps=1) if tune else None
    plan.rk4_step(u, warmup)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clk = Clocks(torch.cuda.current_device())
    clk.start()
    e0.record()
    plan.rk4_step(u, steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    # per-kernel rates from one further, separately profiled step
    L.check(plan.lib.ts_profile_reset(plan.h), "reset")
    L.check(plan.lib.ts_profile_enable(plan.h, 1), "enable")
    plan.rk4_step(u, 1)
    torch.cuda.synchronize()
    L.check(plan.lib.ts_profile_enable(plan.h, 0), "disable")
    kern = {}
    for k, name in enumerate(L.KCLASS_NAMES):
        tot, n, b = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
        L.check(plan.lib.ts_profile_read(plan.h, k, ctypes.byref(tot), ctypes.byref(n), ctypes.byref(b)), "read")
        if n.value and b.value:
            kern[name] = round(b.value / (tot.value / n.value / 1e3) / 1e9, 1)
    n3 = float(shape[0]) * shape[1] * shape[2]
    sb = 4 if prec == "f32" else 8
    out = {"steps_per_s": steps / (ms / 1e3), "kernel_GBps": kern, "energy": plan.energy(u),
           "model_frac": 288.0 * n3 * sb * steps / (ms / 1e3) / 1e9 / measured_peak()[0], "tuning": tuned,
           "clocks": clocks}
    plan.close()
    del u
    torch.cuda.empty_cache()
    return out


def c1_trajectory_leg(steps: int = 2000, every: int = 10, N: int = 256, form: str = "rotational"):
    """Config 1's error report: FP32 and FP64 GPU runs of the forced 256^3 workload (same IC,
    same nonlinear form) advanced side by side; every `every` steps the relative L2 difference
    of the velocity fields, the relative energy difference and max |div u| of each run.  The
    FP64 run is the reference the FP32 path is held to (rel err <= 1e-5); forced turbulence
    is chaotic, so the difference grows with time, and the report says where it crosses 1e-5."""
    import torch
    import tarang_b200 as tb
    nsh = int(math.ceil(math.sqrt(3) * (N // 2))) + 1
    forcing = tb.Forcing(2.0, 3.0, energy_supply(nsh))
    kw = dict(nlin_form=form, dealias="two_thirds", nu=1e-3, dt=5e-4, forcing=forcing)
    p32, p64 = tb.Plan(N, precision="f32", **kw), tb.Plan(N, precision="f64", **kw)
    st = torch.cuda.current_stream()
    p32.set_stream(st)
    p64.set_stream(st)
    u64 = p64.field(3)
    p64.init_energy_spectrum(tb.spectrum_k4_gauss(p64.n_shells, 4.0), 0, 0.5, u64)
    u32 = u64.to(torch.complex64)
    rows = []
    t0 = time.perf_counter()
    for s in range(1, steps + 1):
        p32.rk4_step(u32, 1)
        p64.rk4_step(u64, 1)
        if s % every == 0 or s == 1:
            d = float(torch.linalg.vector_norm(u32.to(torch.complex128) - u64) / torch.linalg.vector_norm(u64))
            e32, e64 = p32.energy(u32), p64.energy(u64)
            rows.append([s, d, abs(e32 - e64) / e64, p32.max_div(u32), p64.max_div(u64), e64])
    p32.status()
    p64.status()
    wall = time.perf_counter() - t0
    first = next((r[0] for r in rows if r[1] > 1e-5), None)
    first_e = next((r[0] for r in rows if r[2] > 1e-5), None)
    out = {"steps": steps, "every": every, "N": N, "form": form,
           "columns": ["step", "rel_l2_u", "rel_energy", "max_div_f32", "max_div_f64", "energy_f64"],
           "series": rows, "first_step_rel_l2_above_1e-5": first, "first_step_rel_energy_above_1e-5": first_e,
           "final": dict(zip(["step", "rel_l2_u", "rel_energy", "max_div_f32", "max_div_f64", "energy_f64"], rows[-1])),
           "max_div_f32_max": max(r[3] for r in rows), "wall_s": wall}
    p32.close()
    p64.close()
    del u32, u64
    torch.cuda.empty_cache()
    return out


def c2_error_leg(steps: int = 200, every: int = 10, shape=(1024, 1024, 1024)):
    """Config 2's error report: the 1024^3 decaying run (rotational, two-thirds, nu = 2e-4,
    dt = 2e-4, IC k^4 exp(-2 (k/8)^2), E = 0.5) in FP32 and then in FP64 (the two do not fit
    on one GPU together: the FP32 state waits in host memory), energies every `every` steps
    and, at the end, the relative L2 difference of the velocity fields."""
    import torch
    import tarang_b200 as tb
    kw = dict(nlin_form="rotational", dealias="two_thirds", nu=2e-4, dt=2e-4)
    energies = {}
    final32 = None
    for prec in ("f32", "f64"):
        plan = tb.Plan(tuple(shape), precision=prec, **kw)
        plan.set_stream(torch.cuda.current_stream())
        u = plan.field(3)
        plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 8.0), 0, 0.5, u)
        es = [[0, plan.energy(u)]]
        t0 = time.perf_counter()
        for s in range(1, steps + 1):
            plan.rk4_step(u, 1)
            if s % every == 0:
                es.append([s, plan.energy(u)])
        plan.status()
        energies[prec] = {"series": es, "wall_s": time.perf_counter() - t0, "max_div": plan.max_div(u)}
        if prec == "f32":
            final32 = u.cpu()
            plan.close()
            del u
            torch.cuda.empty_cache()
        else:
            num = 0.0
            for c in range(3):
                num += float(torch.linalg.vector_norm(final32[c].to("cuda").to(torch.complex128) - u[c]) ** 2)
            rel_l2 = math.sqrt(num) / float(torch.linalg.vector_norm(u))
            plan.close()
            del u
            torch.cuda.empty_cache()
    rel_e = [[a[0], abs(a[1] - b[1]) / b[1]] for a, b in zip(energies["f32"]["series"], energies["f64"]["series"])]
    return {"steps": steps, "shape": list(shape), "rel_l2_u_final": rel_l2, "rel_energy": rel_e,
            "max_rel_energy": max(r[1] for r in rel_e), "energies": energies}


def ensemble_plain_fp64_leg(steps: int = 3, warmup: int = 1):
    """The 64 ensemble members advanced the plain way: one FP64 plan per member, stepped one
    after another with ts_rk4_step_rbc (no batching, no graph, the fixed tile rules).  Returns
    ensemble-steps/s (all 64 members advanced once per ensemble step), CUDA-event timed."""
    import torch
    import tarang_b200 as tb
    members = tb.ensemble_members()
    plans, states = [], []
    for (N, Ra, Pr) in members:
        p = tb.Plan(N, basis="SFF", precision="f64", dealias="reference", Ra=Ra, Pr=Pr, dt=1e-4,
                    nu=math.sqrt(Pr / Ra), kappa=1 / math.sqrt(Pr * Ra), kfactor=(math.pi, 2 * math.pi, 2 * math.pi))
        p.set_stream(torch.cuda.current_stream())
        u, T = p.field(3), p.field(1)
        p.init_temperature_perturbation(1e-3, 4.0, 3, T)
        plans.append(p)
        states.append((u, T))
    for p, (u, T) in zip(plans, states):
        p.rk4_step_rbc(u, T, warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        for p, (u, T) in zip(plans, states):
            p.rk4_step_rbc(u, T, 1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    for p in plans:
        p.close()
    del states
    torch.cuda.empty_cache()
    return {"ensemble_steps_per_s": steps / (ms / 1e3), "members": len(members), "steps": steps,
            "how": "64 FP64 plans stepped one after another, fixed tile rules, CUDA events"}


def coupled_leg(kind: str, N: int, steps: int, warmup: int, prec: str = "f32"):
    """FFF passive scalar ("scalar") or incompressible MHD ("mhd") at N^3: decaying, nu = 1e-3,
    kappa / eta = 1e-3, dt = 5e-4, two-thirds dealias; U (and B) from the k^4 exp(-2(k/4)^2)
    spectrum (seeds 0, 1), the scalar a copy of u1.  Steps/s (CUDA events) and the per-class
    kernel times; model bytes 90 (scalar) / 114 (MHD) S s per right-hand side."""
    import torch
    import ctypes
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = tb.Plan(N, precision=prec, nu=1e-3, kappa=1e-3, dt=5e-4, dealias="two_thirds")
    plan.set_stream(torch.cuda.current_stream())
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    if kind == "mhd":
        w = plan.field(3)
        plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 1, 0.3, w)
        step = lambda n: plan.rk4_step_mhd(u, w, n)
    else:
        w = u[0:1].clone()
        step = lambda n: plan.rk4_step_scalar(u, w, n)
    step(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    step(steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    L.check(plan.lib.ts_profile_reset(plan.h), "reset")
    L.check(plan.lib.ts_profile_enable(plan.h, 1), "enable")
    step(1)
    torch.cuda.synchronize()
    L.check(plan.lib.ts_profile_enable(plan.h, 0), "disable")
    kern = {}
    for k, name in enumerate(L.KCLASS_NAMES):
        tot, n, b = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
        L.check(plan.lib.ts_profile_read(plan.h, k, ctypes.byref(tot), ctypes.byref(n), ctypes.byref(b)), "read")
        if n.value:
            kern[name] = round(tot.value, 4)
    S = N * N * (N // 2 + 1)
    sb = 8 if prec == "f32" else 16
    model = (90 if kind == "scalar" else 114) * 4 * S * sb
    plan.close()
    return {"steps_per_s": steps / (ms / 1e3), "ms_per_step_by_class": kern,
            "model_GBps": model * steps / (ms / 1e3) / 1e9,
            "model_frac": model * steps / (ms / 1e3) / 1e9 / measured_peak()[0]}


def ssf_leg(N: int, steps: int, warmup: int, prec: str = "f32", basis: str = "SSF", rbc: bool = False):
    """SSF (sin/cos along x and y) or SSS (along every axis) fluid step at N^3: conservative,
    unforced, nu = 1e-3, dt = 5e-4, reference dealias, kfactor (pi, pi, 2 pi) / (pi, pi, pi);
    a small seeded random spectral field (amplitude 1e-3; the timing does not depend on the
    values).  With rbc, the Boussinesq step (Ra = 1e6, Pr = 1, ULARGE nu / kappa, dt = 1e-4,
    the basis's RBC kfactor (pi, pi/sqrt2, pi/sqrt2)) with a seeded temperature of the same
    amplitude.  Steps/s, CUDA events."""
    import torch
    import tarang_b200 as tb
    if rbc:
        r2 = math.sqrt(2.0)
        plan = tb.Plan(N, basis=basis, precision=prec, dealias="reference", Ra=1e6, Pr=1.0, dt=1e-4,
                       nu=math.sqrt(1.0 / 1e6), kappa=1.0 / math.sqrt(1e6), kfactor=(math.pi, math.pi / r2, math.pi / r2))
    else:
        plan = tb.Plan(N, basis=basis, precision=prec, nu=1e-3, dt=5e-4, dealias="reference",
                       kfactor=(math.pi, math.pi, 2 * math.pi if basis == "SSF" else math.pi))
    plan.set_stream(torch.cuda.current_stream())
    gen = torch.Generator(device="cuda").manual_seed(0)
    u = plan.field(3)
    u.real.copy_(1e-3 * torch.randn(u.shape, generator=gen, device="cuda"))
    T = plan.field(1)
    T.real.copy_(1e-3 * torch.randn(T.shape, generator=gen, device="cuda"))
    step = (lambda n: plan.rk4_step_rbc(u, T, n)) if rbc else (lambda n: plan.rk4_step(u, n))
    step(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    step(steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"steps_per_s": steps / (ms / 1e3)}
    if rbc:
        out["nusselt"] = plan.nusselt(u, T)
    plan.close()
    return out


def rbc_leg(N: int, steps: int, warmup: int):
    """One Boussinesq (RBC) run on the SFF basis at N^3, FP32, Ra = 1e6, Pr = 1, kfactor (pi, 2pi, 2pi),
    dt = 1e-4, T perturbation 1e-3 on k <= 4 (seed 3): steps/s and per-kernel rates."""
    import torch
    import ctypes
    import tarang_b200 as tb
    from tarang_b200 import _lib as L
    plan = tb.Plan(N, basis="SFF", precision="f32", dealias="reference", Ra=1e6, Pr=1.0, dt=1e-4,
                   kfactor=(math.pi, 2 * math.pi, 2 * math.pi))
    plan.set_stream(torch.cuda.current_stream())
    u, T = plan.field(3), plan.field(1)
    plan.init_temperature_perturbation(1e-3, 4.0, 3, T)
    tuned = tune_plan(plan)
    plan.rk4_step_rbc(u, T, warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.rk4_step_rbc(u, T, steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    L.check(plan.lib.ts_profile_reset(plan.h), "reset")
    L.check(plan.lib.ts_profile_enable(plan.h, 1), "enable")
    plan.rk4_step_rbc(u, T, 1)
    torch.cuda.synchronize()
    L.check(plan.lib.ts_profile_enable(plan.h, 0), "disable")
    kern = {}
    for k, name in enumerate(L.KCLASS_NAMES):
        tot, n, b = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
        L.check(plan.lib.ts_profile_read(plan.h, k, ctypes.byref(tot), ctypes.byref(n), ctypes.byref(b)), "read")
        if n.value:
            kern[name] = {"ms_per_step": round(tot.value, 4),
                          "GBps": round(b.value / (tot.value / n.value / 1e3) / 1e9, 1) if b.value else None}
    nu = plan.nusselt(u, T)
    plan.close()
    return {"steps_per_s": steps / (ms / 1e3), "kernels": kern, "nusselt": nu,
            "model_frac": 408.0 * N ** 3 * 4 * steps / (ms / 1e3) / 1e9 / measured_peak()[0], "tuning": tuned}


def adjoint_leg(prec: str, N: int = 128, window: int = 20, reps: int = 3):
    """Config 4: adjoint/forward cost at 128^3 (nu=5e-3, dt=1e-3, rotational, two-thirds).  Times a
    forward step, one adjoint step (its four adjoint right-hand sides) and one checkpoint window
    (recompute `window` steps keeping stages, then `window` adjoint steps), all with CUDA events."""
    import torch
    import tarang_b200 as tb
    plan = tb.Plan(N, precision=prec, nu=5e-3, dt=1e-3, dealias="two_thirds", nlin_form="rotational")
    plan.set_stream(torch.cuda.current_stream())
    u = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 0, 0.5, u)
    lam = plan.field(3)
    plan.init_energy_spectrum(tb.spectrum_k4_gauss(plan.n_shells, 4.0), 1, 0.5, lam)
    st = torch.empty((9,) + plan.spec_shape, dtype=u.dtype, device=u.device)
    un = u.clone()
    work = torch.empty(plan.adjoint_work_bytes(window), dtype=torch.uint8, device=u.device)

    def timed(fn, n):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    fwd = timed(lambda: plan.rk4_step(un, 1), 10 * reps)
    plan.rk4_step_keep(u, un, st)
    adj = timed(lambda: plan.adjoint_step(u, st, lam), 10 * reps)
    win = timed(lambda: plan.adjoint_window(u, window, lam, work), reps)
    plan.close()
    return {"forward_step_ms": fwd, "adjoint_step_ms": adj, "adjoint_over_forward": adj / fwd,
            "window_ms": win, "window_steps": window,
            "adjoint_with_recompute_over_forward": win / (window * fwd)}


def workload(N):
    return {"workload": f"FFF {N}^3 forced isotropic turbulence (Carati energy supply shell 3, eps=0.1), "
                        f"nu=1e-3, dt=5e-4, IC k^4 exp(-2(k/4)^2) E=0.5 seed 0",
            "N": N, "nu": 1e-3, "dt": 5e-4, "k0": 4.0, "forcing_shell": 3, "epsilon": 0.1,
            "dealias": "two_thirds"}


def energy_supply(nsh):
    es = np.zeros(nsh)
    es[3] = 0.1
    return es


# ---------------------------------------------------------------------------
# clocks sampling (nvidia-smi) during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kclass: str, N: int, prec: str):
    """DRAM bytes per launch of a kernel class from the committed ncu summary, scaled to N^3."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                p = line.split()
                if len(p) >= 5 and p[0] == "traffic" and p[1] == kclass and p[2] == prec:
                    n0, b = int(p[3]), float(p[4])
                    return b * (N / n0) ** 3
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
def cpu_baseline_oracle(N, steps_cap_s=20.0, max_steps=50):
    """Time the FP64 oracle (restatement of the reference algorithm) on this host."""
    from oracle import tarang_ref as R
    g = R.Grid((N, N, N))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=1e-3, dt=5e-4, dealias_mode=R.DEALIAS_TWO_THIRDS,
                        forcing=R.CaratiForcing(2.0, 3.0, energy_supply(g.n_shells())))
    mis = g.modes_in_shell()
    R.rk4_step(cfg, V, mis)  # warm-up (plans, page-in)
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        V = R.rk4_step(cfg, V, mis)
        n += 1
        if time.perf_counter() - t0 > steps_cap_s:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    N = args.N
    from oracle import tarang_ref as R
    g = R.Grid((N, N, N))
    V = R.init_energy_spectrum(g, R.spectrum_k4_gauss(g.n_shells(), 4.0), 0, 0.5)
    cfg = R.FluidConfig(g, nu=1e-3, dt=5e-4, dealias_mode=R.DEALIAS_TWO_THIRDS,
                        forcing=R.CaratiForcing(2.0, 3.0, energy_supply(g.n_shells())))
    mis = g.modes_in_shell()
    for _ in range(args.warmup):
        V = R.rk4_step(cfg, V, mis)
    budget = 150.0
    n, t0 = 0, time.perf_counter()
    while n < args.steps:
        V = R.rk4_step(cfg, V, mis)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = n / el
    cores = os.cpu_count()
    sample = f"{n} of {args.steps} requested RK4 steps at {N}^3 (FP64, scipy.fft workers={R.WORKERS}), {el:.1f} s"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 * el / n, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(N),
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def alt_workload(args, world, rank, local, dev):
    """The ensemble (config 3) or the 1024^3 decaying run (config 2) as the primary line."""
    import torch
    import torch.distributed as dist
    clk = Clocks(local)
    clk.start()
    if args.workload == "ensemble":
        r = ensemble_leg(rank, world, steps=args.steps, warmup=args.warmup)
        sec = r["seconds"]
        mb = r["model_bytes_per_step"]
        if world > 1:
            t = torch.tensor([sec, mb], device=dev, dtype=torch.float64)
            t2 = t.clone()
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dist.all_reduce(t2)
            sec, mb = float(t[0].item()), float(t2[1].item())
        value = args.steps / sec
        line = {"metric": "ensemble RK4 steps/s, 64 RBC members (SFF, N in {32,48,64,96,128}, FP32)",
                "value": value, "unit": "ensemble-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "64 RBC members, Ra log-uniform [1e5,1e7] (seed 2), sizes seed 1, Pr=1, "
                                       "kfactor (pi,2pi,2pi), T amp 1e-3 k<=4 (seed 3), dt=1e-4",
                           "parallelism": f"members packed on {world} GPU(s) by N^3"},
                "roofline": {"bound": "hbm", "achieved": mb * value / 1e9 / world, "peak": measured_peak()[0],
                             "unit": "GB/s", "frac": mb * value / 1e9 / world / measured_peak()[0],
                             "traffic": None, "model": "408 N^3 4 B per member step"},
                "member_steps_per_s": 64 * value}
        line["config"]["tuning"] = r["tuning"]
    elif args.workload in ("scalar", "mhd"):
        n = args.N
        r = coupled_leg(args.workload, n, steps=args.steps, warmup=args.warmup, prec=args.precision)
        what = "passive scalar" if args.workload == "scalar" else "incompressible MHD"
        line = {"metric": f"RK4 steps/s, FFF {what} {n}^3 ({args.precision} transforms, FP64 sums)",
                "value": r["steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / r["steps_per_s"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
                "config": {"workload": f"FFF {what} {n}^3, decaying, nu = kappa/eta = 1e-3, dt = 5e-4, two-thirds"},
                "roofline": {"bound": "hbm", "model_frac": r["model_frac"], "model_GBps": r["model_GBps"],
                             "ms_per_step_by_class": r["ms_per_step_by_class"]}}
    elif args.workload in ("ssf", "sss"):
        n = args.N if args.N != 256 else 128
        bas = args.workload.upper()
        r = ssf_leg(n, steps=args.steps, warmup=args.warmup, prec=args.precision, basis=bas)
        line = {"metric": f"RK4 steps/s, {bas} fluid {n}^3 ({args.precision} transforms)",
                "value": r["steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / r["steps_per_s"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
                "config": {"workload": f"{bas} fluid {n}^3, conservative, unforced, nu = 1e-3, dt = 5e-4, "
                                       "reference dealias, standalone sin/cos passes"}}
    elif args.workload in ("rbc_ssf", "rbc_sss"):
        n = args.N if args.N != 256 else 128
        bas = args.workload[4:].upper()
        r = ssf_leg(n, steps=args.steps, warmup=args.warmup, prec=args.precision, basis=bas, rbc=True)
        line = {"metric": f"RK4 steps/s, {bas} Boussinesq (RBC) {n}^3 ({args.precision} transforms)",
                "value": r["steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / r["steps_per_s"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
                "config": {"workload": f"RBC on {bas} {n}^3, Ra=1e6, Pr=1, kfactor (pi, pi/sqrt2, pi/sqrt2), "
                                       "dt=1e-4, reference dealias, standalone sin/cos passes"},
                "nusselt": r["nusselt"]}
    elif args.workload == "rbc":
        r = rbc_leg(args.N if args.N != 256 else 128, steps=args.steps, warmup=args.warmup)
        n = args.N if args.N != 256 else 128
        line = {"metric": f"RK4 steps/s, SFF Boussinesq (RBC) {n}^3 (FP32 transforms, FP64 sums)",
                "value": r["steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / r["steps_per_s"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"RBC {n}^3, Ra=1e6, Pr=1, kfactor (pi,2pi,2pi), dt=1e-4, T amp 1e-3 k<=4"},
                "roofline": {"bound": "hbm", "model_frac": r["model_frac"], "kernels": r["kernels"]},
                "nusselt": r["nusselt"]}
        line["config"]["tuning"] = r["tuning"]
    elif args.workload in ("c1_trajectory", "c2_error"):
        if args.workload == "c1_trajectory":
            r = c1_trajectory_leg(steps=args.steps if args.steps != 30 else 2000)
            what = "FP32 vs FP64 GPU, FFF 256^3 forced, rel L2 of u after the run"
            v = r["final"]["rel_l2_u"]
        else:
            r = c2_error_leg(steps=args.steps if args.steps != 30 else 200)
            what = "FP32 vs FP64 GPU, FFF 1024^3 decaying, rel L2 of u after the run"
            v = r["rel_l2_u_final"]
        line = {"metric": what, "value": v, "unit": "relative L2", "n_gpus": 1, "steps": r["steps"],
                "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 vs f64", "data": "synthetic", "config": {"workload": args.workload}, "detail": r}
    elif args.workload == "adjoint":
        r = {"f64": adjoint_leg("f64"), "f32": adjoint_leg("f32")}
        line = {"metric": "adjoint step / forward step cost, FFF 128^3 rotational (config 4)",
                "value": r["f64"]["adjoint_over_forward"], "unit": "ratio", "n_gpus": 1, "steps": 30,
                "warmup": 2, "ms_per_step": r["f64"]["adjoint_step_ms"], "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "FFF 128^3, nu=5e-3, dt=1e-3, two-thirds, window 20"}, "detail": r}
    else:
        shape = tuple(int(x) for x in args.shape.split(","))
        r = fff1024_leg(steps=args.steps, warmup=args.warmup, shape=shape)
        sh = "x".join(str(x) for x in shape)
        line = {"metric": f"RK4 steps/s, FFF decaying turbulence {sh} (FP32 transforms, FP64 sums)",
                "value": r["steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / r["steps_per_s"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"FFF {sh} decaying, IC k^4 exp(-2(k/8)^2) E=0.5 seed 0, nu=2e-4, dt=2e-4"},
                "roofline": {"bound": "hbm", "model_frac": r["model_frac"], "kernel_GBps": r["kernel_GBps"]}}
        line["config"]["tuning"] = r["tuning"]
    line["clocks"] = clk.stop()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    TUNE["mode"] = args.tune
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    import tarang_b200 as tb
    from tarang_b200 import _lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    if args.workload != "fff256":
        return alt_workload(args, world, rank, local, dev)

    N = args.N
    nsh = int(math.ceil(math.sqrt(3) * (N // 2))) + 1
    forcing = tb.Forcing(2.0, 3.0, energy_supply(nsh))
    plan = tb.Plan(N, precision=args.precision, nlin_form=args.form, dealias="two_thirds", nu=1e-3, dt=5e-4,
                   forcing=forcing)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    plan.set_stream(stream)
    u = plan.field(3)
    E_ic = tb.spectrum_k4_gauss(plan.n_shells, 4.0)
    plan.init_energy_spectrum(E_ic, 0, 0.5, u)
    u0 = u.clone()
    tuned = tune_plan(plan)

    for _ in range(args.warmup):
        plan.rk4_step(u, 1)
    torch.cuda.synchronize()

    clk = Clocks(local)
    lib = plan.lib
    L.check(lib.ts_profile_reset(plan.h), "profile_reset")
    L.check(lib.ts_profile_enable(plan.h, 1), "profile_enable")
    n_launch0 = tb.kernel_launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        plan.rk4_step(u, 1)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    launches = tb.kernel_launch_count() - n_launch0
    L.check(lib.ts_profile_enable(plan.h, 0), "profile_disable")
    prof = {}
    import ctypes
    for k, name in enumerate(L.KCLASS_NAMES):
        tot, n, b = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
        L.check(lib.ts_profile_read(plan.h, k, ctypes.byref(tot), ctypes.byref(n), ctypes.byref(b)), "profile_read")
        prof[name] = {"total_ms": tot.value, "launches": n.value, "bytes_per_launch": b.value}
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    steps_per_s = world * args.steps / (ms / 1e3)

    # dominant kernel: largest total time
    main_k = max((k for k in prof if k != "other"), key=lambda k: prof[k]["total_ms"])
    pk = prof[main_k]
    avg_s = pk["total_ms"] / max(pk["launches"], 1) / 1e3
    achieved = pk["bytes_per_launch"] / avg_s / 1e9
    peak, peak_kind = measured_peak()
    roofline = {"bound": "hbm", "kernel": main_k, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": ncu_traffic(main_k, N, args.precision),
                "bytes_per_launch": pk["bytes_per_launch"], "avg_launch_ms": avg_s * 1e3}
    # whole-step roofline against the graded byte model 288 * N^3 * s
    s_bytes = 4 if args.precision == "f32" else 8
    model_bytes = 288.0 * N ** 3 * s_bytes
    step_model = {"model_bytes_per_step": model_bytes,
                  "model_GBps": model_bytes * steps_per_s / world / 1e9,
                  "model_frac": model_bytes * steps_per_s / world / 1e9 / peak,
                  "kernels": {k: {"avg_ms": v["total_ms"] / max(v["launches"], 1), "launches": v["launches"],
                                  "GBps": (v["bytes_per_launch"] / (v["total_ms"] / max(v["launches"], 1) / 1e3) / 1e9)
                                  if v["total_ms"] > 0 and v["bytes_per_launch"] > 0 else None,
                                  "share": v["total_ms"] / sum(x["total_ms"] for x in prof.values())}
                              for k, v in prof.items()}}

    extras = {}
    e2e = None
    cpu = None
    if not args.no_extras:
        # e2e: the reference-facing C-ABI call on HOST (pinned) buffers, copies inside the call
        host = u.detach().to("cpu").pin_memory()
        k_e2e = max(3, min(args.steps, 10))
        plan.rk4_step(host, 1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k_e2e):
            plan.rk4_step(host, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        nbytes = host.numel() * host.element_size()
        e2e = {"value": world * k_e2e / (ems / 1e3), "unit": "steps/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": k_e2e}
        # FP32 vs FP64 GPU (same nonlinear form): relative L2 and energy error after 5 steps, FP64 steps/s
        if args.precision == "f32":
            p64 = tb.Plan(N, precision="f64", nlin_form=args.form, dealias="two_thirds", nu=1e-3, dt=5e-4,
                          forcing=forcing)
            p64.set_stream(stream)
            extras["fp64_tuning"] = tune_plan(p64)
            a32 = u0.clone()
            a64 = u0.to(torch.complex128)
            for _ in range(5):
                plan.rk4_step(a32, 1)
                p64.rk4_step(a64, 1)
            torch.cuda.synchronize()
            d = (a32.to(torch.complex128) - a64)
            rel_l2 = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(a64))
            e32, e64 = plan.energy(a32), p64.energy(a64)
            k64 = max(3, min(args.steps, 10))
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            p64.rk4_step(a64, k64)
            f1.record(stream)
            torch.cuda.synchronize()
            extras["fp64_gpu_steps_per_s"] = k64 / (f0.elapsed_time(f1) / 1e3)
            extras["fp32_vs_fp64_after_5_steps"] = {"rel_l2": rel_l2, "rel_energy": abs(e32 - e64) / e64}
            extras["fp32_speedup_vs_fp64"] = (steps_per_s / world) / extras["fp64_gpu_steps_per_s"]
            p64.close()
        extras["max_div_end"] = plan.max_div(u)
        extras["energy_end"] = plan.energy(u)
        if args.precision == "f32" and world == 1:
            # config 1's error report over the full 2000-step run (FP32 vs the FP64 GPU run)
            tr = c1_trajectory_leg(steps=2000, every=100, N=N, form=args.form)
            extras["c1_fp32_vs_fp64_2000_steps"] = {
                "final": tr["final"], "first_step_rel_l2_above_1e-5": tr["first_step_rel_l2_above_1e-5"],
                "first_step_rel_energy_above_1e-5": tr["first_step_rel_energy_above_1e-5"],
                "max_div_f32_max": tr["max_div_f32_max"], "columns": tr["columns"], "every_100_steps": tr["series"],
                "wall_s": tr["wall_s"]}
        # config 3: the RBC ensemble (all ranks; members shared out by N^3)
        plan.close()
        torch.cuda.empty_cache()
        ens = ensemble_leg(rank, world, steps=10, warmup=2)
        esec = ens["seconds"]
        if world > 1:
            t = torch.tensor([esec], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            esec = float(t.item())
            mb = torch.tensor([ens["model_bytes_per_step"]], device=dev, dtype=torch.float64)
            dist.all_reduce(mb)
            ens["model_bytes_per_step"] = float(mb.item())
        extras["ensemble_rbc_64"] = {"ensemble_steps_per_s": ens["steps"] / esec,
                                     "member_steps_per_s": 64 * ens["steps"] / esec,
                                     "model_GBps": ens["model_bytes_per_step"] * ens["steps"] / esec / 1e9,
                                     "nusselt_mean_rank0": ens["nusselt_mean"], "finite": ens["nusselt_finite"],
                                     "timing": "wall clock around synchronised graph launches, max over ranks"}
        if world == 1:
            extras["fff1024_f32"] = fff1024_leg()
            # the plain FP64 GPU path at the same sizes: 1024^3 (2 steps) and the ensemble members
            # one plan at a time; the north-star target is FP32 / plain FP64 >= 3
            extras["fff1024_f64_plain"] = fff1024_leg(steps=2, warmup=1, prec="f64", tune=False)
            extras["ensemble_rbc_64_fp64_plain"] = ensemble_plain_fp64_leg()
            extras["scalar_256_f32"] = coupled_leg("scalar", 256, steps=5, warmup=2)
            extras["mhd_256_f32"] = coupled_leg("mhd", 256, steps=5, warmup=2)
            extras["ssf_128_f32"] = ssf_leg(128, steps=10, warmup=3, basis="SSF")
            extras["sss_128_f32"] = ssf_leg(128, steps=10, warmup=3, basis="SSS")
            extras["rbc_sss_128_f32"] = ssf_leg(128, steps=10, warmup=3, basis="SSS", rbc=True)
            extras["fp32_over_plain_fp64"] = {
                "fff1024": extras["fff1024_f32"]["steps_per_s"] / extras["fff1024_f64_plain"]["steps_per_s"],
                "ensemble": extras["ensemble_rbc_64"]["ensemble_steps_per_s"]
                / extras["ensemble_rbc_64_fp64_plain"]["ensemble_steps_per_s"]}
            extras["adjoint_128"] = {"f64": adjoint_leg("f64"), "f32": adjoint_leg("f32")}
        if rank == 0 and world == 1:
            v, n, el = cpu_baseline_oracle(N)
            from oracle import tarang_ref as R
            cpu = {"value": v, "unit": "steps/s", "cores": R.WORKERS, "kind": "port",
                   "sample": f"{n} RK4 steps of the same {N}^3 workload in FP64 (oracle/tarang_ref.py, "
                             f"scipy.fft workers={R.WORKERS}), {el:.1f} s"}

    if rank == 0:
        line = {"metric": METRIC, "value": steps_per_s, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": args.precision, "data": "synthetic",
                "config": dict(workload(N), precision=args.precision, nlin_form=args.form,
                               parallelism=f"replicas x{world}", tuning=tuned,
                               l2="working set (12 spectral fields, %.2f GB) > L2 126 MB: inputs larger than L2"
                                  % (12 * plan.N[0] * plan.N[1] * (plan.N[2] // 2 + 1) * (8 if args.precision == "f32" else 16) / 1e9)),
                "roofline": roofline, "step_roofline": step_model, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clocks, "extras": extras}
        print(json.dumps(line), flush=True)
    if plan.h:
        plan.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
