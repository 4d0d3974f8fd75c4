"""Benchmark of the RT-TDDFT propagation hot path on the periodic-bulk workload.

Workload (one bench step): the periodic bulk system -- cubic cell a = 10.26
bohr, 8 atoms at diamond positions with 4 Gaussian KB projectors each,
16^3 grid, 64 k-points (4^3 Monkhorst-Pack), 32 complex128 orbitals per k --
propagated ``--nt`` (default 2000) middlepoint Taylor-4 steps under an
Asin2cos vector potential (omega = 1.55 eV, peak A/c = 1e-3 au), with J(t)
computed every step.  Metric: grid-point x orbital Taylor steps per second
(16^3 x 2048 x nt units per bench step), whole job over all ranks.

* ``value``: orbitals resident in HBM before the timed region (the device
  loop of sb200_rt_propagate, captured as CUDA graphs).
* ``e2e``: the same metric through the reference-facing C ABI with host
  buffers: per bench step the pinned reference-layout orbitals are uploaded
  (sb200_orbitals_from_ref), propagated, and J(t) plus the final orbitals are
  read back to the host (sb200_orbitals_to_ref) into the same buffer, which
  the next step uploads: the propagation continues through host memory.
  ``--workload isolated`` instead starts every bench step (both legs) from the
  kicked orbitals: its configuration is the run of nt steps after the kick.
* ``roofline``: the kernel that applies H (on this workload k_step_blk, the
  whole Taylor step of a block of orbitals per CTA), timed with CUDA events on the
  library's stream in an instrumented replay right after the timed region;
  algorithmic bytes 224 B per unit per Taylor step.
* ``cpu_baseline``: the CPU oracle (a C++/OpenMP restatement of the
  reference's Fortran path) on a bounded sample of the same workload.

``--impl reference`` times the reference's CPU path instead (the oracle port:
the Fortran reference cannot be compiled on these machines).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

UNIT_BYTES = {"fp64": 224.0, "mixed": 144.0}  # algorithmic bytes per grid-point x orbital Taylor step
METRIC = "grid-pt*orbital Taylor steps/s"
UNIT = "grid-pt*orbital*step/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--nt", type=int, default=None,
                    help="Taylor time steps per bench step (default 2000; 40 for the batch workload)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-steps", type=int, default=4, help="Taylor steps in each CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-supercell", action="store_true",
                    help="skip the supercell leg (FP64 and mixed) that the default periodic-bulk run adds")
    ap.add_argument("--supercell-nt", type=int, default=100, help="Taylor steps per supercell sample")
    ap.add_argument("--self-consistent", action="store_true",
                    help="V_local = Vpsl + Vh[rho] + Vxc[rho] (PZ) recomputed after every Taylor step inside the "
                         "time loop (the fixed Gaussian potential stands in for Vpsl)")
    ap.add_argument("--poisson", default="cg", choices=["cg", "ft"],
                    help="isolated self-consistent workload: Hartree by CG with the multipole boundary "
                         "(the reference's default) or by transforms on the doubled box")
    ap.add_argument("--small", action="store_true", help="8 k-points instead of 64 (quick check)")
    ap.add_argument("--workload", default="bulk", choices=["bulk", "supercell", "batch", "isolated"],
                    help="bulk: 16^3 x 64 k x 32 orbitals; supercell: its 2x2x2 supercell, 32^3 x 8 k x 256; "
                         "batch: 16 isolated systems 32^3..96^3 x 4..64 orbitals in one batch; "
                         "isolated: a 64^3 molecule (h = 0.25 A), 5 orbitals, 4 atoms, after an impulse kick")
    return ap.parse_args()


def workload(args, rank=0, world=1):
    from salmon2_b200 import synth
    if args.workload == "isolated":
        # 64^3 Dirichlet grid, h = 0.25 A, 5 complex orbitals, 4 atoms x 4 KB
        # projectors (rc = 1.2 A), 1e-3 au impulse kick along z, dt = 0.05 au;
        # every rank propagates its own copy (replicas: nothing to exchange)
        s = synth.isolated_system(num=64, h_aa=0.25, no=5, natom=4, seed=1, rc_aa=1.2)
        import dataclasses
        s = dataclasses.replace(s, psi=synth.impulse_kick(s.grid, s.psi, 1e-3))
        dt = 0.05
        return s, args.nt, dt, None, synth.taylor_zc(dt)
    if args.workload == "supercell":
        nkgrid = 1 if args.small else 2
        s = synth.periodic_system(a=10.26, num=16, nkgrid=nkgrid, no=256, supercell=2, seed=3,
                                  name="periodic_supercell")
    else:
        nkgrid = 2 if args.small else 4
        s = synth.periodic_system(a=10.26, num=16, nkgrid=nkgrid, no=32, seed=2, name="periodic_bulk")
    # weak scaling: rank r owns a shifted copy of the k-mesh (a denser mesh
    # overall); J(t) is summed over ranks
    s = synth.kpoint_shard(s, rank, world, 10.26 * (2 if args.workload == "supercell" else 1), nkgrid)
    nt = args.nt
    dt = 0.08
    omega = 1.55 / synth.AU_ENERGY_EV
    Ac = synth.asin2cos(nt, dt, omega=omega, f0=omega * 1e-3, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    return s, nt, dt, Ac, zc


def config_dict(args, s, nt, world):
    units = int(np.prod(s.grid.shape)) * s.norb * nt
    if args.workload == "isolated":
        desc = (f"isolated molecule {s.grid.shape[0]}^3 grid h=0.25 A Dirichlet, {s.no} complex128 orbitals, "
                f"{s.pp.natom} atoms x 4 KB projectors, 1e-3 au kick, dt=0.05 au, {nt} Taylor-4 steps per bench "
                f"step, dipole every step (orbital blocks fit in L2)")
    else:
        desc = (f"periodic {'supercell' if args.workload == 'supercell' else 'bulk'} a=10.26 bohr, "
                f"{s.pp.natom} atoms (diamond), {s.grid.shape[0]}^3 grid, "
                f"{s.nk} k-points, {s.no} complex128 orbitals/k, Asin2cos A(t) omega=1.55 eV "
                f"peak 1e-3 au, {nt} Taylor-4 steps per bench step, J(t) every step")
    if getattr(args, "self_consistent", False):
        desc += ", self-consistent: density, Hartree and PZ-LDA potential every step"
        if args.workload == "isolated":
            desc += (" (Hartree by CG with the multipole boundary from the extrapolated potential, layout 3, "
                     "threshold 1e-15)" if getattr(args, "poisson", "cg") == "cg"
                     else " (Hartree by transforms on the doubled box)")
    return {
        "workload": desc,
        "grid": list(s.grid.shape), "k_points": s.nk, "orbitals_per_k": s.no, "atoms": s.pp.natom,
        "projectors": s.pp.nlma, "taylor_steps_per_bench_step": nt, "units_per_bench_step_per_rank": units,
        "precision": args.precision,
        "self_consistent": bool(getattr(args, "self_consistent", False)),
        "bench_step": ("the kicked orbitals copied in (device leg) or uploaded (e2e leg), "
                       + ("their density, Hartree and PZ-LDA potential, " if getattr(
                           args, "self_consistent", False) else "")
                       + f"then {nt} steps: every step times the first {nt} steps after the kick"
                       if args.workload == "isolated" else
                       f"{nt} steps continuing the previous step's orbitals (e2e: through host memory)"),
        "parallelism": f"replicas x{world}" if args.workload == "isolated" else f"k-point shards x{world}",
        "l2": ("inputs larger than L2 (3 orbital blocks of %.0f MB each)" % (units / nt * 16 / 1e6)
               if units / nt * 16 * 3 > 126e6 else
               "orbital blocks of %.0f MB each: L2-resident, the HBM fraction is reported, not claimed"
               % (units / nt * 16 / 1e6)),
        "seed": s.seed,
    }


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        self.index = ids[index] if index < len(ids) else str(index)
        self.proc = None
        # the raw samples go to SB200_CLOCKS_DIR (default: the system temp
        # directory); their summary goes into the JSON line
        import tempfile
        self.path = os.path.join(os.environ.get("SB200_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return None
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def orbital_path(s, args):
    """The one-CTA-per-orbital kernels run periodic 16^3 grids in FP64."""
    return s.grid.periodic and tuple(s.grid.shape) == (16, 16, 16) and args.precision == "fp64"


def hpsi_kernel(s, args, units_per_launch):
    """(name, algorithmic bytes per launch) of the kernel that applies H.

    The algorithmic bytes of a Taylor step are 224 B per unit (FP64; 144 B
    mixed) whatever the kernel split: a per-term kernel is credited a quarter
    per launch, the fused-step kernel (all four terms in one launch, which
    itself moves only psi in and psi_out out) the whole 224 B."""
    if orbital_path(s, args):
        v = os.environ.get("SB200_ORBITAL", "fused")
        if v.startswith("p"):
            return "k_term_orbital_tma", UNIT_BYTES["fp64"] / 4.0 * units_per_launch
        if v.startswith("t"):
            return "k_term_orbital", UNIT_BYTES["fp64"] / 4.0 * units_per_launch
        if v.startswith("u") or (v.startswith("s") and s.pp.nlma == 0):
            return "k_step_orbital", UNIT_BYTES["fp64"] * units_per_launch
        if v.startswith("s"):
            return "k_step_orbital_st", UNIT_BYTES["fp64"] * units_per_launch  # KB tables in shared memory
        return "k_step_blk", UNIT_BYTES["fp64"] * units_per_launch  # register-blocked fused step
    name = "k_hpsi_tiled" if os.environ.get("SB200_TMA", "on").startswith("of") else "k_hpsi_tma"
    return name, UNIT_BYTES[args.precision] / 4.0 * units_per_launch


def supercell_leg(args, local):
    """The 2x2x2 supercell (32^3 grid, 64 atoms, 8 k-points, 256 orbitals/k,
    band-limited orbitals |k+G|^2/2 <= 2 Ha) propagated in the FP64 and the mixed
    form from the same start: throughput of each (resident orbitals, CUDA events
    on the library stream, 1 warm-up + 2 timed samples of `--supercell-nt`
    Taylor steps), the H psi kernel's roofline fraction, and the mixed form's
    J(t) error against the FP64 run over one sample."""
    import torch
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = synth.periodic_system(a=10.26, num=16, nkgrid=2, no=256, supercell=2, seed=3, ecut=2.0,
                              name="periodic_supercell")
    nt, dt = args.supercell_nt, 0.08
    omega = 1.55 / synth.AU_ENERGY_EV
    Ac = synth.asin2cos(nt, dt, omega=omega, f0=omega * 1e-3, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    units = int(np.prod(s.grid.shape)) * s.norb * nt
    peak, peak_kind = measured_peaks()
    out = {"workload": (f"periodic supercell a=20.52 bohr, {s.pp.natom} atoms, {s.grid.shape[0]}^3 grid, {s.nk} "
                        f"k-points, {s.no} complex128 orbitals/k (band-limited, |k+G|^2/2 <= 2 Ha), Asin2cos "
                        f"A(t) peak 1e-3 au, {nt} Taylor-4 steps per sample"),
           "units_per_sample": units, "peak_gbs": peak, "peak_source": peak_kind}
    curr = {}
    for prec in ("fp64", "mixed"):
        ctx = Context(s, device=local, precision=prec)
        stream = torch.cuda.Stream(device=local)
        ctx.set_stream(stream)
        psi0 = ctx.upload(s.psi)
        a, b, w = ctx.empty(), ctx.zeros(), ctx.zeros()
        a.copy_(psi0)
        res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)  # warm-up; J(t) of the comparison
        curr[prec] = np.array(res["curr"])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(2):
            ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
        e1.record(stream)
        torch.cuda.synchronize()
        value = units * 2 / (e0.elapsed_time(e1) / 1e3)
        ctx.set_timing(True)
        ctx.kernel_times(reset=True)
        ctx.rt_propagate(a, b, w, min(nt, 20), dt, zc, Ac_ext=Ac[:, : min(nt, 20) + 2])
        kt = ctx.kernel_times(reset=True)
        ctx.set_timing(False)
        h_ms, h_cnt = kt.get("hpsi", (float("nan"), 1))
        bytes_launch = UNIT_BYTES[prec] / 4.0 * units / nt
        ach = bytes_launch / (h_ms / h_cnt / 1e3) / 1e9
        out[prec] = {"value": value, "kernel": "k_hpsi_tma", "avg_launch_ms": h_ms / h_cnt,
                     "algorithmic_bytes_per_launch": bytes_launch, "achieved_gbs": ach, "frac": ach / peak,
                     "traffic": ncu_traffic("k_hpsi_tma", "supercell") if prec == "fp64" else None}
        ctx.close()
        del a, b, w, psi0
        torch.cuda.empty_cache()
    jmax = float(np.max(np.abs(curr["fp64"])))
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed"]["j_rel_err"] = float(np.max(np.abs(curr["mixed"] - curr["fp64"]))) / jmax
    out["mixed"]["j_rel_err_budget"] = 1e-6
    return out


def ncu_traffic(kernel, workload):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summary profiles/<kernel>_<workload>.md, if present."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("traffic_bytes_per_launch_full_workload:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_baseline(args, s, dt, Ac, zc, nsteps, min_seconds=10.0):
    """The oracle's time loop (all host threads) on the full system, repeated in
    runs of `nsteps` Taylor steps from the same start until `min_seconds` of CPU
    work have been timed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, lib as olib
    threads = os.cpu_count() or 1
    O = Oracle(s, threads=threads)
    Ac_s = None if Ac is None else Ac[:, : nsteps + 2].copy(order="F")
    scf = getattr(args, "self_consistent", False)
    if scf:  # the same per-step potential update as the GPU loop
        import oracle as OR
        brl = np.diag([2.0 * np.pi / (n * h) for n, h in zip(s.grid.shape, s.grid.hgs)])
        vpsl = np.array(s.V_local[..., 0])
        rho0 = O.density(s.psi)[..., 0]
        cg = None
        if s.grid.periodic:
            vh0 = OR.poisson_ft(rho0, brl)
        elif args.poisson == "cg":
            vh0, _ = O.poisson_isolated_cg(rho0)
            cg = dict(vh0=vh0)
        else:
            vh0 = OR.poisson_isolated_ft(rho0, brl)
        v0 = OR.update_vlocal(vpsl, vh0, OR.exc_cor_pz(rho0, s.grid.hvol)[0][..., None])[..., 0]
    el, runs = 0.0, 0
    while el < min_seconds or runs == 0:
        t0 = time.perf_counter()
        if scf:
            O.rt_run_scf(s.psi, nsteps, dt, zc, vpsl, brl, v0, Ac_ext=Ac_s, cg=cg)
        else:
            O.rt_run(s.psi, nsteps, dt, zc, Ac_ext=Ac_s)
        el += time.perf_counter() - t0
        runs += 1
    units = int(np.prod(s.grid.shape)) * s.norb * nsteps * runs
    return {"value": units / el, "unit": UNIT, "cores": int(olib().sbo_get_threads()), "kind": "port",
            "sample": f"{runs} runs of {nsteps} Taylor steps of the full workload ({units} units) in {el:.1f} s",
            "seconds": el}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    s, nt, dt, Ac, zc = workload(args)
    n = max(1, args.cpu_steps)
    vals, secs = [], []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(args, s, dt, Ac, zc, n, min_seconds=5.0)  # each bench step: >= 5 s of CPU work
        if i >= args.warmup:
            vals.append(cb["value"])
            secs.append(cb["seconds"])
    v = float(np.mean(vals))
    cb = {k: cb[k] for k in ("unit", "cores", "kind")}
    cb.update(value=v, sample=f"per bench step, runs of {n} Taylor steps of the full workload "
                              f"repeated for at least 5 s of CPU work")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": float(np.mean(secs)) * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
           "config": config_dict(args, s, n, 1),
           "cpu_baseline": cb,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def batch_workload(args):
    from salmon2_b200 import synth
    systems = synth.uneven_batch(4 if args.small else 16, seed=4)
    psi0 = [synth.impulse_kick(s.grid, s.psi, 1e-3) for s in systems]
    return systems, psi0, 0.05, synth.taylor_zc(0.05)


def batch_config(args, systems, nt):
    units = sum(int(np.prod(s.grid.shape)) * s.norb for s in systems)
    return {
        "workload": (f"{len(systems)} independent isolated systems (seed 4), grids "
                     f"{min(s.grid.shape[0] for s in systems)}^3..{max(s.grid.shape[0] for s in systems)}^3, "
                     f"{min(s.no for s in systems)}..{max(s.no for s in systems)} complex128 orbitals, "
                     f"{min(s.pp.natom for s in systems)}..{max(s.pp.natom for s in systems)} atoms, "
                     f"h=0.25 A, Dirichlet, kick 1e-3 au, dt=0.05 au, {nt} Taylor-4 steps per bench step, "
                     f"dipole every step, one batch (autotuned tiles)"),
        "systems": [[int(s.grid.shape[0]), int(s.no), int(s.pp.natom)] for s in systems],
        "units_per_taylor_step": units, "taylor_steps_per_bench_step": nt, "precision": args.precision,
        "parallelism": "replicas" if int(os.environ.get("WORLD_SIZE", "1")) > 1 else "single GPU",
        "l2": "inputs larger than L2 (%.1f GB per orbital array set)" % (units * 16 / 1e9),
    }


def main_batch(args):
    """Uneven batch: every system advanced by one persistent launch per Taylor
    term (sb200_batch_propagate), against the same systems run one after the
    other through their own sb200_rt_propagate."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        systems, psi0, dt, zc = batch_workload(args)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Oracle, lib as olib
        n = max(1, args.cpu_steps // 2)
        vals = []
        for i in range(args.warmup + args.steps):
            s = systems[i % len(systems)]
            O = Oracle(s, threads=os.cpu_count() or 1)
            t0 = time.perf_counter()
            O.rt_run(psi0[i % len(systems)], n, dt, zc)
            el = time.perf_counter() - t0
            if i >= args.warmup:
                vals.append(int(np.prod(s.grid.shape)) * s.norb * n / el)
        v = float(np.mean(vals))
        cb = {"value": v, "unit": UNIT, "cores": int(olib().sbo_get_threads()), "kind": "port",
              "sample": f"{n} Taylor steps of one system of the batch per bench step (systems in turn)"}
        print(json.dumps({"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                          "impl": "reference", "config": batch_config(args, systems, args.nt),
                          "cpu_baseline": cb,
                          "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    from salmon2_b200.rt import Batch, Context
    systems, psi0, dt, zc = batch_workload(args)
    nt = args.nt
    ctxs = [Context(s, device=local, precision=args.precision) for s in systems]
    stream = torch.cuda.Stream(device=local)
    for c in ctxs:
        c.set_stream(stream)
    A = [c.upload(p) for c, p in zip(ctxs, psi0)]
    B = [c.zeros() for c in ctxs]
    W = [c.zeros() for c in ctxs]
    units = sum(int(np.prod(s.grid.shape)) * s.norb for s in systems) * nt
    batch = Batch(ctxs)
    tiles = batch.autotune(A, W, reps=3)

    def timed(fn, k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def batch_step():
        batch.propagate(A, B, W, nt, dt, zc, rbox=False)

    def solo_step():
        for c, a, b, w in zip(ctxs, A, B, W):
            c.rt_propagate(a, b, w, nt, dt, zc)

    for _ in range(args.warmup):
        batch_step()
    with Clocks(local) as clk:
        ms = timed(batch_step, args.steps)
    value = units * args.steps / (ms / 1e3)
    solo_step()
    ms_solo = timed(solo_step, max(1, args.steps // 2))
    solo_value = units * max(1, args.steps // 2) / (ms_solo / 1e3)

    # e2e through the C ABI with host buffers: upload every system from pinned
    # reference-layout arrays, propagate the batch, read every psi(t) back
    host = [torch.from_numpy(np.ascontiguousarray(p.ravel(order="F").view(np.float64))).pin_memory() for p in psi0]
    back = [torch.empty_like(h).pin_memory() for h in host]
    bytes_io = sum(h.numel() * 8 for h in host)

    def e2e_step():
        for c, h, a in zip(ctxs, host, A):
            c.upload(h, out=a)
        res = batch.propagate(A, B, W, nt, dt, zc)
        for c, p, o in zip(ctxs, res["psi"], back):
            c.download(p, out=o)

    e2e_step()
    ne = max(1, min(args.steps, 3))
    ms_e2e = timed(e2e_step, ne)
    e2e_value = units * ne / (ms_e2e / 1e3)

    # instrumented replay: per-kernel device times through the first context
    ctxs[0].set_timing(True)
    ctxs[0].kernel_times(reset=True)
    nt_i = min(nt, 20)
    batch.propagate(A, B, W, nt_i, dt, zc, rbox=False)
    kt = ctxs[0].kernel_times(reset=True)
    ctxs[0].set_timing(False)
    peak, peak_kind = measured_peaks()
    h_ms, h_cnt = kt.get("hpsi", (float("nan"), 1))
    avg_ms = h_ms / h_cnt
    bytes_per_launch = UNIT_BYTES[args.precision] / 4.0 * units / nt
    achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
    total_ms = sum(v[0] for v in kt.values())
    launches_per_tstep = sum(v[1] for v in kt.values()) / nt_i
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32",
        "data": "synthetic (seeded; shapes of the uneven-batch configuration)",
        "config": batch_config(args, systems, nt),
        "solo_value": solo_value, "batch_over_solo": value / solo_value,
        "tiles": {"shape": tiles[0].tolist(), "zchunk": tiles[1].tolist()},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_io,
                "d2h_bytes_per_step": bytes_io + 4 * nt * 8 * len(systems)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "kernel": "k_hpsi_batch_tma" if all(t == 2 for t in tiles[0]) else "k_hpsi_batch",
                     "avg_launch_ms": avg_ms,
                     "algorithmic_bytes_per_launch": bytes_per_launch},
        "kernel_shares": {k: round(v[0] / total_ms, 4) for k, v in kt.items()},
        "gpu_launches": int(round(launches_per_tstep * nt * args.steps)),
        "clocks": clk.summary(),
        "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    batch.close()
    for c in ctxs:
        c.close()


def main():
    args = parse()
    if args.nt is None:
        args.nt = {"batch": 40, "isolated": 1000}.get(args.workload, 2000)
    if args.workload == "batch":
        return main_batch(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from salmon2_b200.rt import Context

    s, nt, dt, Ac, zc = workload(args, rank, world)
    ctx = Context(s, device=local, precision=args.precision)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    units_rank = int(np.prod(s.grid.shape)) * s.norb * nt
    if world > 1 and args.workload != "isolated":
        # k-point shards: J(t) and the dipole sums of every step (and, self-consistent,
        # the density) are summed over the ranks by an NCCL all-reduce inside the
        # loop's CUDA graph -- the exchange step of the path
        from salmon2_b200.rt import nccl_unique_id
        uid = torch.zeros(128, dtype=torch.uint8, device=f"cuda:{local}")
        if rank == 0:
            uid.copy_(torch.frombuffer(bytearray(nccl_unique_id()), dtype=torch.uint8))
        dist.broadcast(uid, 0)
        ctx.set_density_comm(world, rank, bytes(uid.cpu().numpy().tobytes()))
    if args.self_consistent:
        if s.nspin != 1:
            raise SystemExit("--self-consistent needs a workload with one spin")
        # orthogonal box: primitive_b = 2 pi / L (the Hartree solve is poisson_ft on the
        # periodic cell, poisson_isolated_ft on an isolated box); V_local from rho(t=0),
        # then the update every step
        brl = np.diag([2.0 * np.pi / (n * h) for n, h in zip(s.grid.shape, s.grid.hgs)])
        vpsl = torch.from_numpy(np.ascontiguousarray(s.V_local[..., 0].ravel(order="F"))).cuda(local)

    def set_up():
        """The self-consistent loop's initial potential from the orbitals in a
        (initialization_rt): V_local, the Hartree potential and, with CG, its
        extrapolation history; on the context's stream."""
        if not args.self_consistent:
            return
        with torch.cuda.stream(stream):
            if s.grid.periodic or args.poisson == "ft":
                ctx.update_potential(a, vpsl, brl)
            else:  # method_poisson = 'cg': CG from the extrapolated potential every step
                ctx.update_potential(a, vpsl, brl, poisson="cg")
                ctx.set_hartree_cg(ctx.last_vh)
            ctx.set_self_consistent(True, vpsl, brl)

    # the isolated-molecule workload is the run of nt steps after the kick: every
    # bench step starts again from the kicked orbitals (and, self-consistent, from
    # their potential), so each step times the same stretch of the dynamics
    restart = args.workload == "isolated"
    psi0 = ctx.upload(s.psi) if restart else None

    def restart_from_kick():
        if restart:
            with torch.cuda.stream(stream):
                a.copy_(psi0)
            set_up()

    set_up()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def one_step():
        restart_from_kick()
        return ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)

    for _ in range(args.warmup):
        one_step()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            res = one_step()
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    t = torch.tensor([ms], device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = units_rank * world * args.steps / (ms_max / 1e3)

    # e2e: host (pinned, reference layout) -> device -> propagate -> host.  The
    # isolated workload uploads the kicked orbitals every step (and sets up
    # their potential) as the device-resident loop above does; the periodic ones
    # carry the propagation on through host memory: each step uploads what the
    # previous one read back
    host_state = torch.from_numpy(np.ascontiguousarray(s.psi.ravel(order="F").view(np.float64))).pin_memory()
    host_out = torch.empty_like(host_state).pin_memory() if restart else host_state
    if not restart and args.steps > 0:
        ctx.download(res["psi"], out=host_state)
    bytes_io = host_state.numel() * 8

    def e2e_step():
        ctx.upload(host_state, out=a)
        if restart:
            set_up()
        res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
        ctx.download(res["psi"], out=host_out)
        return res

    e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ne2e = max(1, min(args.steps, 3))
    e0.record(stream)
    for _ in range(ne2e):
        e2e_step()
    e1.record(stream)
    barrier()
    te = torch.tensor([e0.elapsed_time(e1)], device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = units_rank * world * ne2e / (float(te.item()) / 1e3)

    # instrumented replay for per-kernel device times (roofline + shares)
    restart_from_kick()
    torch.cuda.synchronize()
    ctx.set_timing(True)
    ctx.kernel_times(reset=True)
    nt_i = min(nt, 200)
    ctx.rt_propagate(a, b, w, nt_i, dt, zc, Ac_ext=None if Ac is None else Ac[:, : nt_i + 2])
    kt = ctx.kernel_times(reset=True)
    ctx.set_timing(False)
    launches_per_tstep = sum(v[1] for v in kt.values()) / nt_i
    gpu_launches = int(round(launches_per_tstep * nt * args.steps))
    units_per_launch = int(np.prod(s.grid.shape)) * s.norb
    kname, bytes_per_launch = hpsi_kernel(s, args, units_per_launch)
    peak, peak_kind = measured_peaks()
    h_ms, h_cnt = kt.get("hpsi", (float("nan"), 1))
    avg_ms = h_ms / h_cnt
    achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
    traffic = ncu_traffic(kname, args.workload)
    total_ms = sum(v[0] for v in kt.values())
    shares = {k: round(v[0] / total_ms, 4) for k, v in kt.items()}

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args, s, dt, Ac, zc, max(1, args.cpu_steps))
            cpu.pop("seconds", None)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32",
            "data": ("synthetic (seeded; shapes of the isolated-molecule configuration)" if args.workload == "isolated"
                 else f"synthetic (seeded; shapes of the periodic-{args.workload} configuration)"),
            "config": config_dict(args, s, nt, world),
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": bytes_io + (0 if Ac is None else Ac.nbytes),
                    "d2h_bytes_per_step": bytes_io + 3 * nt * 8 + 4 * nt * 8},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "traffic_source": (f"profiles/{kname}_{args.workload}.md: DRAM bytes of one launch "
                                            "from an ncu capture of this workload, not measured in this run"
                                            if traffic is not None else None),
                         "kernel": kname, "avg_launch_ms": avg_ms,
                         "algorithmic_bytes_per_launch": bytes_per_launch},
            "kernel_shares": shares,
            "gpu_launches": gpu_launches,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        if world == 1 and args.workload == "bulk" and args.precision == "fp64" and not args.self_consistent \
                and not args.no_supercell:
            ctx.close()
            out["supercell"] = supercell_leg(args, local)
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
