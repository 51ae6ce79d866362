#!/usr/bin/env python
"""Benchmark: relaxed systems per second on one B200 (per rank), JSON line on stdout.

Workload (default): 4096 replicas of the 40-atom polyaromatic (random lateral
offset, z rotation, height U[2.5, 4] A, 0.05 A jitter) over a 2-layer 4x4-cell
NaCl(100) slab, FP32 B-spline grid 226x226x121 (0.1 A) built on the device;
FIRE (dt0 0.001, dt_max 0.05) to max|F| < 1e-3 eV/A or 2000 steps.

One bench step = relaxing the whole batch from its start positions.  The device
time of each step is taken with CUDA events on the library's stream around the
relaxation launch; L2 is flushed (256 MB write) before every step.  Under
torchrun each rank relaxes its own batch (weak scaling, no collective on the
data path); the reported time is the max over ranks.

--impl reference times the FP64 CPU restatement of the same path (oracle/), the
reference's own algorithm, on all host cores, on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "relaxed systems/sec at ≤1e-4 eV/Å force error; p50/p99 relax latency; HBM GB/s"
FIRE = dict(dt0=0.001, dt_max=0.05, fconv=1e-3)
MAX_STEPS = 2000
SEED = 20261203
# FIRE steps [0, 1000) in the rounds form (a warp per system: throughput), then the gather form
# with 64 and from step 1400 128 threads per system (latency of the slow tail)
STAGES = "0:rounds:0,1000:gather:64,1400:gather:128"
FORMS = {"rounds": 0, "gather": 1, "owner": 2}


def parse_stages(txt):
    """'start:form:team,...' -> (starts, forms, teams)"""
    st, fm, tm = [], [], []
    for part in txt.split(","):
        a, f, t = part.split(":")
        st.append(int(a))
        fm.append(FORMS[f])
        tm.append(int(t))
    return st, fm, tm


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier_max(ws, value):
    """Max over ranks of a float (device time); the all-reduce is also the barrier."""
    if ws == 1:
        return value
    from surfmol_b200.shard import max_over_ranks
    return max_over_ranks(value)


def make_workload(seed, nsys):
    from surfmol_b200 import synth
    return synth.config1(seed, nsys)


def workload_desc(w, nsys, substrate="grid"):
    g = w.grid
    if substrate == "folded":
        return (f"config1 on the folded surface: {nsys} replicas of a 40-atom polyaromatic (24 C, 12 H, 2 N, 2 O) "
                f"over the NaCl-like SurfaceFolded basis (2x2 harmonics x 3 z decays, a=5.66 A, plane at the slab top), "
                f"forces clamped at 100 eV/A; FIRE to max|F|<1e-3 or {MAX_STEPS} steps")
    return (f"config1: {nsys} replicas of a 40-atom polyaromatic (24 C, 12 H, 2 N, 2 O) over NaCl(100) "
            f"2 layers 4x4 cells, fp32 B-spline grid {g.nx}x{g.ny}x{g.nz} at 0.1 A; FIRE to max|F|<1e-3 or {MAX_STEPS} steps")


def folded_surface(slab):
    """The NaCl-like folded surface of the reference's editor, its plane at the slab's top layer."""
    from surfmol_b200.folded import nacl
    return nacl(z0=slab.z_top)


# ---------------------------------------------------------------------------------------- reference arm
def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    from oracle import oracle as O
    w = make_workload(SEED, args.nsys)
    slab, g = w.slab, w.grid
    t0 = time.perf_counter()
    if args.substrate == "folded":
        grid = O.Folded(**folded_surface(slab).as_dict())
    else:
        coef = O.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step)
        grid = O.Grid(coef.astype(np.float32), g.p0, g.step)
    tgrid = time.perf_counter() - t0
    sys0 = O.System.from_molecule(w.Z[0], w.pos[0], w.q[0])
    threads = os.cpu_count() or 1
    sample = max(threads, args.ref_sample)

    def one(k0):
        idx = [(k0 + i) % args.nsys for i in range(sample)]
        t = time.perf_counter()
        r = O.relax_batch([sys0] * sample, [w.pos[i] for i in idx], grid, max_steps=MAX_STEPS, nthreads=threads,
                          **FIRE)
        return time.perf_counter() - t, r

    for k in range(args.warmup):
        one(k * sample)
    tt, conv, steps = 0.0, 0, []
    for k in range(args.steps):
        dt, r = one((args.warmup + k) * sample)
        tt += dt
        conv += int(r["conv"].sum())
        steps += list(r["steps"])
    v = sample * args.steps / tt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "systems/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_desc(w, args.nsys, args.substrate), "sample_per_step": sample,
                       "grid_build_s": round(tgrid, 2), "converged_fraction": conv / (sample * args.steps),
                       "fire_steps_p50": float(np.percentile(steps, 50)), "fire_steps_p99": float(np.percentile(steps, 99))},
            "cpu_baseline": {"value": v, "unit": "systems/s", "cores": threads, "kind": "port",
                             "sample": f"{sample} systems of the workload per step, FP64 oracle (oracle/oracle.cpp), "
                                       f"OpenMP one system per thread"},
            "e2e": {"value": v, "unit": "systems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------- our arm
def cpu_baseline(w, grid, budget_s=15.0):
    """grid: the oracle's substrate (oracle.Grid or oracle.Folded)."""
    from oracle import oracle as O
    sys0 = O.System.from_molecule(w.Z[0], w.pos[0], w.q[0])
    threads = os.cpu_count() or 1
    chunk = max(threads, 16)
    done, t_total, k = 0, 0.0, 0
    while t_total < budget_s and done < len(w.pos):
        idx = [(k + i) % len(w.pos) for i in range(chunk)]
        t = time.perf_counter()
        O.relax_batch([sys0] * chunk, [w.pos[i] for i in idx], grid, max_steps=MAX_STEPS, nthreads=threads, **FIRE)
        t_total += time.perf_counter() - t
        done += chunk
        k += chunk
    return {"value": done / t_total, "unit": "systems/s", "cores": threads, "kind": "port",
            "sample": f"{done} systems of the same workload (relaxed to convergence or {MAX_STEPS} steps), FP64 oracle, "
                      f"OpenMP one system per thread, {t_total:.1f} s"}


def run_ours(args, ws, rank, local):
    import torch
    from surfmol_b200 import RelaxMulti

    dev = local
    torch.cuda.set_device(dev)
    w = make_workload(SEED + 7919 * rank, args.nsys)
    slab, g = w.slab, w.grid
    natoms = sum(len(p) for p in w.pos)
    R = RelaxMulti(max_systems=args.nsys, max_atoms=natoms, device=dev)
    R.set_nb(rdamp=1.0, alpha_morse=1.5)
    t0 = time.perf_counter()
    if args.substrate == "folded":
        R.set_surface_folded(folded_surface(slab))
    elif ws > 1:
        # each rank evaluates an x-slab, one all-gather over NVLink, each rank fits the whole grid
        from surfmol_b200.shard import build_grid_sharded
        build_grid_sharded(R, slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step,
                           alpha_morse=1.5, npbc=1)
    else:
        R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step, alpha_morse=1.5, npbc=1)
    torch.cuda.synchronize()
    tgrid = time.perf_counter() - t0
    tid = R.add_molecule(w.Z[0], w.pos[0], w.q[0])
    slots = R.add_systems([tid] * args.nsys, w.pos)
    R.set_stages(*parse_stages(args.stages))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2

    def reset():
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)

    def step():
        reset()
        flush.zero_()
        torch.cuda.synchronize()
        R.run_fire(args.max_steps, step_budget=args.max_steps, **FIRE)
        ms, launches = R.last_timing()
        return ms, launches

    for _ in range(args.warmup):
        step()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    dev_ms, launches, atom_steps, steps_all, conv = 0.0, 0, 0, [], 0
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            ms, nl = step()
            dev_ms += ms
            launches += nl
            out = R.download(slots, pos=False, forces=False)
            atom_steps += int(out["steps"].sum()) * 40
            steps_all += list(out["steps"])
            conv += int((out["status"] == 1).sum())
        torch.cuda.synchronize()
    dev_ms = barrier_max(ws, dev_ms)
    clocks = clk.summary()
    ms_step = dev_ms / args.steps
    value = ws * args.nsys / (ms_step * 1e-3)

    if args.profile:
        R.finish()
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms_step, "atom_steps": atom_steps, "launches": launches}))
        return 0
    # end to end through the public API with host buffers: H2D positions, relax, D2H positions + results
    e2e_k = max(1, min(args.steps, 3))
    pos_host = np.stack(w.pos).astype(np.float32)          # the inputs, in host memory, before timing
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_k):
        R.set_positions(slots, pos_host)
        R.reset_fire(slots)
        R.run_fire(MAX_STEPS, step_budget=MAX_STEPS, **FIRE)
        res = R.download(slots, pos=True, forces=False)
    torch.cuda.synchronize()
    t_e2e = barrier_max(ws, time.perf_counter() - t0)
    slot_bytes = 64 * args.nsys
    e2e = {"value": ws * args.nsys * e2e_k / t_e2e, "unit": "systems/s",
           "h2d_bytes_per_step": 16 * natoms + slot_bytes + 12 * args.nsys,
           "d2h_bytes_per_step": 16 * natoms + 2 * slot_bytes}

    # the plain form on a sample: each system alone on a one-slot handle, one kernel launch per FIRE step
    plain_n = 8
    R1 = RelaxMulti(max_systems=1, max_atoms=64, device=dev)
    R1.set_nb(rdamp=1.0, alpha_morse=1.5)
    if args.substrate == "folded":
        R1.set_surface_folded(folded_surface(slab))
    else:
        gd = R.get_grid()
        R1.set_grid(gd["coef"], gd["p0"], gd["step"])
    tid1 = R1.add_molecule(w.Z[0], w.pos[0], w.q[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(plain_n):
        s1 = R1.add_systems([tid1], [w.pos[k]])
        R1.run_fire(MAX_STEPS, step_budget=MAX_STEPS, mode=1, **FIRE)
        R1.remove_systems(s1)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    plain_sps = plain_n / t_plain
    R1.finish()
    hbm, peak_kind = peaks()
    algo_bytes = 1024.0 * atom_steps / args.steps          # 64 fp32 float4 voxels per atom-step
    achieved = algo_bytes / (ms_step * 1e-3) / 1e9
    # DRAM bytes per atom-step of the relax kernel from one ncu capture (profiles/), scaled to the
    # atom-steps of one timed step: the grid stays L2-resident, so DRAM traffic grows with the work
    traffic = None
    prof = os.path.join(ROOT, "profiles", "relax_config1_traffic.json")
    if os.path.exists(prof):
        pj = json.load(open(prof))
        if "dram_bytes_per_atom_step" in pj:
            traffic = pj["dram_bytes_per_atom_step"] * atom_steps / args.steps
    line = {"metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_desc(w, args.nsys, args.substrate), "nsys_per_gpu": args.nsys, "atoms_per_system": 40,
                       "parallelism": f"systems sharded over {ws} GPU(s), no collective in the step"
                                      + ("; grid built in x-slabs, one all-gather" if ws > 1 and args.substrate == "grid" else ""),
                       "l2": "flushed (256 MB write) before every timed step", "grid_build_s": round(tgrid, 3),
                       "converged_fraction": conv / (args.nsys * args.steps),
                       "fire_steps_p50": float(np.percentile(steps_all, 50)),
                       "fire_steps_p99": float(np.percentile(steps_all, 99)),
                       "mode": "batched persistent kernel, one launch per schedule stage", "stages": args.stages,
                       "plain_systems_per_s": plain_sps, "batched_over_plain": value / plain_sps,
                       "plain": f"{plain_n} systems, each alone, one kernel launch per FIRE step (wall clock)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes": "1024 B per atom-step (64 float4 grid voxels), state resident in shared memory"},
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks}
    if args.substrate == "folded":
        # no grid stream: the basis (12 float4 coefficients) stays in L1; the kernel is bound by
        # its FP32 / SFU issue rate, which the ncu summary of this workload shows
        line["roofline"] = None
        line["roofline_note"] = "folded surface: no HBM stream to bound the kernel (basis in L1); issue-bound"
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if args.substrate == "folded":
            og = O.Folded(**folded_surface(slab).as_dict())
        else:
            gd = R.get_grid()
            og = O.Grid(gd["coef"], gd["p0"], gd["step"])
        line["cpu_baseline"] = cpu_baseline(w, og, budget_s=args.cpu_budget)
    R.finish()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------------------- ragged workload
RAGGED = dict(nsys=16384, nmin=20, nmax=400, rcut=10.0, fconv=1e-4, max_steps=3000, tune_sample=4096)


def ragged_desc(w, nsys):
    g = w.grid
    return (f"ragged: {nsys} distinct planar C/H/N/O molecules, atoms log-uniform in [{RAGGED['nmin']}, {RAGGED['nmax']}], "
            f"over NaCl(100) 3 layers 8x8 cells, fp32 B-spline grid {g.nx}x{g.ny}x{g.nz} at 0.1 A; intramolecular "
            f"cutoff {RAGGED['rcut']} A; FIRE to max|F|<{RAGGED['fconv']} or {RAGGED['max_steps']} steps")


def ragged_workload(seed, nsys):
    from surfmol_b200 import synth
    return synth.ragged(seed, nsys, RAGGED["nmin"], RAGGED["nmax"], ncell=8, nlayers=3, nz=161,
                        workers=min(32, os.cpu_count() or 1))


def run_reference_ragged(args, ws, rank):
    if rank != 0:
        return 0
    from oracle import oracle as O
    nsys = args.nsys or RAGGED["nsys"]
    w = ragged_workload(SEED, nsys)
    slab, g = w.slab, w.grid
    coef = O.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step)
    grid = O.Grid(coef.astype(np.float32), g.p0, g.step)
    threads = os.cpu_count() or 1
    sample = max(threads, args.ref_sample)
    nb = dict(rdamp=1.0, alpha=1.5, rcut=RAGGED["rcut"])
    fire = dict(FIRE, fconv=RAGGED["fconv"])

    def one(k0):
        idx = [(k0 + i) % nsys for i in range(sample)]
        systems = [O.System.from_molecule(w.Z[i], w.pos[i], w.q[i]) for i in idx]
        t = time.perf_counter()
        r = O.relax_batch(systems, [w.pos[i] for i in idx], grid, max_steps=RAGGED["max_steps"], nthreads=threads, nb=nb, **fire)
        return time.perf_counter() - t, r, sum(len(w.Z[i]) for i in idx)

    for k in range(args.warmup):
        one(k * sample)
    tt, conv = 0.0, 0
    for k in range(args.steps):
        dt, r, _ = one((args.warmup + k) * sample)
        tt += dt
        conv += int(r["conv"].sum())
    v = sample * args.steps / tt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "systems/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": ragged_desc(w, nsys), "sample_per_step": sample, "converged_fraction": conv / (sample * args.steps)},
            "cpu_baseline": {"value": v, "unit": "systems/s", "cores": threads, "kind": "port",
                             "sample": f"{sample} molecules of the workload per step, FP64 oracle, OpenMP one system per thread"},
            "e2e": {"value": v, "unit": "systems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ragged(args, ws, rank, local):
    nsys = args.nsys or RAGGED["nsys"]
    t0 = time.perf_counter()
    w = ragged_workload(SEED + 7919 * rank, nsys)          # generated before any CUDA work (spawned pool)
    tgen = time.perf_counter() - t0
    import torch
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.autotune import Autotuner, TuneResult
    torch.cuda.set_device(local)
    slab, g = w.slab, w.grid
    natoms = np.array([len(z) for z in w.Z])
    fire = dict(FIRE, fconv=RAGGED["fconv"])
    max_steps = args.max_steps if args.max_steps != MAX_STEPS else RAGGED["max_steps"]

    def make_handle(ms, ma):
        R = RelaxMulti(max_systems=ms, max_atoms=ma, device=local)
        R.set_nb(rdamp=1.0, alpha_morse=1.5, rcut=RAGGED["rcut"])
        R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step, alpha_morse=1.5, npbc=1)
        return R

    t0 = time.perf_counter()
    if args.no_tune:
        tune = None
    else:
        rng = np.random.default_rng(SEED)
        pick = np.sort(rng.choice(nsys, size=min(nsys, RAGGED["tune_sample"]), replace=False))
        # the probes hold as many systems as the real run (copies of the sample, moved laterally):
        # with fewer, one wave fits on the GPU and latency-oriented shapes win the probe but not the run
        tune = Autotuner(make_handle, fire, probe_steps=100, max_steps=max_steps, max_probe_systems=nsys).tune(
            [w.Z[i] for i in pick], [w.pos[i] for i in pick], [w.q[i] for i in pick], full_count=nsys)
    ttune = time.perf_counter() - t0
    R = make_handle(nsys, int(natoms.sum()))
    if tune is not None:
        tune.apply(R)
    t0 = time.perf_counter()
    tids = R.add_molecules(w.Z, w.pos, w.q)
    tadd = time.perf_counter() - t0
    slots = R.add_systems(tids, w.pos)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step():
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)
        flush.zero_()
        torch.cuda.synchronize()
        R.run_fire(max_steps, step_budget=max_steps, **fire)
        return R.last_timing()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    dev_ms, launches, atom_steps, conv, steps_all = 0.0, 0, 0, 0, []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ms, nl = step()
            dev_ms += ms
            launches += nl
            out = R.download(slots, pos=False, forces=False)
            atom_steps += int((out["steps"] * natoms).sum())
            conv += int((out["status"] == 1).sum())
            steps_all += list(out["steps"])
        torch.cuda.synchronize()
    dev_ms = barrier_max(ws, dev_ms)
    ms_step = dev_ms / args.steps
    value = ws * nsys / (ms_step * 1e-3)
    e2e_k = max(1, min(args.steps, 2))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_k):
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)
        R.run_fire(max_steps, step_budget=max_steps, **fire)
        R.download(slots, pos=True, forces=False)
    t_e2e = barrier_max(ws, time.perf_counter() - t0)
    hbm, peak_kind = peaks()
    achieved = 1024.0 * atom_steps / args.steps / (ms_step * 1e-3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": ragged_desc(w, nsys), "nsys_per_gpu": nsys, "atoms_total": int(natoms.sum()),
                       "atoms_mean": float(natoms.mean()), "parallelism": f"systems sharded over {ws} GPU(s), no collective",
                       "l2": "flushed (256 MB write) before every timed step", "converged_fraction": conv / (nsys * args.steps),
                       "fire_steps_p50": float(np.percentile(steps_all, 50)), "fire_steps_p99": float(np.percentile(steps_all, 99)),
                       "host_s": {"generate": round(tgen, 2), "autotune": round(ttune, 2), "add_molecules": round(tadd, 2)},
                       "tuned": None if tune is None else {"team_by_class": tune.team_by_class, "form0": tune.form0,
                                                            "nb_lanes": tune.nb_lanes, "stages": tune.stages,
                                                            "sample_relax_ms": {k: round(tune.timings[k], 1) for k in
                                                                                ("relax_ms_tuned_shape", "relax_ms_default_shape",
                                                                                 "relax_ms_tuned") if k in tune.timings}}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None, "peak_source": peak_kind,
                         "algorithmic_bytes": "1024 B per atom-step (64 float4 grid voxels), state resident in shared memory"},
            "e2e": {"value": ws * nsys * e2e_k / t_e2e, "unit": "systems/s", "h2d_bytes_per_step": int(16 * natoms.sum() + 76 * nsys),
                    "d2h_bytes_per_step": int(16 * natoms.sum() + 128 * nsys)},
            "gpu_launches": launches, "clocks": clk.summary()}
    R.finish()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------- served workload
SERVE = dict(nmin=20, nmax=2000, rcut=10.0, fconv=1e-4, max_steps=3000, chunk=200, budget_gb=150.0,
             rates=(200.0, 2000.0, 10000.0, 50000.0), per_rate=1500, max_systems=2048, plain_sample=8, resident=0)


def run_serve(args, local):
    from surfmol_b200 import synth
    slab, g = synth.config3_slab_grid()
    per = args.nsys or SERVE["per_rate"]
    workers = min(32, os.cpu_count() or 1)
    # every request stream generated up front in a spawned pool, before any CUDA work
    streams = {"warm": synth.serve_requests(SEED + 1, 64, 1e5, slab, SERVE["nmin"], SERVE["nmax"], workers),
               "plain": synth.serve_requests(SEED + 999, SERVE["plain_sample"], 1e5, slab, SERVE["nmin"], SERVE["nmax"])}
    for k, rate in enumerate(SERVE["rates"]):
        streams[k] = synth.serve_requests(SEED + 100 + k, per, rate, slab, SERVE["nmin"], SERVE["nmax"], workers)
    import torch
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.relax import GRID_F16
    from surfmol_b200.serve import Request, Server
    torch.cuda.set_device(local)
    fire = dict(FIRE, fconv=SERVE["fconv"])
    max_atoms = SERVE["max_systems"] * 1200
    R = RelaxMulti(max_systems=SERVE["max_systems"], max_atoms=max_atoms, device=local)
    R.set_nb(rdamp=1.0, alpha_morse=1.5, rcut=SERVE["rcut"])
    t0 = time.perf_counter()
    R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step, alpha_morse=1.5,
                 npbc=1, dtype=GRID_F16)
    tgrid = time.perf_counter() - t0
    resident = args.resident or SERVE["resident"] or SERVE["max_systems"]
    srv = Server(R, resident, max_atoms, SERVE["budget_gb"] * 1e9, chunk_steps=SERVE["chunk"],
                 max_steps=SERVE["max_steps"], fire=fire, typers=min(16, os.cpu_count() or 1))

    def reqs(key):
        return [Request(i, Z, P, q, t) for i, (Z, P, q, t) in enumerate(streams[key])]
    srv.run(reqs("warm"))                                  # warm-up: loads every kernel shape
    points = []
    for k, rate in enumerate(SERVE["rates"]):
        rq = reqs(k)
        st = srv.run(rq)
        d = st.summary()
        d.update(rate_req_s=rate, atoms_mean=float(np.mean([len(r.Z) for r in rq])),
                 converged_fraction=float(np.mean([r.status == 1 for r in rq])))
        points.append(d)
        print(json.dumps({"serve_point": d}), file=sys.stderr, flush=True)
    # the plain form: each request alone, one kernel launch per FIRE step
    rq = reqs("plain")
    tp = time.perf_counter()
    for r in rq:
        s = R.add_systems([R.add_molecule(r.Z, r.pos, r.q)], [r.pos])
        R.run_fire(SERVE["max_steps"], step_budget=SERVE["max_steps"], mode=1, **fire)
        R.remove_systems(s)
    tp = time.perf_counter() - tp
    plain = {"requests": len(rq), "wall_s": tp, "throughput_req_s": len(rq) / tp,
             "atoms_mean": float(np.mean([len(r.Z) for r in rq]))}
    best = max(p["throughput_req_s"] for p in points)
    line = {"metric": METRIC, "value": best, "unit": "requests/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32 (fp16 grid)", "data": "synthetic",
            "config": {"workload": f"served: Poisson arrivals at {list(SERVE['rates'])} req/s, {per} requests per rate, "
                                   f"molecules log-uniform {SERVE['nmin']}-{SERVE['nmax']} atoms, fp16 grid "
                                   f"{g.nx}x{g.ny}x{g.nz} of a 3-layer 16x16-cell NaCl(100) slab, intramolecular cutoff "
                                   f"{SERVE['rcut']} A, FIRE to {SERVE['fconv']} or {SERVE['max_steps']} steps, "
                                   f"chunks of {SERVE['chunk']} steps, HBM budget {SERVE['budget_gb']} GB",
                       "grid_build_s": round(tgrid, 2), "resident_cap": resident},
            "serve": points, "plain": plain, "served_over_plain": best / plain["throughput_req_s"]}
    R.finish()
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------- grid precision
PREC = dict(nsys=8192, nmin=20, nmax=400, rcut=10.0, fconv=1e-4, max_steps=3000, sample=256)


def run_precision(args, local):
    """Config-3 grid (3-layer 16x16-cell slab, 904x904x160) stored as FP32, FP16 and BF16 with
    per-channel scales: relax the same molecules on each and report the force / energy error
    against the FP64 oracle (evaluated on the FP32 coefficients) at the same positions."""
    from surfmol_b200 import synth
    slab, g = synth.config3_slab_grid()
    nsys = args.nsys or PREC["nsys"]
    w = synth.ragged(SEED + 3, nsys, PREC["nmin"], PREC["nmax"], ncell=16, nlayers=3, nz=160,
                     workers=min(32, os.cpu_count() or 1))
    import torch
    from oracle import oracle as O
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.relax import GRID_BF16, GRID_F16, GRID_F32
    torch.cuda.set_device(local)
    natoms = np.array([len(z) for z in w.Z])
    fire = dict(FIRE, fconv=PREC["fconv"])
    R = RelaxMulti(max_systems=nsys, max_atoms=int(natoms.sum()), device=local)
    R.set_nb(rdamp=1.0, alpha_morse=1.5, rcut=PREC["rcut"])
    t0 = time.perf_counter()
    R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step, alpha_morse=1.5, npbc=1)
    tgrid = time.perf_counter() - t0
    gd = R.get_grid()
    og = O.Grid(gd["coef"], gd["p0"], gd["step"])
    tids = R.add_molecules(w.Z, w.pos, w.q)
    slots = R.add_systems(tids, w.pos)
    pick = np.linspace(0, nsys - 1, min(nsys, PREC["sample"])).astype(int)
    osys = {int(i): O.System.from_molecule(w.Z[i], w.pos[i], w.q[i]) for i in pick}
    nb = dict(rdamp=1.0, alpha=1.5, rcut=PREC["rcut"])
    relaxed = None
    variants = {}
    for name, dt in (("f32", GRID_F32), ("f16", GRID_F16), ("bf16", GRID_BF16)):
        R.set_grid(gd["coef"], gd["p0"], gd["step"])          # from the FP32 coefficients each time
        if dt != GRID_F32:
            R.convert_grid(dt)
        scale = R.get_grid()["scale"] if dt != GRID_F32 else np.ones(4)
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)
        R.run_fire(PREC["max_steps"], step_budget=PREC["max_steps"], **fire)
        ms = R.last_timing()[0]
        st = R.download(slots, pos=False, forces=False)
        if relaxed is None:
            relaxed = R.download_pos64([slots[i] for i in pick])
        errs = {}
        for label, P in (("start", [w.pos[i].astype(np.float32).astype(np.float64) for i in pick]), ("relaxed", relaxed)):
            sel = [slots[i] for i in pick]
            R.set_positions(sel, [p.astype(np.float32) for p in P])
            F, E = R.eval_forces(sel)
            fa, fr, er = [], [], []
            for k, i in enumerate(pick):
                P32 = P[k].astype(np.float32).astype(np.float64)
                Fo, _, Eo = osys[int(i)].eval(P32, og, **nb)
                d = np.abs(F[k][:, :3].astype(np.float64) - Fo).max()
                fa.append(d)
                fr.append(d / max(1.0, np.abs(Fo).max()))
                er.append(abs(E[k, 0] - Eo[0]) / max(1.0, np.abs(Eo[1:7]).sum()))
            errs[label] = {"force_abs_max": float(np.max(fa)), "force_abs_p99": float(np.percentile(fa, 99)),
                           "force_rel_max": float(np.max(fr)), "energy_rel_max": float(np.max(er))}
        variants[name] = {"grid_bytes": int(g.nx * g.ny * g.nz * (16 if dt == GRID_F32 else 8)),
                          "channel_scales": [float(x) for x in scale], "relax_ms": ms, "systems_per_s": nsys / (ms * 1e-3),
                          "converged_fraction": float((st["status"] == 1).mean()),
                          "fire_steps_p50": float(np.median(st["steps"])), "error_vs_fp64_oracle": errs}
        print(json.dumps({name: variants[name]}), file=sys.stderr, flush=True)
    line = {"metric": "FP64-oracle force / energy error per grid storage type", "n_gpus": 1, "data": "synthetic",
            "config": {"workload": f"{nsys} molecules log-uniform {PREC['nmin']}-{PREC['nmax']} atoms over a 3-layer "
                                   f"16x16-cell NaCl(100) slab, grid {g.nx}x{g.ny}x{g.nz}; errors on {len(pick)} systems "
                                   f"at their start and FP32-relaxed positions; FIRE to {PREC['fconv']} or {PREC['max_steps']}",
                       "grid_build_s": round(tgrid, 2), "atoms_total": int(natoms.sum())},
            "variants": variants}
    R.finish()
    print(json.dumps(line), flush=True)
    return 0


def run_ragged_dist(args):
    # the workload is generated in a spawned pool before CUDA and before the process group exists
    ws, rank, local = int(os.environ["WORLD_SIZE"]), int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    import datetime
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    r = run_ragged(args, ws, rank, local)
    dist.barrier()
    dist.destroy_process_group()
    return r


# ---------------------------------------------------------------------------------------- RAFF multi-replica
RAFF = dict(nsys=5000, k=200.0, dt=0.1, relaxation=0.5, beta=0.0, amp=0.2, amp_h=0.3, steps_per_call=10000)
RAFF_METRIC = "RAFF multi-replica real atom-steps/s"


def raff_workload(seed, nsys):
    """The reference's raff_ocl_benchmark configuration: nsys replicas of a 22-atom xylitol-like
    pentitol, ports of stiffness 200 along the rest bonds, each replica perturbed uniformly by
    +-0.2 A (+-0.3 A on H), no collisions, no momentum."""
    from surfmol_b200 import synth
    from surfmol_b200.raff import prepare
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds, k_stiff=RAFF["k"])
    rng = np.random.default_rng(seed)
    amp = np.where(prep.Z == 1, RAFF["amp_h"], RAFF["amp"])[None, :, None]
    P = (prep.pos[None].astype(np.float64) + amp * rng.uniform(-1, 1, (nsys, prep.natoms, 3))).astype(np.float32)
    return prep, P


def raff_cpu(prep, P, nsteps, budget_s):
    """The FP64 oracle step (opencl/RRsp3.cl restated, OpenMP over replicas on all host cores) on blocks of
    replicas until budget_s: atom-steps/s and the replicas done."""
    from oracle import oracle as O
    n = prep.natoms
    blk = 4 * (os.cpu_count() or 1)
    topo = dict(radius=np.zeros(n), neighs=prep.neighs, excl1=prep.excl1, excl2=prep.excl2, fixmask=np.zeros(n, int),
                port_local=prep.port_local[:prep.nnode], k=prep.k[:prep.nnode], bk=prep.bk_slots)
    done, t = 0, 0.0
    while done == 0 or (t < budget_s and done < len(P)):        # at least one block
        m = min(blk, len(P) - done)
        pos4 = np.zeros((m, n, 4)); pos4[..., :3] = P[done:done + m]; pos4[..., 3] = prep.inv_mass
        quat = np.zeros((m, n, 4)); quat[..., 3] = 1
        t0 = time.perf_counter()
        O.raff_step(pos4, quat, n, prep.nnode, nsteps, topo, dt=RAFF["dt"], relaxation=RAFF["relaxation"])
        t += time.perf_counter() - t0
        done += m
    return done * n * nsteps / t, done


def run_raff(args, impl):
    prep, P = raff_workload(SEED, args.nsys)
    n, nsteps = prep.natoms, RAFF["steps_per_call"]
    desc = (f"raff: {args.nsys} replicas of a 22-atom xylitol-like pentitol (C5H12O5, 10 nodes), ports K=200, "
            f"dt 0.1, relaxation 0.5, no momentum, no collisions, perturbation 0.2 A (H 0.3 A); "
            f"{nsteps} RAFF steps per bench step")
    if impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        for _ in range(args.warmup):
            raff_cpu(prep, P[:8], nsteps, 0.0)
        vals = [raff_cpu(prep, P, nsteps, args.cpu_budget / max(1, args.steps))[0] for _ in range(args.steps)]
        v = float(np.mean(vals))
        line = {"impl": "reference", "metric": RAFF_METRIC, "value": v, "unit": "atom-steps/s", "n_gpus": 1,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.nsys * n * nsteps / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": desc},
                "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": os.cpu_count() or 1, "kind": "port",
                                 "sample": "blocks of replicas of the workload, FP64 oracle step (oracle/oracle.cpp), OpenMP over replicas"},
                "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    import torch
    from surfmol_b200.raff import RaffMulti
    torch.cuda.set_device(0)
    R = RaffMulti(n, args.nsys)
    R.upload_prepared(prep, P)
    cfg = dict(dt=RAFF["dt"], relaxation=RAFF["relaxation"], momentum_beta=RAFF["beta"])
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step():
        R.upload_state_multi(P, prep.inv_mass)          # every bench step relaxes the same perturbed replicas
        flush.zero_()
        torch.cuda.synchronize()
        R.step_cluster_multi(nsteps, **cfg)
        return R.last_ms()

    for _ in range(args.warmup):
        step()
    ms = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            ms.append(step())
    ms_step = float(np.mean(ms))
    value = args.nsys * n * nsteps / (ms_step * 1e-3)
    # end to end: positions H2D, the steps, positions D2H, through the public API
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 3))):
        R.upload_state_multi(P, prep.inv_mass)
        R.step_cluster_multi(nsteps, **cfg)
        out = R.download_pos_multi()
    t_e2e = (time.perf_counter() - t0) / max(1, min(args.steps, 3))
    # residual after the timed calls, per replica 0 (the reference's convergence probe)
    res = float(np.abs(R.download_dpos_node_replica(0)).max())
    line = {"metric": RAFF_METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "nsys": args.nsys, "atoms_per_replica": n,
                       "l2": "flushed (256 MB write) before every timed step",
                       "last_step_max_dpos_node": res, "finite": bool(np.isfinite(out).all())},
            "roofline": None,
            "roofline_note": "state stays on chip for all steps of a call (48 B/atom in, 48 B/atom out); issue-bound",
            "e2e": {"value": args.nsys * n * nsteps / t_e2e, "unit": "atom-steps/s",
                    "h2d_bytes_per_step": int(P.nbytes + 16 * P.shape[0] * n), "d2h_bytes_per_step": int(16 * P.shape[0] * n)},
            "gpu_launches": args.steps, "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        v, k = raff_cpu(prep, P, nsteps, args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": "atom-steps/s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"{k} replicas x {nsteps} steps, FP64 oracle step, OpenMP over replicas"}
    R.finish()
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="uniform", choices=["uniform", "ragged", "serve", "precision", "raff"],
                    help="uniform: 4096 replicas of the 40-atom molecule (default); ragged: 16384 molecules of 20-400 atoms")
    ap.add_argument("--substrate", default="grid", choices=["grid", "folded"],
                    help="uniform workload: B-spline grid (default) or the reference's folded surface")
    ap.add_argument("--nsys", type=int, default=0, help="systems per GPU (0: the workload's default)")
    ap.add_argument("--no-tune", action="store_true", help="ragged: skip the autotuner (library defaults)")
    ap.add_argument("--resident", type=int, default=0, help="serve: cap on resident systems (0: the handle's slots)")
    ap.add_argument("--ref-sample", type=int, default=64)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-steps", type=int, default=MAX_STEPS, help="FIRE step cap per system (profiling runs)")
    ap.add_argument("--stages", default=STAGES, help="schedule: start:form:team,... (form rounds / gather / owner; team 0 = by size)")
    ap.add_argument("--profile", action="store_true", help="timed steps only: no e2e leg, no CPU baseline")
    args = ap.parse_args()
    if args.workload == "raff":
        args.nsys = args.nsys or RAFF["nsys"]
        return run_raff(args, args.impl)
    if args.impl == "reference":
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if args.workload == "ragged":
            return run_reference_ragged(args, ws, rank)
        args.nsys = args.nsys or 4096
        return run_reference(args, ws, rank)
    if args.workload == "serve":
        return run_serve(args, int(os.environ.get("LOCAL_RANK", "0")))
    if args.workload == "precision":
        return run_precision(args, int(os.environ.get("LOCAL_RANK", "0")))
    if args.workload == "ragged":
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        if ws > 1:
            return run_ragged_dist(args)
        return run_ragged(args, ws, rank, local)
    args.nsys = args.nsys or 4096
    ws, rank, local = dist_init()
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
