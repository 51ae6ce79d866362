#!/usr/bin/env python
"""Benchmark: relaxed systems per second on one B200 (per rank), JSON line on stdout.

Default workload (the metric's configuration): 16384 distinct planar C/H/N/O molecules of 20-400
atoms (log-uniform), each at a random lateral position, rotation and height 2.5-4 A over a
3-layer 8x8-cell NaCl(100) slab; FP32 B-spline grid 451x451x161 (0.1 A, 524 MB) built on the
device; intramolecular LJ + Coulomb with a 10 A cutoff; FIRE (dt0 0.001, dt_max 0.05) to
max|F| < 1e-4 eV/A.  `value` counts the systems that relaxed to that tolerance per second; the
all-systems rate, converged fraction, served p50 / p99 latency (continuous batching of the same
molecules below capacity) and the HBM roofline sit beside it.

One bench step = relaxing the whole batch from its start positions.  The device time of each
step is taken with CUDA events on the library's stream around the relaxation launches; L2 is
flushed (256 MB write) before every step.  Under torchrun (or --gpus N, which starts N ranks)
each rank relaxes its own batch (weak scaling, no collective on the data path); the reported
time is the max over ranks.

--impl reference times the FP64 CPU restatement of the same path (oracle/), the reference's own
algorithm, on all host cores, on a bounded sample per step.  --workload uniform runs 4096 replicas
of the 40-atom molecule (to 1e-3 eV/A); serve, precision and raff run the other configurations.
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
    sample = min(args.nsys, 8 * threads)          # the cpu_baseline leg's sample: one batch of 8 x cores

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
def cpu_baseline(w, grid, per_core=8):
    """grid: the oracle's substrate (oracle.Grid or oracle.Folded).  One OpenMP batch (one system per
    thread, dynamic schedule) over per_core x cores systems of the workload, so the 2000-step tails
    spread over the threads as they would in a long run."""
    from oracle import oracle as O
    sys0 = O.System.from_molecule(w.Z[0], w.pos[0], w.q[0])
    threads = os.cpu_count() or 1
    n = min(len(w.pos), per_core * threads)
    t = time.perf_counter()
    r = O.relax_batch([sys0] * n, [w.pos[i] for i in range(n)], grid, max_steps=MAX_STEPS, nthreads=threads, **FIRE)
    dt = time.perf_counter() - t
    return {"value": n / dt, "unit": "systems/s", "cores": threads, "kind": "port",
            "sample": f"{n} systems of the same workload in one OpenMP batch (relaxed to convergence or {MAX_STEPS} "
                      f"steps, {int(r['conv'].sum())} converged), FP64 oracle, {dt:.1f} s"}


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
        line["cpu_baseline"] = cpu_baseline(w, og)
    R.finish()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------------------- ragged workload
# The metric's configuration: 16384 distinct molecules of 20-400 atoms, 10 A intramolecular cutoff,
# FIRE to 1e-4 eV/A.  The step cap is set where ~95 % of the molecules converge: FIRE needs ~2000
# steps for the small ones and 4000+ for the large (the FP64 oracle needs the same counts).
RAGGED = dict(nsys=16384, nmin=20, nmax=400, rcut=10.0, fconv=1e-4, max_steps=10000, tune_sample=4096,
              cpu_per_core=8, serve_requests=4096, serve_rate=400.0, serve_chunk=200)


def ragged_desc(nsys, g, max_steps):
    return (f"ragged: {nsys} distinct planar C/H/N/O molecules, atoms log-uniform in [{RAGGED['nmin']}, {RAGGED['nmax']}], "
            f"over NaCl(100) 3 layers 8x8 cells, fp32 B-spline grid {g.nx}x{g.ny}x{g.nz} at 0.1 A; intramolecular "
            f"cutoff {RAGGED['rcut']} A; FIRE to max|F|<{RAGGED['fconv']} eV/A or {max_steps} steps")


def ragged_workload(seed, nsys):
    from surfmol_b200 import synth
    return synth.ragged(seed, nsys, RAGGED["nmin"], RAGGED["nmax"], ncell=8, nlayers=3, nz=161,
                        workers=min(32, os.cpu_count() or 1))


def ragged_cpu_grid(w):
    """The FP64 oracle's grid of the workload (Morse terms of ion images beyond 25 A dropped: below
    1e-15 of the nearest ion's), stored as float32 like the GPU's."""
    from oracle import oracle as O
    slab, g = w.slab, w.grid
    coef = O.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step, morse_rcut=25.0)
    return O.Grid(coef.astype(np.float32), g.p0, g.step)


def ragged_cpu_batch(w, grid, idx, max_steps, threads):
    """One OpenMP batch (one system per thread, dynamic schedule) over the molecules idx:
    (seconds, converged count, steps)."""
    from oracle import oracle as O
    systems = [O.System.from_molecule(w.Z[i], w.pos[i], w.q[i]) for i in idx]
    t = time.perf_counter()
    r = O.relax_batch(systems, [w.pos[i] for i in idx], grid, max_steps=max_steps, nthreads=threads,
                      nb=dict(rdamp=1.0, alpha=1.5, rcut=RAGGED["rcut"]), **dict(FIRE, fconv=RAGGED["fconv"]))
    return time.perf_counter() - t, int(r["conv"].sum()), r["steps"]


def run_reference_ragged(args, ws, rank):
    if rank != 0:
        return 0
    nsys = args.nsys or RAGGED["nsys"]
    max_steps = args.max_steps or RAGGED["max_steps"]
    w = ragged_workload(SEED, nsys)
    t0 = time.perf_counter()
    grid = ragged_cpu_grid(w)
    tgrid = time.perf_counter() - t0
    threads = os.cpu_count() or 1
    sample = RAGGED["cpu_per_core"] * threads
    k0 = 0
    for _ in range(args.warmup):                 # warm-up batches: a quarter of the sample
        n = max(threads, sample // 4)
        ragged_cpu_batch(w, grid, [(k0 + i) % nsys for i in range(n)], max_steps, threads)
        k0 += n
    tt, conv, done, steps = 0.0, 0, 0, []
    for _ in range(args.steps):
        dt, c, st = ragged_cpu_batch(w, grid, [(k0 + i) % nsys for i in range(sample)], max_steps, threads)
        k0 += sample
        tt += dt; conv += c; done += sample; steps += list(st)
    v = conv / tt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "relaxed systems/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": ragged_desc(nsys, w.grid, max_steps), "sample_per_step": sample,
                       "all_systems_per_s": done / tt, "converged_fraction": conv / done,
                       "fire_steps_p50": float(np.percentile(steps, 50)), "fire_steps_p99": float(np.percentile(steps, 99)),
                       "grid_build_s": round(tgrid, 1)},
            "cpu_baseline": {"value": v, "unit": "relaxed systems/s", "cores": threads, "kind": "port",
                             "sample": f"{sample} molecules of the workload per step in one OpenMP batch "
                                       f"(FP64 oracle, oracle/oracle.cpp, one system per thread, dynamic schedule)"},
            "e2e": {"value": v, "unit": "relaxed systems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def parse_shape(txt):
    """'64:64,160:64,448:128/2' -> a TuneResult: threads per system for systems up to each atom
    count, NB lanes per atom after the slash, one rounds-form stage (a shape the autotuner picked)."""
    from surfmol_b200.autotune import TuneResult
    part, _, rest = txt.partition("/")
    teams = {int(a): int(b) for a, b in (x.split(":") for x in part.split(","))}
    lanes = int(rest) if rest else 0
    return TuneResult(team_by_class=teams, form0=0, nb_lanes=lanes, stages=((0,), (0,), (0,)))


def served_latency(R, w, rate, nreq, max_steps, fire, natoms_max):
    """Continuous batching on the workload's own molecules: the first nreq arrive Poisson at `rate`
    per second and are served by the same handle (surfmol_b200/serve.py); arrival-to-result
    latencies.  A few requests run first to load every kernel shape."""
    from surfmol_b200.serve import Request, Server
    rng = np.random.default_rng([SEED, 77])
    t_arr = np.cumsum(rng.exponential(1.0 / rate, nreq))
    srv = Server(R, R.max_systems, natoms_max, 150e9, chunk_steps=RAGGED["serve_chunk"], max_steps=max_steps, fire=fire,
                 typers=min(16, os.cpu_count() or 1))
    srv.run([Request(i, w.Z[i], w.pos[i], w.q[i], 0.0) for i in range(min(64, nreq))])
    rq = [Request(i, w.Z[i], w.pos[i], w.q[i], float(t_arr[i])) for i in range(nreq)]
    d = srv.run(rq).summary()
    d.update(rate_req_s=rate, converged_fraction=float(np.mean([r.status == 1 for r in rq])),
             workload=f"the first {nreq} molecules of the workload, Poisson arrivals at {rate:.0f} req/s (below the "
                      f"~800 req/s at which host-side typing and admission saturate), chunks of {RAGGED['serve_chunk']} FIRE steps")
    return d


def run_ragged(args, ws, rank, local):
    nsys = args.nsys or RAGGED["nsys"]
    max_steps = args.max_steps or RAGGED["max_steps"]
    t0 = time.perf_counter()
    w = ragged_workload(SEED + 7919 * rank, nsys)          # generated before any CUDA work (spawned pool)
    tgen = time.perf_counter() - t0
    import torch
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.autotune import Autotuner
    torch.cuda.set_device(local)
    slab, g = w.slab, w.grid
    natoms = np.array([len(z) for z in w.Z])
    fire = dict(FIRE, fconv=RAGGED["fconv"])

    def make_handle(ms, ma):
        R = RelaxMulti(max_systems=ms, max_atoms=ma, device=local)
        R.set_nb(rdamp=1.0, alpha_morse=1.5, rcut=RAGGED["rcut"])
        R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step, alpha_morse=1.5, npbc=1)
        if args.grid_bricks is not None:
            R.set_grid_bricks(args.grid_bricks)
        return R

    t0 = time.perf_counter()
    tune = None
    if args.shape:
        tune = parse_shape(args.shape)
    elif not args.no_tune:
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
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2

    def step():
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)
        flush.zero_()
        torch.cuda.synchronize()
        R.run_fire(max_steps, step_budget=max_steps, **fire)
        return R.last_timing()

    for _ in range(args.warmup):
        step()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    dev_ms, launches, atom_steps, conv, steps_all = 0.0, 0, 0, 0, []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ms, nl = step()
            dev_ms += ms
            launches += nl
            out = R.download(slots, pos=False, forces=False)
            atom_steps += int((out["steps"].astype(np.int64) * natoms).sum())
            conv += int((out["status"] == 1).sum())
            steps_all += list(out["steps"])
        torch.cuda.synchronize()
    from surfmol_b200.shard import sum_over_ranks
    dev_ms = barrier_max(ws, dev_ms)
    conv_all = sum_over_ranks(conv)
    ms_step = dev_ms / args.steps
    value = conv_all / args.steps / (ms_step * 1e-3)
    all_rate = ws * nsys / (ms_step * 1e-3)
    if args.profile:
        R.finish()
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms_step, "atom_steps": atom_steps, "launches": launches}))
        return 0
    # end to end through the public API with host buffers: positions H2D, relax, positions + status D2H
    e2e_k = max(1, min(args.steps, 2))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    conv_e2e = 0
    for _ in range(e2e_k):
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)
        R.run_fire(max_steps, step_budget=max_steps, **fire)
        res = R.download(slots, pos=True, forces=False)
        conv_e2e += int((res["status"] == 1).sum())
    t_e2e = barrier_max(ws, time.perf_counter() - t0)
    conv_e2e = sum_over_ranks(conv_e2e)
    hbm, peak_kind = peaks()
    grid_layout = "bricks" if R.grid_bricks_active() else "z-fastest"
    achieved = 1024.0 * atom_steps / args.steps / (ms_step * 1e-3) / 1e9
    traffic, issue = None, None
    prof = os.path.join(ROOT, "profiles", f"relax_ragged_traffic_{grid_layout}.json")
    if os.path.exists(prof):
        pj = json.load(open(prof))
        traffic = pj["dram_bytes_per_atom_step"] * atom_steps / args.steps
        # the bound the kernel actually meets: warp-instruction issue (ncu instructions per atom-step
        # x atom-steps / time, against 4 schedulers x 148 SMs at the sampled SM clock)
        mhz = clk.summary()["sm_mhz"] or 1965.0
        if "warp_inst_per_atom_step" in pj:
            rate = pj["warp_inst_per_atom_step"] * atom_steps / args.steps / (ms_step * 1e-3)
            ipeak = 4 * 148 * mhz * 1e6
            issue = {"achieved": rate, "peak": ipeak, "unit": "warp-instructions/s", "frac": rate / ipeak,
                     "inst_per_atom_step": pj["warp_inst_per_atom_step"]}
    line = {"metric": METRIC, "value": value, "unit": "relaxed systems/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": ragged_desc(nsys, g, max_steps), "nsys_per_gpu": nsys, "atoms_total": int(natoms.sum()),
                       "atoms_mean": float(natoms.mean()),
                       "parallelism": f"systems sharded over {ws} GPU(s), no collective in the step",
                       "l2": "flushed (256 MB write) before every timed step; the 524 MB grid exceeds L2",
                       "value_counts": "systems relaxed to max|F| < 1e-4 eV/A per second (unconverged ones excluded)",
                       "all_systems_per_s": all_rate, "converged_fraction": conv / (nsys * args.steps),
                       "fire_steps_p50": float(np.percentile(steps_all, 50)), "fire_steps_p99": float(np.percentile(steps_all, 99)),
                       "grid_layout": grid_layout,
                       "host_s": {"generate": round(tgen, 2), "autotune": round(ttune, 2), "add_molecules": round(tadd, 2)},
                       "tuned": None if tune is None else {"team_by_class": tune.team_by_class, "form0": tune.form0,
                                                            "nb_lanes": tune.nb_lanes, "stages": tune.stages}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes": "1024 B per atom-step (64 float4 grid voxels), state resident in shared memory",
                         "issue": issue},
            "e2e": {"value": conv_e2e / e2e_k / (t_e2e / e2e_k), "unit": "relaxed systems/s",
                    "h2d_bytes_per_step": int(16 * natoms.sum() + 76 * nsys), "d2h_bytes_per_step": int(16 * natoms.sum() + 128 * nsys)},
            "latency": {"batch_s": t_e2e / e2e_k},
            "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        gd = R.get_grid()
        og = O.Grid(gd["coef"], gd["p0"], gd["step"])
        threads = os.cpu_count() or 1
        # twice the reference arm's per-step sample: one batch's time is set by its slowest
        # molecules, and this leg has one batch where the reference arm averages many
        n = 2 * RAGGED["cpu_per_core"] * threads
        dt, c, _ = ragged_cpu_batch(w, og, list(range(n)), max_steps, threads)
        line["cpu_baseline"] = {"value": c / dt, "unit": "relaxed systems/s", "cores": threads, "kind": "port",
                                "sample": f"{n} molecules of the workload in one OpenMP batch (FP64 oracle, one system per "
                                          f"thread, dynamic schedule), {dt:.1f} s, {c} converged"}
    if rank == 0 and not args.no_serve:
        R.remove_systems(slots)
        R.remove_topologies(tids)
        line["latency"]["served"] = served_latency(R, w, RAGGED["serve_rate"], RAGGED["serve_requests"], max_steps, fire,
                                                   int(natoms.sum()))
    R.finish()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------- served workload
SERVE = dict(nmin=20, nmax=2000, rcut=10.0, fconv=1e-4, max_steps=10000, chunk=200, budget_gb=150.0,
             rates=(100.0, 150.0, 200.0, 300.0, 2000.0, 10000.0, 50000.0), per_rate=20000, max_systems=2048,
             plain_sample=8, resident=0)


def run_serve(args, local):
    from surfmol_b200 import synth
    slab, g = synth.config3_slab_grid()
    per = args.nsys or SERVE["per_rate"]
    rates = tuple(float(x) for x in args.rates.split(",")) if args.rates else SERVE["rates"]
    workers = min(32, os.cpu_count() or 1)
    # every request generated up front in a spawned pool, before any CUDA work; one set of `per`
    # molecules serves every rate, each rate with its own Poisson arrival times
    streams = {"warm": synth.serve_requests(SEED + 1, 64, 1e5, slab, SERVE["nmin"], SERVE["nmax"], workers),
               "plain": synth.serve_requests(SEED + 999, SERVE["plain_sample"], 1e5, slab, SERVE["nmin"], SERVE["nmax"])}
    base = synth.serve_requests(SEED + 100, per, 1.0, slab, SERVE["nmin"], SERVE["nmax"], workers)
    for k, rate in enumerate(rates):
        t = np.cumsum(np.random.default_rng([SEED, 100 + k]).exponential(1.0 / rate, per))
        streams[k] = [(Z, P, q, float(t[i])) for i, (Z, P, q, _) in enumerate(base)]
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
                 npbc=1)
    # the fp16 grid, with FP32 planes near the surface unless --plain-fp16 (the precision workload
    # measures the force error of each storage)
    zsplit = 0 if args.plain_fp16 else split_plane(slab, g)
    if zsplit:
        R.convert_grid_split(GRID_F16, zsplit)
    else:
        R.convert_grid(GRID_F16)
    tgrid = time.perf_counter() - t0
    resident = args.resident or SERVE["resident"] or SERVE["max_systems"]
    srv = Server(R, resident, max_atoms, SERVE["budget_gb"] * 1e9, chunk_steps=SERVE["chunk"],
                 max_steps=SERVE["max_steps"], fire=fire, typers=min(16, os.cpu_count() or 1))

    def reqs(key):
        return [Request(i, Z, P, q, t) for i, (Z, P, q, t) in enumerate(streams[key])]
    srv.run(reqs("warm"))                                  # warm-up: loads every kernel shape
    points = []
    for k, rate in enumerate(rates):
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
            "config": {"workload": f"served: Poisson arrivals at {list(rates)} req/s, {per} requests per rate, "
                                   f"molecules log-uniform {SERVE['nmin']}-{SERVE['nmax']} atoms, fp16 grid "
                                   + (f"(FP32 planes below {SPLIT_HEIGHT} A above the top ion layer) " if zsplit else "") +
                                   f"{g.nx}x{g.ny}x{g.nz} of a 3-layer 16x16-cell NaCl(100) slab, intramolecular cutoff "
                                   f"{SERVE['rcut']} A, FIRE to {SERVE['fconv']} or {SERVE['max_steps']} steps, "
                                   f"chunks of {SERVE['chunk']} steps, HBM budget {SERVE['budget_gb']} GB",
                       "grid_build_s": round(tgrid, 2), "resident_cap": resident,
                       "grid_precision": ("fp16 above the split plane, FP32 below it: the FP64-oracle force error at "
                                          "relaxed positions is the FP32 grid's (--workload precision)") if zsplit else
                                         ("the plain fp16 grid carries ~3.9e-3 eV/A of force error at relaxed positions "
                                          "against the FP64 oracle (--workload precision): served results miss the "
                                          "1e-4 eV/A bar by that margin"),
                       "fp16_split_plane": zsplit},
            "serve": points, "plain": plain, "served_over_plain": best / plain["throughput_req_s"]}
    R.finish()
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------- grid precision
PREC = dict(nsys=8192, nmin=20, nmax=400, rcut=10.0, fconv=1e-4, max_steps=3000, sample=256)
# split 16-bit grids keep FP32 planes for the stencils that start below this height above the top ion
# layer: there the channels are large and cancel at a relaxed position
SPLIT_HEIGHT = 5.0


def split_plane(slab, g):
    """first stencil start plane that reads the 16-bit grid of a split grid"""
    return max(1, min(g.nz - 3, int(round((slab.z_top + SPLIT_HEIGHT - g.p0[2]) / g.step[2]))))


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
    if args.grid_bricks is not None:
        R.set_grid_bricks(args.grid_bricks)
    max_steps = args.max_steps or PREC["max_steps"]
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
    zsplit = split_plane(slab, g)
    for name, dt in (("f32", GRID_F32), ("f16", GRID_F16), ("bf16", GRID_BF16), ("f16_split", GRID_F16),
                     ("bf16_split", GRID_BF16)):
        R.set_grid(gd["coef"], gd["p0"], gd["step"])          # from the FP32 coefficients each time
        split = name.endswith("_split")
        if split:
            R.convert_grid_split(dt, zsplit)
        elif dt != GRID_F32:
            R.convert_grid(dt)
        scale = R.get_grid()["scale"] if dt != GRID_F32 else np.ones(4)
        R.set_positions(slots, w.pos)
        R.reset_fire(slots)
        R.run_fire(max_steps, step_budget=max_steps, **fire)
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
        gbytes = g.nx * g.ny * g.nz * (16 if dt == GRID_F32 else 8) + (g.nx * g.ny * (zsplit + 3) * 16 if split else 0)
        variants[name] = {"grid_bytes": int(gbytes),
                          "fp32_planes": (zsplit + 3) if split else (g.nz if dt == GRID_F32 else 0),
                          "grid_layout": "bricks" if R.grid_bricks_active() else "z-fastest",
                          "channel_scales": [float(x) for x in scale], "relax_ms": ms, "systems_per_s": nsys / (ms * 1e-3),
                          "converged_fraction": float((st["status"] == 1).mean()),
                          "fire_steps_p50": float(np.median(st["steps"])), "error_vs_fp64_oracle": errs}
        print(json.dumps({name: variants[name]}), file=sys.stderr, flush=True)
    line = {"metric": "FP64-oracle force / energy error per grid storage type", "n_gpus": 1, "data": "synthetic",
            "config": {"workload": f"{nsys} molecules log-uniform {PREC['nmin']}-{PREC['nmax']} atoms over a 3-layer "
                                   f"16x16-cell NaCl(100) slab, grid {g.nx}x{g.ny}x{g.nz}; errors on {len(pick)} systems "
                                   f"at their start and FP32-relaxed positions; FIRE to {PREC['fconv']} or {max_steps}",
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


def spawn_ranks(n):
    """--gpus N without a launcher: run this command again under torch.distributed.run with N
    ranks on this node (rendezvous on 127.0.0.1), and return its exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def launch_check(args):
    """The launch path alone (no GPU work): every rank joins a gloo group, takes the max over ranks
    of its rank number, and rank 0 prints the rank count it saw."""
    import datetime
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    top = barrier_max(ws, float(rank))
    if rank == 0:
        print(json.dumps({"launch_check": True, "n_gpus": ws, "max_rank": top, "requested": args.gpus}), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ragged", choices=["uniform", "ragged", "serve", "precision", "raff"],
                    help="ragged (default): 16384 molecules of 20-400 atoms, FIRE to 1e-4; uniform: 4096 replicas of "
                         "the 40-atom molecule to 1e-3")
    ap.add_argument("--substrate", default="grid", choices=["grid", "folded"],
                    help="uniform workload: B-spline grid (default) or the reference's folded surface")
    ap.add_argument("--nsys", type=int, default=0, help="systems per GPU (0: the workload's default)")
    ap.add_argument("--no-tune", action="store_true", help="ragged: skip the autotuner (library defaults)")
    ap.add_argument("--no-serve", action="store_true", help="ragged: skip the served-latency measurement")
    ap.add_argument("--shape", default="", help="ragged: launch shape instead of the autotuner, e.g. 64:64,160:64,448:128/2")
    ap.add_argument("--grid-bricks", type=int, default=None, choices=[-1, 0, 1],
                    help="grid layout the kernel reads (-1 auto, 0 z-fastest, 1 brick copy)")
    ap.add_argument("--resident", type=int, default=0, help="serve: cap on resident systems (0: the handle's slots)")
    ap.add_argument("--plain-fp16", action="store_true", help="serve: the plain fp16 grid, without FP32 near-surface planes")
    ap.add_argument("--rates", default="", help="serve: comma-separated arrival rates in req/s (default: the workload's)")
    ap.add_argument("--ref-sample", type=int, default=64)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-steps", type=int, default=0, help="FIRE step cap per system (0: the workload's default)")
    ap.add_argument("--stages", default=STAGES, help="schedule: start:form:team,... (form rounds / gather / owner; team 0 = by size)")
    ap.add_argument("--profile", action="store_true", help="timed steps only: no e2e leg, no CPU baseline")
    ap.add_argument("--launch-check", action="store_true", help="test the --gpus N launch path without GPU work")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    if args.launch_check:
        return launch_check(args)
    if args.workload == "raff":
        args.nsys = args.nsys or RAFF["nsys"]
        return run_raff(args, args.impl)
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.workload == "ragged":
            return run_reference_ragged(args, ws, rank)
        args.nsys = args.nsys or 4096
        args.max_steps = args.max_steps or MAX_STEPS
        return run_reference(args, ws, rank)
    if args.workload == "serve":
        return run_serve(args, local)
    if args.workload == "precision":
        return run_precision(args, local)
    if args.workload == "ragged":
        if ws > 1:
            return run_ragged_dist(args)
        return run_ragged(args, ws, rank, local)
    args.nsys = args.nsys or 4096
    args.max_steps = args.max_steps or MAX_STEPS
    ws, rank, local = dist_init()
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
