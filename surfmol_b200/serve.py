"""Continuous-batching relaxation server over one RelaxMulti handle.

Requests (a molecule each) arrive over time.  The server keeps every admitted system's state
resident on the device and runs the batched persistent kernel in chunks of FIRE steps over all of
them; after each chunk it retires the systems that converged or used their step budget (reading
back their results and freeing their slot, atoms and topology) and backfills the freed capacity
with waiting requests, so requests that arrive while others are on the GPU join the running batch
at the next chunk boundary.

Admission is bounded by an HBM budget: each system is charged its resident bytes (state plus
topology records, ``bytes_per_atom`` per atom) and by the handle's slot and atom capacity.

Typing and term packing of arriving molecules (host work) run on a background thread while the
GPU relaxes the current batch, so they stay off the critical path.

A system's trajectory depends only on its own FIRE step count (the kernel schedule is chosen per
system from it, and chunk boundaries save and restore the full state), so every result is
bitwise the same whether the request runs alone or in any mix.

The reference has no serving loop; its multi-system driver (crates/libs/oclff/src/rrsp3.rs:
699-1088) steps a fixed set of replicas.
"""
from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .relax import ST_RUNNING, RelaxMulti, Topology

# resident bytes per atom: pos, low parts, vel, force, staging (80 B) and the topology arenas
# (parameters, neighbours, bond constants, three record forms: ~900 B for planar C/H/N/O)
BYTES_PER_ATOM = 1024


@dataclass
class Request:
    rid: int
    Z: np.ndarray
    pos: np.ndarray
    q: np.ndarray
    arrival: float                    # seconds after the start of the run
    # filled in by the server
    t_admit: float = -1.0
    t_done: float = -1.0
    out_pos: np.ndarray | None = None
    out_pos64: np.ndarray | None = None
    energy: float = 0.0
    steps: int = 0
    status: int = 0

    @property
    def latency(self):
        return self.t_done - self.arrival


@dataclass
class ServeStats:
    n: int = 0
    wall_s: float = 0.0
    gpu_ms: float = 0.0
    chunks: int = 0
    launches: int = 0
    max_resident: int = 0
    latencies: list = field(default_factory=list)
    host_s: dict = field(default_factory=lambda: {"admit": 0.0, "run_call": 0.0, "status": 0.0, "retire": 0.0})

    def summary(self):
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        return {"requests": self.n, "wall_s": self.wall_s, "throughput_req_s": self.n / max(self.wall_s, 1e-9),
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "gpu_busy": self.gpu_ms * 1e-3 / max(self.wall_s, 1e-9), "chunks": self.chunks,
                "gpu_launches": self.launches, "max_resident": self.max_resident,
                "wall_split_s": {k: round(v, 3) for k, v in self.host_s.items()}}


class Server:
    def __init__(self, R: RelaxMulti, max_systems: int, max_atoms: int, hbm_budget_bytes: float,
                 chunk_steps: int = 200, max_steps: int = 3000, fire: dict | None = None,
                 bytes_per_atom: int = BYTES_PER_ATOM, keep_pos64: bool = False, typers: int = 8):
        self.R = R
        self.max_systems = max_systems
        self.max_atoms = max_atoms
        self.budget = float(hbm_budget_bytes)
        self.chunk = int(chunk_steps)
        self.max_steps = int(max_steps)
        self.fire = dict(fire or {})
        self.bpa = int(bytes_per_atom)
        self.keep_pos64 = keep_pos64
        self.typers = max(1, int(typers))

    # -- background typing: Topology objects of arrived requests, made by a pool of host threads
    #    (the native typing and packing release the GIL) and queued as they complete
    def _typer(self, reqs, t0, out: queue.Queue, stop: threading.Event):
        lock = threading.Lock()
        nxt = [0]
        left = [self.typers]

        def work():
            while not stop.is_set():
                with lock:
                    i = nxt[0]
                    nxt[0] += 1
                if i >= len(reqs):
                    break
                r = reqs[i]
                while not stop.is_set():
                    dt = r.arrival - (time.perf_counter() - t0)
                    if dt <= 0:
                        break
                    time.sleep(min(dt, 0.002))
                if stop.is_set():
                    break
                topo = Topology(r.Z, r.pos, r.q)
                topo.prepare(0)
                out.put((r, topo))
            with lock:
                left[0] -= 1
                last = left[0] == 0
            if last:
                out.put(None)

        pool = [threading.Thread(target=work, daemon=True) for _ in range(self.typers)]
        for t in pool:
            t.start()
        for t in pool:
            t.join()

    def run(self, requests: list[Request]) -> ServeStats:
        """Serve the requests (sorted by arrival) in real time; returns the statistics.  Each
        request gets its results, admission and completion times filled in."""
        R = self.R
        reqs = sorted(requests, key=lambda r: r.arrival)
        st = ServeStats(n=len(reqs))
        typed: queue.Queue = queue.Queue()
        stop = threading.Event()
        t0 = time.perf_counter()
        th = threading.Thread(target=self._typer, args=(reqs, t0, typed, stop), daemon=True)
        th.start()
        waiting = []                     # typed, not yet admitted: (request, topology)
        resident = {}                    # slot -> (request, topology id, atoms)
        used_bytes, used_atoms = 0.0, 0
        typer_done = False
        done = 0
        try:
            while done < len(reqs):
                # collect typed arrivals (block only when nothing is resident)
                while True:
                    try:
                        item = typed.get(block=not resident and not waiting and not typer_done, timeout=0.05)
                    except queue.Empty:
                        break
                    if item is None:
                        typer_done = True
                        break
                    waiting.append(item)
                    waiting.sort(key=lambda x: x[0].arrival)
                    if not resident:
                        break
                # admit in arrival order while slots, atoms and the HBM budget allow
                t_a = time.perf_counter()
                adm_t, adm_p, adm_r = [], [], []
                while waiting:
                    r, topo = waiting[0]
                    na = len(r.Z)
                    cost = na * self.bpa
                    if (len(resident) + len(adm_r) >= self.max_systems or used_atoms + na > self.max_atoms
                            or used_bytes + cost > self.budget):
                        break
                    waiting.pop(0)
                    adm_t.append(topo)
                    adm_p.append(r.pos)
                    adm_r.append([r, -1, na])
                    used_bytes += cost
                    used_atoms += na
                if not resident and not adm_r and waiting:
                    # larger than the whole capacity: rejected (status -1), never admitted
                    r, topo = waiting.pop(0)
                    r.status, r.t_done = -1, time.perf_counter() - t0
                    done += 1
                    continue
                if adm_r:
                    tids = R.add_topos(adm_t)                  # one upload for the whole batch
                    for x, tid in zip(adm_r, tids):
                        x[1] = int(tid)
                    slots = R.add_systems(tids, adm_p)
                    now = time.perf_counter() - t0
                    for s, (r, tid, na) in zip(slots, adm_r):
                        r.t_admit = now
                        resident[int(s)] = (r, tid, na)
                st.host_s["admit"] += time.perf_counter() - t_a
                if not resident:
                    continue
                st.max_resident = max(st.max_resident, len(resident))
                # one chunk of FIRE steps over every resident system
                t_r = time.perf_counter()
                R.run_fire(self.chunk, step_budget=self.max_steps, **self.fire)
                t_s = time.perf_counter()
                st.host_s["run_call"] += t_s - t_r
                ms, nl = R.last_timing()
                st.gpu_ms += ms
                st.launches += nl
                st.chunks += 1
                # retire finished systems
                slots = np.array(sorted(resident), np.int32)
                stat = R.download(slots, pos=False, forces=False)
                fin = slots[stat["status"] != ST_RUNNING]
                t_x = time.perf_counter()
                st.host_s["status"] += t_x - t_s
                if len(fin):
                    out = R.download(fin, pos=True, forces=False)
                    p64 = R.download_pos64(fin) if self.keep_pos64 else None
                    now = time.perf_counter() - t0
                    tids = []
                    for k, s in enumerate(fin):
                        r, tid, na = resident.pop(int(s))
                        r.out_pos = out["pos"][k]
                        r.out_pos64 = None if p64 is None else p64[k]
                        r.energy = float(out["energy"][k])
                        r.steps = int(out["steps"][k])
                        r.status = int(out["status"][k])
                        r.t_done = now
                        st.latencies.append(r.latency)
                        used_bytes -= na * self.bpa
                        used_atoms -= na
                        tids.append(tid)
                        done += 1
                    R.remove_systems(fin)
                    R.remove_topologies(tids)        # each request has its own topology
                    st.host_s["retire"] += time.perf_counter() - t_x
        finally:
            stop.set()
            th.join(timeout=5)
        st.wall_s = time.perf_counter() - t0
        return st
