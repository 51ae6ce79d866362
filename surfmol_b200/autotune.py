"""Autotuner for the batched relaxation kernels.

The reference runs one OpenCL kernel shape for every system (opencl/UFF.cl with a fixed
work-group per system, crates/libs/oclff/src/rrsp3.rs:843-852); here the launch shape is chosen
by measurement on the device, on a sample of the workload:

* per size class (systems of up to 64 / 160 / 448 / 1024 / more atoms): the threads per system
  of the throughput form, and that form itself (rounds or owner);
* the lanes per atom of the intramolecular NB loop (the interaction tiling);
* the FIRE step at which systems move to the latency-oriented gather form (the tail of a batch
  is a few slow systems, which want more threads each).

The per-class picks are timed one class at a time, while in a real run the classes share the GPU;
so the whole tuned shape is checked against the library's default shape on a full relaxation of
the sample, and the default is kept when it is faster.  Copies of sample systems (when the sample
is smaller than the probe) start at other lateral positions: identical copies would share their
grid lines in L2 and make memory-bound shapes look faster than they are on distinct systems.

Everything is timed with the library's own CUDA-event timer (``RelaxMulti.last_timing``) around
the relaxation launches; each candidate runs from the same start positions.
"""
from __future__ import annotations

import json
from dataclasses import asdict, dataclass, field

import numpy as np

from .relax import FORM_GATHER, FORM_OWNER, FORM_ROUNDS, RelaxMulti

# upper atom counts of the size classes (the library's default team changes at these sizes)
CLASS_MAX = (64, 160, 448, 1024, 1 << 20)
TEAMS = (32, 64, 128, 256, 512)


@dataclass
class TuneResult:
    team_by_class: dict = field(default_factory=dict)     # class max atoms -> threads per system
    form0: int = FORM_ROUNDS                               # throughput form of stage 0
    nb_lanes: int = 0
    stages: tuple = ((0,), (FORM_ROUNDS,), (0,))           # starts, forms, teams
    timings: dict = field(default_factory=dict)            # candidate -> atom-steps per ms

    def apply(self, R: RelaxMulti):
        """Set the tuned launch shape on a handle (call before adding molecules: a team change
        repacks every topology already added)."""
        for cmax, t in sorted(self.team_by_class.items()):
            R.set_team_size(int(cmax), int(t))
        R.set_nb_lanes(self.nb_lanes)
        R.set_stages(*[list(x) for x in self.stages])

    def save(self, path):
        d = asdict(self)
        d["team_by_class"] = {str(k): v for k, v in self.team_by_class.items()}
        json.dump(d, open(path, "w"), indent=1)

    @staticmethod
    def load(path):
        d = json.load(open(path))
        d["team_by_class"] = {int(k): v for k, v in d["team_by_class"].items()}
        d["stages"] = tuple(tuple(x) for x in d["stages"])
        return TuneResult(**d)


def _class_of(n):
    for c in CLASS_MAX:
        if n <= c:
            return c
    return CLASS_MAX[-1]


def copy_start(pos, copy: int):
    """Start positions of probe copy `copy` of a sample system: copy 0 is the system itself; later
    copies move laterally by a low-discrepancy offset of up to 37 A (the grid is periodic in x and
    y), so that they read other grid lines, as distinct systems of the real run do, instead of
    sharing the original's cached lines.  z is unchanged."""
    if copy == 0:
        return pos
    shift = np.array([(copy * 0.6180339887) % 1.0, (copy * 0.4142135624) % 1.0, 0.0]) * 37.0
    return np.asarray(pos, float) + shift


def _candidates(cmax):
    lo = {64: 32, 160: 32, 448: 64, 1024: 128}.get(cmax, 256)
    return [t for t in TEAMS if t >= lo][:3]


class Autotuner:
    """Measure launch shapes on a sample of a workload.

    make_handle(max_systems, max_atoms) must return a RelaxMulti with the workload's grid and NB
    parameters set (the tuner adds the sample's molecules itself)."""

    def __init__(self, make_handle, fire: dict, probe_steps: int = 100, max_steps: int = 2000, verbose: bool = False,
                 max_probe_systems: int = 8192):
        self.make_handle = make_handle
        self.max_probe_systems = max_probe_systems
        self.fire = dict(fire)
        self.probe_steps = probe_steps
        self.max_steps = max_steps
        self.verbose = verbose

    def _log(self, *a):
        if self.verbose:
            print("[autotune]", *a, flush=True)

    def _rate(self, R, slots, natoms, steps):
        """atom-steps per ms of `steps` FIRE steps of `slots` from their start positions."""
        R.reset_fire(slots)
        R.run_fire(steps, step_budget=steps, **self.fire)
        ms = R.last_timing()[0]
        done = R.download(slots, pos=False, forces=False)["steps"]
        return float((np.asarray(natoms) * done).sum()) / max(ms, 1e-6)

    def tune(self, Zs, poss, qs, full_count: int | None = None) -> TuneResult:
        """Zs / poss / qs: a sample of the workload; full_count: systems in the whole workload.  The
        probes replicate the sample towards full_count (at most max_probe_systems), so the GPU is
        as full as in the real run: occupancy decides which team size wins.  A probe that fits on
        the GPU in one wave measures latency, and favours large teams that lose on a full run."""
        n = np.array([len(z) for z in Zs])
        res = TuneResult()
        rep_f = max(1.0, min(float(full_count or len(Zs)), float(self.max_probe_systems)) / len(Zs))

        def replicate(idx):
            """probe systems for sample systems idx: (sample index, copy number) towards full_count"""
            k = max(1, int(round(len(idx) * rep_f)))
            return [(int(idx[j % len(idx)]), j // len(idx)) for j in range(k)]

        def start(i, copy):
            return copy_start(poss[i], copy)
        classes = sorted({_class_of(int(k)) for k in n})
        # 1. per class: form and threads per system of stage 0 (probe_steps from the start positions)
        best_forms = {}
        for c in classes:
            idx = np.nonzero([_class_of(int(k)) == c for k in n])[0]
            probe = replicate(idx)                            # systems of this class in the probe
            sys_idx = [i for i, _ in probe]
            pos_of = {int(i): j for j, i in enumerate(idx)}
            best = None
            for t in _candidates(c):
                R = self.make_handle(len(sys_idx), int(n[sys_idx].sum()))
                try:
                    R.set_team_size(c, t)
                    tids = R.add_molecules([Zs[i] for i in idx], [poss[i] for i in idx], [qs[i] for i in idx])
                    slots = R.add_systems([tids[pos_of[i]] for i in sys_idx], [start(i, cp) for i, cp in probe])
                    for form in (FORM_ROUNDS, FORM_OWNER):
                        R.set_stages([0], [form], [0])
                        self._rate(R, slots, n[sys_idx], 5)   # first launch of this shape: not timed
                        r = self._rate(R, slots, n[sys_idx], self.probe_steps)
                        res.timings[f"class<={c} team={t} form={form}"] = r
                        self._log(f"class <= {c} atoms: team {t} form {form}: {r:.0f} atom-steps/ms")
                        if best is None or r > best[0]:
                            best = (r, t, form)
                finally:
                    R.finish()
            res.team_by_class[c] = best[1]
            best_forms[c] = (best[0], best[2])
        # the stage-0 form is one for all classes: the one with the larger summed rate share
        score = {FORM_ROUNDS: 0.0, FORM_OWNER: 0.0}
        for c in classes:
            w = float(n[[_class_of(int(k)) == c for k in n]].sum())
            for form in score:
                r = res.timings.get(f"class<={c} team={res.team_by_class[c]} form={form}", 0.0)
                score[form] += w / max(r, 1e-9)
        res.form0 = min(score, key=score.get)
        # 2. interaction tiling and 3. the tail switch, on the whole sample (replicated)
        all_probe = replicate(np.arange(len(Zs)))
        all_idx = [i for i, _ in all_probe]
        n_all = n[all_idx]
        handles = []

        def sample_handle(teams):
            H = self.make_handle(len(all_idx), int(n_all.sum()))
            handles.append(H)
            for c, t in teams.items():
                H.set_team_size(c, t)
            tids = H.add_molecules(Zs, poss, qs)
            return H, H.add_systems([tids[i] for i in all_idx], [start(i, cp) for i, cp in all_probe])

        def full_ms(H, slots):
            """device ms of a full relaxation of the sample (best of two) and its step counts"""
            best = None
            for _ in range(2):
                H.reset_fire(slots)
                H.run_fire(self.max_steps, step_budget=self.max_steps, **self.fire)
                ms = H.last_timing()[0]
                best = ms if best is None else min(best, ms)
            return best, H.download(slots, pos=False, forces=False)["steps"]

        try:
            R, slots = sample_handle(res.team_by_class)
            n = n_all
            R.set_stages([0], [res.form0], [0])
            # two timings of every candidate, the second sweep in reverse order, best of the two:
            # neighbouring candidates differ by a few percent, about the spread of one timing
            rates = {}
            for order in ((0, 1, 2, 4, 8), (8, 4, 2, 1, 0)):
                for lanes in order:
                    R.set_nb_lanes(lanes)
                    self._rate(R, slots, n, 5)
                    r = self._rate(R, slots, n, self.probe_steps)
                    rates[lanes] = max(rates.get(lanes, 0.0), r)
            for lanes, r in rates.items():
                res.timings[f"nb_lanes={lanes}"] = r
                self._log(f"nb lanes {lanes}: {r:.0f} atom-steps/ms")
            best_l = max(rates, key=rates.get)
            res.nb_lanes = best_l
            R.set_nb_lanes(best_l)
            # full relaxation of the sample in the throughput form: the step distribution
            base_ms, steps = full_ms(R, slots)
            # the per-class picks were timed one class at a time, but in the real run the classes
            # share the GPU: keep them only if the whole shape beats the library's default shape
            D, dslots = sample_handle({})
            D.set_stages([0], [FORM_ROUNDS], [0])
            D.set_nb_lanes(0)
            def_ms, def_steps = full_ms(D, dslots)
            res.timings["relax_ms_tuned_shape"] = base_ms
            res.timings["relax_ms_default_shape"] = def_ms
            self._log(f"tuned shape {base_ms:.1f} ms, default shape {def_ms:.1f} ms")
            if def_ms < base_ms:
                res.team_by_class, res.form0, res.nb_lanes = {}, FORM_ROUNDS, 0
                R, slots, base_ms, steps = D, dslots, def_ms, def_steps
            cands = [((0,), (res.form0,), (0,), base_ms)]
            for q in (0.5, 0.65, 0.8):
                s1 = int(np.quantile(steps, q))
                if s1 < 10 or s1 >= self.max_steps:
                    continue
                s2 = int(min(self.max_steps - 1, s1 + 0.5 * (self.max_steps - s1)))
                for st, fm, tm in (((0, s1), (res.form0, FORM_GATHER), (0, 0)),
                                   ((0, s1, s2), (res.form0, FORM_GATHER, FORM_GATHER), (0, 64, 128))):
                    R.set_stages(list(st), list(fm), list(tm))
                    R.reset_fire(slots)
                    R.run_fire(self.max_steps, step_budget=self.max_steps, **self.fire)
                    ms = R.last_timing()[0]
                    cands.append((st, fm, tm, ms))
                    self._log(f"stages {st} forms {fm} teams {tm}: {ms:.1f} ms")
            st, fm, tm, ms = min(cands, key=lambda x: x[3])
            res.stages = (tuple(st), tuple(fm), tuple(tm))
            res.timings["relax_ms_single_stage"] = base_ms
            res.timings["relax_ms_tuned"] = ms
        finally:
            for H in handles:
                H.finish()
        return res
