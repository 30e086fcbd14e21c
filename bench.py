"""Benchmark of the BacColonyGrowth hot path on B200.

One step = one pass of the hot path over the colony: MoveCell + GrowCell for
every cell (two-stage integration with forces from the neighbour lists,
growth), the division loop with its partial neighbour rebuilds, the full
neighbour rebuild on the reference's UpdateTime cadence (every 100 steps),
and one agar solve (Multigrid::solve with `--vcycles` V-cycles) -- the
"1,000 mechanics steps with one V-cycle nutrient solve per step" schedule,
on the 1,048,576-cell workload restated in the reference's 2-D x-z geometry.

Metric: cell-steps/s (cells x steps / time), with the multigrid DOF/s of
the solve reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference      # the reference's own CPU code
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="mixed_1m")
    ap.add_argument("--vcycles", type=int, default=1)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mg-tol", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-members", type=int, default=64)
    ap.add_argument("--no-output", action="store_true", help="skip the output-step measurement")
    ap.add_argument("--no-dense", action="store_true", help="skip the densely packed colony's mechanics line")
    ap.add_argument("--no-field-update", action="store_true",
                    help="skip the field update at the reference's cadence (266 solves + 200 sweeps each)")
    ap.add_argument("--smoother-warps", type=int, default=0,
                    help="pin the agar smoother's resident-warp target instead of autotuning it (profiling)")
    ap.add_argument("--relax-mode", type=int, default=-1,
                    help="agar smoother form (bcg_set_relax_mode; default: the library's)")
    ap.add_argument("--force-group", type=int, default=0,
                    help="pin the force loop's lanes per cell instead of autotuning it (profiling)")
    return ap.parse_args()


def mg_dof(p):
    """3 species x the finest composite levels' points (the work unit of one
    V-cycle; coarser levels count as work, not DOF)."""
    A = p.max_levels_mg
    return 3 * A * (p.box_x + 1) * (p.box_z_agar + 1)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
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


def set_depleted_wall(lib, ctx, p, rows=None):
    """Level-0 wall rows depleted under the colony, so that the agar solve
    has a non-zero right-hand side (from the uniform start it has none).
    Returns the rows (computed from the context's INSIDE field if not given)."""
    import numpy as np
    from baccolonygrowth_b200 import _abi
    from baccolonygrowth_b200.colony import depleted_wall
    if rows is None:
        ins = np.zeros(p.box_x * p.box_z)
        _abi.check(lib.bcg_get_field(ctx, _abi.FIELDS["INSIDE"], 0, _abi.ptr(ins, ctypes.c_double), ins.size), "inside")
        rows = [np.ascontiguousarray(v) for v in depleted_wall(p, ins)]
    for name, v in zip(("WALLF_CARBON", "WALLF_OXYGEN", "WALLF_ACETATE"), rows):
        _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS[name], 0, _abi.ptr(v, ctypes.c_double), v.size), name)
    return rows


def ensemble_bench(lib, args, steps=5, warmup=2):
    """bcg_ensemble_run over `args.ensemble_members` colonies vs bcg_sim_run
    on the same members in turn.  Host wall time with the device
    synchronised on both sides (the members run on their own streams)."""
    import numpy as np
    import torch
    from baccolonygrowth_b200 import _abi, params as _params
    from baccolonygrowth_b200.colony import synth_colony
    rng = np.random.default_rng(20261209)
    sizes = np.exp(rng.uniform(np.log(1000), np.log(100000), args.ensemble_members)).astype(int)

    def build():
        sims, total = [], 0
        for j, n in enumerate(sizes):
            p = _params.ensemble_member(int(n))
            w, h = _params.dome_size(int(n), 1.0 / 20.0)
            cells = np.ascontiguousarray(synth_colony(int(n), w, h, seed=7000 + j, div_phase_spread=1.0))
            sim = ctypes.c_void_p()
            _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(cells), len(cells), 100 + j, 0, ctypes.byref(sim)), "member")
            _abi.check(lib.bcg_sim_set_step_mode(sim, 0, args.vcycles), "member mode")
            ctx = lib.bcg_sim_ctx(sim)
            g = np.full(p.box_x * p.box_z, 0.9)
            _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size), "g")
            _abi.check(lib.bcg_update_density(ctx), "density")
            set_depleted_wall(lib, ctx, p)
            sims.append(sim)
            total += len(cells)
        return sims, total

    def cells_of(sims):
        tot = 0
        for s in sims:
            n = ctypes.c_int()
            lib.bcg_num_cells(lib.bcg_sim_ctx(s), ctypes.byref(n))
            tot += n.value
        return tot

    # together
    sims, total = build()
    arr = (ctypes.c_void_p * len(sims))(*[s.value for s in sims])
    e = ctypes.c_void_p()
    _abi.check(lib.bcg_ensemble_create(arr, len(sims), ctypes.byref(e)), "ensemble")
    _abi.check(lib.bcg_ensemble_run(e, warmup), "ensemble warmup")
    torch.cuda.synchronize()
    c0 = cells_of(sims)
    t0 = time.perf_counter()
    _abi.check(lib.bcg_ensemble_run(e, steps), "ensemble run")
    torch.cuda.synchronize()
    t_ens = time.perf_counter() - t0
    work_ens = 0.5 * (c0 + cells_of(sims)) * steps
    lib.bcg_ensemble_destroy(e)
    for s in sims:
        lib.bcg_sim_destroy(s)
    # one after another
    sims, _ = build()
    for s in sims:
        _abi.check(lib.bcg_sim_run(s, warmup), "warmup")
    torch.cuda.synchronize()
    c0 = cells_of(sims)
    t0 = time.perf_counter()
    for s in sims:
        _abi.check(lib.bcg_sim_run(s, steps), "sequential run")
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    work_seq = 0.5 * (c0 + cells_of(sims)) * steps
    for s in sims:
        lib.bcg_sim_destroy(s)
    return {"members": len(sizes), "cells_total": int(total), "cells_min": int(sizes.min()), "cells_max": int(sizes.max()),
            "steps": steps, "vcycles_per_step": args.vcycles,
            "ensemble_cell_steps_per_s": work_ens / t_ens, "sequential_cell_steps_per_s": work_seq / t_seq,
            "speedup": (work_ens / t_ens) / (work_seq / t_seq), "timing": "host wall clock, device synchronised"}


def output_step_bench(lib, sim, ctx, p, stream, steps=100):
    """One output step of the colony through the asynchronous writer (all of
    Cells, Restart, Density, Environment, AgarField, WallField in the
    reference's formats, under a temporary directory) while the simulation
    keeps stepping.  A first step, waited for, allocates the pinned staging;
    the second is timed: the simulation thread's time to queue both halves,
    the device time per step of the `steps` steps run while the host thread
    writes, and the time until the files are on disk."""
    import shutil
    import tempfile
    import torch
    from baccolonygrowth_b200 import _abi
    tmp = tempfile.mkdtemp(prefix="bcg_output_")
    res = {"steps_while_writing": steps}
    try:
        if shutil.disk_usage(tmp).free < 6 * 2 ** 30:
            return {"skipped": "less than 6 GiB free under %s" % tempfile.gettempdir()}
        threads = max(1, (os.cpu_count() or 2) - 1)
        w = ctypes.c_void_p()
        _abi.check(lib.bcg_writer_create(tmp.encode(), 0, threads, 2, ctypes.byref(w)), "bcg_writer_create")
        fcw = ctypes.c_int64()
        try:
            for rep in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                _abi.check(lib.bcg_output_cells(w, ctx, 0, 0.0, ctypes.byref(fcw)), "bcg_output_cells")
                _abi.check(lib.bcg_output_fields(w, ctx, 0, 0.0, p.dt), "bcg_output_fields")
                t1 = time.perf_counter()
                if rep == 0:
                    _abi.check(lib.bcg_writer_wait(w), "bcg_writer_wait")
                    res["first_step_s"] = time.perf_counter() - t0
                    continue
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                _abi.check(lib.bcg_sim_run(sim, steps), "steps while writing")
                e1.record(stream)
                torch.cuda.synchronize()
                t2 = time.perf_counter()
                _abi.check(lib.bcg_writer_wait(w), "bcg_writer_wait")
                t3 = time.perf_counter()
                res.update(queue_ms=(t1 - t0) * 1e3, ms_per_step_while_writing=e0.elapsed_time(e1) / steps,
                           steps_done_s=t2 - t0, write_s=t3 - t0)
        finally:
            lib.bcg_writer_destroy(w)
        nbytes = 0
        for root, _, files in os.walk(tmp):
            nbytes += sum(os.path.getsize(os.path.join(root, f)) for f in files)
        res.update(bytes=nbytes, write_gb_s=nbytes / res["write_s"] / 1e9, format_threads=threads)
        return res
    except Exception as e:      # reported, not required
        res["error"] = str(e)
        return res
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def source_digest(rel):
    import hashlib
    with open(os.path.join(ROOT, rel), "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()[:16]


def profiled_traffic(summary, workload):
    """DRAM bytes (read + write) of one launch from the committed ncu summary
    of the kernel (profiles/<summary>), and where they come from.  The
    summary records the digest of the kernel's source file at capture time
    (a line "- source: <file> sha256[:16] <digest>"); the bytes are used
    only when it was captured on this workload and the source is unchanged,
    else (None, reason)."""
    path = os.path.join(ROOT, "profiles", summary)
    try:
        text = open(path).read()
    except OSError:
        return None, "no ncu summary"
    if workload not in summary:
        return None, "no ncu summary of this workload"
    src = None
    for line in text.splitlines():
        if line.startswith("- source: "):
            f = line.split()
            src = (f[2], f[-1])
    if src is None:
        return None, "ncu summary without a source digest"
    try:
        if source_digest(src[0]) != src[1]:
            return None, "kernel source changed since the ncu capture in profiles/%s" % summary
    except OSError:
        return None, "kernel source file missing"
    unit = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    total = 0.0
    for key in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
        for line in text.splitlines():
            if line.startswith("- " + key + ":"):
                v, u = line.split(":", 1)[1].split()[:2]
                total += float(v) * unit.get(u, float("nan"))
                break
        else:
            return None, "ncu summary without DRAM bytes"
    return total, "ncu capture of one launch of the same source (profiles/%s), not this run" % summary


def timeline_summary(tags, ms):
    """Median phase ends of the steps whose seven marks (bcg_timeline_tag)
    all came back, in ms from each step's start; the period is the start
    of one step to the start of the next."""
    import numpy as np
    steps, cur = [], None
    for t, m in zip(tags, ms):
        if t == 1:
            cur = {}
            steps.append(cur)
        if cur is not None:
            cur[int(t)] = float(m)
    full = [s for s in steps if len(s) == 7]
    if not full:
        return None
    rel = lambda k: float(np.median([s[k] - s[1] for s in full]))
    periods = [steps[i + 1][1] - steps[i][1] for i in range(len(steps) - 1) if len(steps[i]) == 7]
    return {"steps": len(full), "solve_end_ms": rel(3), "move_grow_end_ms": rel(5), "divide_end_ms": rel(6),
            "step_end_ms": rel(7), "period_ms": float(np.median(periods)) if periods else None,
            "source": "bcg_timeline marks, median over the steps"}


def timeline_bench(lib, sim, ctx, steps):
    """`steps` steps of the bench schedule with the step timeline on."""
    import numpy as np
    from baccolonygrowth_b200 import _abi
    cap = 7 * steps + 8
    _abi.check(lib.bcg_timeline_enable(ctx, cap), "timeline")
    try:
        _abi.check(lib.bcg_sim_run(sim, steps), "timeline steps")
        tags = np.zeros(cap, dtype=np.int32)
        ms = np.zeros(cap, dtype=np.float32)
        n = ctypes.c_int()
        _abi.check(lib.bcg_timeline_read(ctx, _abi.ptr(tags, ctypes.c_int), _abi.ptr(ms, ctypes.c_float), cap,
                                         ctypes.byref(n)), "timeline read")
    finally:
        lib.bcg_timeline_enable(ctx, 0)
    return timeline_summary(tags[:n.value], ms[:n.value])


def sim_rebuilds(lib, sim):
    r = ctypes.c_int64()
    f = ctypes.c_int64()
    lib.bcg_sim_counters(sim, ctypes.byref(r), ctypes.byref(f))
    return int(r.value)


def apply_shapes(lib, ctx, tuned):
    """Give a new context the kernel shapes chosen for the bench colony
    (kernel choices belong to a context)."""
    from baccolonygrowth_b200 import _abi
    if tuned.get("relax_mode", -1) >= 0:
        _abi.check(lib.bcg_set_relax_mode(ctx, tuned["relax_mode"]), "set relax mode")
    if tuned.get("smoother", 0) > 0:
        _abi.check(lib.bcg_set_smoother_warps(ctx, tuned["smoother"]), "set smoother warps")
    if tuned.get("force_group", 0) > 0:
        _abi.check(lib.bcg_set_force_group(ctx, tuned["force_group"]), "set force group")


def mean_neighbours(lib, ctx):
    """Mean length of the reduced neighbour lists (the k of the per-pair work)."""
    import numpy as np
    from baccolonygrowth_b200 import _abi
    n = ctypes.c_int()
    lib.bcg_num_cells(ctx, ctypes.byref(n))
    counts = np.zeros(max(n.value, 1), dtype=np.int32)
    lists = np.zeros(max(n.value, 1), dtype=np.int32)
    _abi.check(lib.bcg_get_neighbours(ctx, _abi.ptr(counts, ctypes.c_int), _abi.ptr(lists, ctypes.c_int), 1),
               "bcg_get_neighbours")
    return float(counts[:n.value].mean()) if n.value else 0.0


def dense_mechanics_bench(lib, p, steps, warmup):
    """Mechanics alone (neighbour rebuild on its cadence, MoveCell/GrowCell,
    divisions; no agar solve) on a densely packed 1M-cell colony
    (colony.packed_colony: layers of touching cells, about 8 neighbours a
    cell), on the bench grid, timed like the main line."""
    import numpy as np
    import torch
    from baccolonygrowth_b200 import _abi, params as _params
    from baccolonygrowth_b200.colony import packed_colony
    out = {}
    try:
        n = 1048576
        w, h = _params.dome_size(n, 25.0 / 600.0, 0.9)
        cells = np.ascontiguousarray(packed_colony(n, w, h))
        sim = ctypes.c_void_p()
        _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(cells), n, 12345, 0, ctypes.byref(sim)), "dense sim")
        try:
            _abi.check(lib.bcg_sim_set_step_mode(sim, 0, 0), "dense mode")
            ctx = lib.bcg_sim_ctx(sim)
            g = np.full(p.box_x * p.box_z, 0.9)
            _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size), "g")
            _abi.check(lib.bcg_update_density(ctx), "density")
            _abi.check(lib.bcg_rebuild_neighbours(ctx), "rebuild")
            ch = ctypes.c_int()
            _abi.check(lib.bcg_autotune(ctx, _abi.TUNE["FORCE_GROUP"], ctypes.byref(ch)), "autotune")
            _abi.check(lib.bcg_sim_run(sim, warmup), "dense warmup")
            stream = torch.cuda.ExternalStream(lib.bcg_stream(ctx))
            rb0 = sim_rebuilds(lib, sim)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            _abi.check(lib.bcg_sim_run(sim, steps), "dense steps")
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            rb = time_rebuild(lib, ctx)
            every = steps_per_update(p)
            ms = ms - (sim_rebuilds(lib, sim) - rb0) * rb + steps * rb / every
            _abi.check(lib.bcg_enable_timers(ctx, 1), "timers")
            _abi.check(lib.bcg_sim_run(sim, min(steps, 10)), "dense timer steps")
            mg = ctypes.c_double(); nl = ctypes.c_int64()
            lib.bcg_get_timer(ctx, _abi.TIMERS["MOVE_GROW"], ctypes.byref(mg), ctypes.byref(nl))
            _abi.check(lib.bcg_enable_timers(ctx, 0), "timers off")
            k = mean_neighbours(lib, ctx)
            out.update(cells=n, mean_neighbours=k, force_group=ch.value, ms_per_step=ms / steps,
                       move_grow_ms=mg.value / min(steps, 10), rebuild_ms=rb,
                       cell_steps_per_s=n * steps / (ms / 1e3),
                       note="mechanics only: no agar solve in the step")
        finally:
            lib.bcg_sim_destroy(sim)
    except Exception as e:      # reported, not required
        out["error"] = str(e)
    return out


def time_rebuild(lib, ctx, reps=3):
    """Device time (ms) of one full neighbour rebuild (binning + lists) of
    the context's colony, the mean of `reps` (the lists do not change)."""
    from baccolonygrowth_b200 import _abi
    _abi.check(lib.bcg_rebuild_neighbours(ctx), "rebuild warm-up")
    _abi.check(lib.bcg_enable_timers(ctx, 1), "timers")
    for _ in range(reps):
        _abi.check(lib.bcg_rebuild_neighbours(ctx), "rebuild")
    ms = ctypes.c_double(); nl = ctypes.c_int64()
    lib.bcg_get_timer(ctx, _abi.TIMERS["NEIGHBOURS"], ctypes.byref(ms), ctypes.byref(nl))
    _abi.check(lib.bcg_enable_timers(ctx, 0), "timers off")
    return ms.value / reps


def field_update_bench(lib, ctx, p, timers, rebuild_ms, n_cells):
    """The reference's field update (Simulation.cpp:261-294) on the bench
    colony, each part timed on the device: the density chain
    (bcg_update_density), UpdateEnvArrayMG_OxygenAcetate at the reference's
    schedule (bcg_nutrient_update: n solves of 3 V-cycles + 200 colony/wall
    sweeps each, n = int(3600 UpdateTime 740 / 100)) and the full neighbour
    rebuild; the height update of every UpdateTime/10 beside it.  The step
    rate at the reference's cadence puts one update and 10 height updates
    over the UpdateTime/dt mechanics steps (MoveCell/GrowCell + divisions,
    no per-step solve) of one period."""
    from baccolonygrowth_b200 import _abi
    out = {}
    try:
        def timed(fn, tid):
            _abi.check(lib.bcg_enable_timers(ctx, 1), "timers")
            fn()
            ms = ctypes.c_double(); nl = ctypes.c_int64()
            lib.bcg_get_timer(ctx, _abi.TIMERS[tid], ctypes.byref(ms), ctypes.byref(nl))
            _abi.check(lib.bcg_enable_timers(ctx, 0), "timers off")
            return ms.value, int(nl.value)
        # capture both [solve + sweeps] graphs before timing
        _abi.check(lib.bcg_nutrient_update(ctx, 2, -1), "nutrient update warm-up")
        d_ms, _ = timed(lambda: _abi.check(lib.bcg_update_density(ctx), "density"), "DENSITY")
        n_ms, n_l = timed(lambda: _abi.check(lib.bcg_nutrient_update(ctx, 0, -1), "nutrient update"), "SWEEPS")
        h_ms, _ = timed(lambda: _abi.check(lib.bcg_update_height(ctx), "height"), "DENSITY")
        n_solves = nutrient_solves(p)
        upd = d_ms + n_ms + rebuild_ms
        S = steps_per_update(p)
        mech = timers["MOVE_GROW"] + timers["DIVIDE"]
        per_step = (S * mech + upd + (S / 10.0) * h_ms) / S
        out.update(solves_per_update=n_solves, sweeps_per_solve=p.sweeps_per_solve,
                   vcycles_per_solve=p.mg_vcycles, density_ms=d_ms, nutrient_ms=n_ms, rebuild_ms=rebuild_ms,
                   height_ms=h_ms, update_ms=upd, nutrient_launches=n_l,
                   steps_per_update=S, mechanics_ms_per_step=mech,
                   cell_steps_per_s=n_cells / (per_step / 1e3),
                   timing="CUDA events on the context's stream, one update")
    except Exception as e:      # reported, not required
        out["error"] = str(e)
    return out


def mg_level_points(p):
    """3 species x (nx+1)(nz+1) per multigrid level (mg_nx/mg_nz of the
    Multigrid constructor, Multigrid.cpp:5-33)."""
    A = p.max_levels_mg
    d0 = 1 << A
    pts = []
    for l in range(p.mg_levels):
        d = 1 << l
        nx = min(p.box_x * d0 // d // 2, p.box_x)
        nz = min(p.box_z_agar * d0 // d // 2, p.box_z_agar)
        pts.append(3 * (nx + 1) * (nz + 1))
    return pts


def mg_solve_bytes(p, vcycles):
    """Algorithmic DRAM bytes of one Multigrid::solve with `vcycles` V-cycles
    as the library runs it (FP64): per point and species, the fused
    3-sweep smoother reads R and E and writes E once (24 B) before and after
    the coarse correction; the restriction reads E and R (12 B: R is read
    on the even rows only) and writes 8 B per coarse point; the prolongation
    reads and writes E (16 B) and reads 8 B per coarse point; the coarsest
    level's relaxations run in shared memory (E and R in, E out).  Per
    solve: setup's residual (S in, R out: 16 B) and reset's update (S, E in,
    S out, E and R zeroed: 40 B) on the composite levels, zeroing (16 B) on
    the others."""
    pts = mg_level_points(p)
    A, L = p.max_levels_mg, len(pts)
    sweeps = max(1, (p.mg_mu1 + 2) // 3)     # fused launches per smoothing
    v = 0.0
    for l in range(L - 1):
        v += 2 * sweeps * 24.0 * pts[l]
        v += 12.0 * pts[l] + 8.0 * min(pts[l + 1], pts[l] // 4)
        v += 16.0 * pts[l] + 8.0 * min(pts[l + 1], pts[l] // 4)
    v += 24.0 * pts[L - 1]
    per_solve = sum(56.0 * pts[l] for l in range(A)) + sum(16.0 * pts[l] for l in range(A, L))
    return vcycles * v + per_solve


def colony_sweep_bench(lib, ctx, sweeps=200):
    """The colony sweeps of the nutrient update (UpdateEnvironment_OxygenAcetate
    and the wall rows, Multigrid.cpp:1017-1120) on the bench colony: points
    of the field chain's bounding box x sweeps per second, with 73 B per
    point-sweep (read C, W, A, O, DensityShiftP and the inside flag, write
    the four species) against the HBM peak.  Reported, not required."""
    from baccolonygrowth_b200 import _abi
    try:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _abi.check(lib.bcg_get_bbox(ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "bcg_get_bbox")
        pts = (b.value - a.value + 1) * (c.value + 1)
        _abi.check(lib.bcg_colony_sweeps(ctx, 2, 0), "sweep warm-up")
        _abi.check(lib.bcg_enable_timers(ctx, 1), "timers")
        _abi.check(lib.bcg_colony_sweeps(ctx, sweeps, 0), "sweeps")
        ms = ctypes.c_double(); nl = ctypes.c_int64()
        lib.bcg_get_timer(ctx, _abi.TIMERS["SWEEPS"], ctypes.byref(ms), ctypes.byref(nl))
        _abi.check(lib.bcg_enable_timers(ctx, 0), "timers off")
        rate = pts * sweeps / (ms.value / 1e3)
        peak, src = measured_peaks()
        return {"points_in_bbox": pts, "sweeps": sweeps, "ms_per_sweep": ms.value / sweeps,
                "point_sweeps_per_s": rate, "achieved_gb_s": 73.0 * rate / 1e9,
                "frac": 73.0 * rate / 1e9 / peak, "peak_source": src}
    except Exception as e:      # reported, not required
        return {"error": str(e)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU side: the reference's own code (oracle/_ref) or, where it is not built,
# the C restatement, on a bounded sample of the same workload
# ---------------------------------------------------------------------------
def cpu_model(pp, kind, threads):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import checkers
    if kind == "reference":
        return checkers.Reference(pp, seed=12345, threads=threads)
    return checkers.Oracle(pp, seed=12345)


def cpu_kind():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import checkers
    return "reference" if checkers.have_ref() else "port"


def cpu_run(p, cells, steps, threads, sample_cells=131072):
    """Time the CPU implementation on a bounded sample of the workload: the
    mechanics on a central x-window of `sample_cells` cells (per-cell cost
    does not depend on the colony size), the agar solve on the full grid.
    Returns per-step time for the whole workload (cells / mechanics rate +
    one 1-V-cycle solve + the neighbour rebuild amortised over 100 steps)."""
    import numpy as np
    from baccolonygrowth_b200 import _abi
    kind = cpu_kind()
    n = len(cells)
    m_cells = min(n, sample_cells)
    order = np.argsort(np.abs(0.5 * (cells["p"][:, 0] + cells["q"][:, 0])), kind="stable")
    sample = np.ascontiguousarray(cells[np.sort(order[:m_cells])])
    ps = p.copy()
    ps.max_cells = int(m_cells * 1.1) + 1024
    m = cpu_model(ps, kind, threads)
    m.load(sample)
    m.set_field(_abi.FIELDS["ENV_GROWTH1"], np.full(p.box_x * p.box_z, 0.9))
    t0 = time.perf_counter()
    m.rebuild()
    t_rebuild = time.perf_counter() - t0
    t = 0.0
    t0 = time.perf_counter()
    for s in range(steps):
        m.step(p.dt, t)
        t += p.dt
    t_mech = (time.perf_counter() - t0) / steps
    m.close()
    del m
    pg = p.copy()
    pg.max_cells = 4096
    g = cpu_model(pg, kind, threads)
    t0 = time.perf_counter()
    g.mg_solve(1, p.mg_dt)
    t_solve = time.perf_counter() - t0
    t0 = time.perf_counter()
    g.mg_solve(3, p.mg_dt)
    t_v = max((time.perf_counter() - t0 - t_solve) / 2.0, 1e-9)
    g.close()
    rate = m_cells / (t_mech + t_rebuild / 100.0)
    per_step = n / rate + t_solve
    return dict(kind=kind, threads=threads if kind == "reference" else 1, per_step=per_step,
                t_mech=t_mech, t_solve=t_solve, t_vcycle=t_v, cell_steps=n / per_step,
                t_rebuild_full=t_rebuild * n / m_cells, mech_cell_steps=rate,
                mg_dof_s=mg_dof(p) / t_v,
                sample="mechanics: %d of the %d cells (central x-window), %d steps + 1 full neighbour rebuild "
                       "(amortised over 100 steps); agar: Multigrid::solve with 1 and 3 V-cycles on the full "
                       "%dx%d composite grid; per step = cells/mechanics rate + one 1-V-cycle solve"
                       % (m_cells, n, steps, p.box_x + 1, p.box_z_agar + 1))


def cpu_field_update(p, cells, threads, mech=None):
    """The reference's field update (Simulation.cpp:261-294) on the CPU, on
    the full colony and grid: the density chain (GetDensity .. GetSurfaceNormal)
    and one outer iteration of UpdateEnvArrayMG_OxygenAcetate (one
    Multigrid::solve + 200 colony/wall sweeps) are timed; the update is the
    density chain + n outer iterations + the full neighbour rebuild (from the
    mechanics sample, scaled to the colony).  The per-step figure at the
    reference's cadence adds UpdateTime/dt mechanics steps and the
    UpdateTime/10 height updates."""
    import numpy as np
    kind = cpu_kind()
    pp = p.copy()
    pp.max_cells = len(cells) + 1024
    m = cpu_model(pp, kind, threads)
    m.load(np.ascontiguousarray(cells))
    t0 = time.perf_counter()
    m.update_density()
    t_density = time.perf_counter() - t0
    t0 = time.perf_counter()
    m.update_height()
    t_height = time.perf_counter() - t0
    t0 = time.perf_counter()
    m.nutrient_update(1)
    t_iter = time.perf_counter() - t0
    m.close()
    n_solves = nutrient_solves(p)
    out = {"kind": kind, "cores": threads if kind == "reference" else 1,
           "density_ms": t_density * 1e3, "height_ms": t_height * 1e3,
           "outer_iteration_ms": t_iter * 1e3, "solves_per_update": n_solves,
           "sample": "density chain + 1 of the %d outer iterations (Multigrid::solve, 3 V-cycles, + %d sweeps) "
                     "on the full colony and grid, scaled" % (n_solves, p.sweeps_per_solve)}
    if mech is not None:
        upd = t_density + n_solves * t_iter + mech["t_rebuild_full"]
        S = steps_per_update(p)
        per_step = (S * len(cells) / mech["mech_cell_steps"] + upd + (S / 10.0) * t_height) / S
        out.update(update_ms=upd * 1e3, cell_steps_per_s=len(cells) / per_step)
    return out


def nutrient_solves(p):
    """n of UpdateEnvArrayMG_OxygenAcetate: int(3600 UpdateTime 740 / 100)
    (Multigrid.cpp:995-996)."""
    return p.solves_per_update if p.solves_per_update > 0 else int(3600 * p.update_time * 740 / p.mg_dt)


def steps_per_update(p):
    return max(1, int(round(p.update_time / p.dt)))


def loaded_repo_libraries():
    """Shared libraries of this repository mapped into this process."""
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(ROOT):
                    libs.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(libs)


def reference_arm(args):
    """The reference's own CPU code on the same workload and metric.  The
    workload (parameters and colony) is built with the oracle's restatement
    of bcg_params_default / bcg_synth_colony, so this arm never loads the
    CUDA library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import checkers
    from baccolonygrowth_b200 import params
    from baccolonygrowth_b200.colony import workload_colony
    p = params.workload_params(args.workload, entries=checkers.oracle_param_entries())
    cells = workload_colony(args.workload, entry=checkers.oracle_synth_entry())
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, args.cpu_sample_steps))
    # warm-up sample (page-in), then the timed samples
    cpu_run(p, cells[:4096], 1, threads)
    r = cpu_run(p, cells, steps, threads)
    fu = None
    if not args.no_field_update:
        try:
            fu = cpu_field_update(p, cells, threads, mech=r)
        except Exception as e:      # reported, not required
            fu = {"error": str(e)}
    v = r["cell_steps"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["per_step"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "cells": len(cells), "box": [p.box_x, p.box_y, p.box_z],
                   "box_z_agar": p.box_z_agar, "agar_levels": p.max_levels_mg, "vcycles_per_step": 1,
                   "neighbour_rebuild_every": 100},
        "mg_dof_per_s": r["mg_dof_s"],
        "field_update": fu,
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": r["threads"], "kind": r["kind"],
                         "sample": r["sample"]},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "repo_libraries_loaded": loaded_repo_libraries(),
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def b200_arm(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from baccolonygrowth_b200 import _abi, params
    from baccolonygrowth_b200.colony import workload_colony
    lib = _abi.load()
    p = params.workload_params(args.workload)
    # replicas: every rank runs its own colony (different seed), no
    # data-path collective
    from baccolonygrowth_b200 import replicas as _rep
    cells = workload_colony(args.workload, seed=_rep.replica_seed(20261205, rank))
    n0 = len(cells)
    cells = np.ascontiguousarray(cells)
    pinned = torch.empty(cells.nbytes, dtype=torch.uint8, pin_memory=True)
    hostbuf = pinned.numpy().view(_abi.CELL_DTYPE)
    hostbuf[:] = cells

    def make_sim():
        sim = ctypes.c_void_p()
        _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(hostbuf), n0, 12345 + rank, 0, ctypes.byref(sim)), "bcg_sim_create")
        _abi.check(lib.bcg_sim_set_step_mode(sim, 0, args.vcycles), "bcg_sim_set_step_mode")
        ctx = lib.bcg_sim_ctx(sim)
        # growth field of a colony in steady nutrient supply (no field update
        # runs inside the timed steps)
        g = np.full(p.box_x * p.box_z, 0.9)
        _abi.check(lib.bcg_set_field(ctx, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size), "set growth")
        _abi.check(lib.bcg_update_density(ctx), "bcg_update_density")
        rows = set_depleted_wall(lib, ctx, p)
        # kernel shapes for this colony and grid (project autotuner)
        _abi.check(lib.bcg_rebuild_neighbours(ctx), "rebuild")
        tuned = {}
        if args.relax_mode >= 0:
            _abi.check(lib.bcg_set_relax_mode(ctx, args.relax_mode), "set relax mode")
            tuned["relax_mode"] = args.relax_mode
        for name in ("SMOOTHER", "FORCE_GROUP"):
            if name == "SMOOTHER" and args.smoother_warps > 0:
                _abi.check(lib.bcg_set_smoother_warps(ctx, args.smoother_warps), "set smoother warps")
                tuned["smoother"] = args.smoother_warps
                continue
            if name == "FORCE_GROUP" and args.force_group > 0:
                _abi.check(lib.bcg_set_force_group(ctx, args.force_group), "set force group")
                tuned["force_group"] = args.force_group
                continue
            ch = ctypes.c_int()
            _abi.check(lib.bcg_autotune(ctx, _abi.TUNE[name], ctypes.byref(ch)), "autotune " + name)
            tuned[name.lower()] = ch.value
            if name == "SMOOTHER":
                ms_s = ctypes.c_double()
                lib.bcg_smoother_launch_ms(ctx, ctypes.byref(ms_s))
                tuned["smoother_launch_ms"] = ms_s.value
        return sim, ctx, rows, tuned

    sim, ctx, wall_rows, tuned = make_sim()
    stream = torch.cuda.ExternalStream(lib.bcg_stream(ctx))
    _abi.check(lib.bcg_sim_run(sim, args.warmup), "warmup")
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    rb0 = sim_rebuilds(lib, sim)
    launches0 = int(lib.bcg_kernel_launches(ctx))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    _abi.check(lib.bcg_sim_run(sim, args.steps), "timed steps")
    e1.record(stream)
    torch.cuda.synchronize()
    launches = int(lib.bcg_kernel_launches(ctx)) - launches0
    clocks = sampler.stop()
    rebuilds_timed = sim_rebuilds(lib, sim) - rb0
    ms_raw = e0.elapsed_time(e1)
    # the full neighbour rebuild runs every UpdateTime/dt steps (100): take
    # the rebuilds that fell inside the timed steps out and put 1/100 of one
    # timed rebuild into every step, so that the figure does not depend on
    # where --steps falls in the rebuild period
    rebuild_ms = time_rebuild(lib, ctx)
    every = steps_per_update(p)
    ms = ms_raw - rebuilds_timed * rebuild_ms + args.steps * rebuild_ms / every
    t_ = ctypes.c_double(); n_ = ctypes.c_int(); d_ = ctypes.c_int64()
    lib.bcg_sim_time(sim, ctypes.byref(t_), ctypes.byref(n_), ctypes.byref(d_))
    n_end = n_.value
    cells_mean = 0.5 * (n0 + n_end)

    # per-kernel device time of the same schedule with timers on (separate run,
    # so the event syncs of the timers do not enter the timed region above)
    _abi.check(lib.bcg_enable_timers(ctx, 1), "timers")
    kt_steps = min(20, args.steps)
    _abi.check(lib.bcg_sim_run(sim, kt_steps), "timer steps")
    timers = {}
    for name, tid in _abi.TIMERS.items():
        msx = ctypes.c_double(); nl = ctypes.c_int64()
        lib.bcg_get_timer(ctx, tid, ctypes.byref(msx), ctypes.byref(nl))
        timers[name] = msx.value / kt_steps
    _abi.check(lib.bcg_enable_timers(ctx, 0), "timers off")
    # the same schedule with its phases marked by CUDA events on the stream
    # each phase runs on (bcg_timeline_*), which do not synchronise: where
    # the overlapped step's time goes
    try:
        step_timeline = timeline_bench(lib, sim, ctx, 10)
    except Exception as e:      # reported, not required
        step_timeline = {"error": str(e)}
    # MoveCell + GrowCell with the contact search in FP32 (the precision
    # form), same schedule, device time per step against the FP64 search
    pair32 = None
    try:
        _abi.check(lib.bcg_set_pair_precision(ctx, 32), "pair precision 32")
        _abi.check(lib.bcg_enable_timers(ctx, 1), "timers")
        _abi.check(lib.bcg_sim_run(sim, kt_steps), "fp32 search steps")
        msx = ctypes.c_double(); nl = ctypes.c_int64()
        lib.bcg_get_timer(ctx, _abi.TIMERS["MOVE_GROW"], ctypes.byref(msx), ctypes.byref(nl))
        _abi.check(lib.bcg_enable_timers(ctx, 0), "timers off")
        _abi.check(lib.bcg_set_pair_precision(ctx, 64), "pair precision 64")
        pair32 = {"move_grow_ms_fp64_search": timers["MOVE_GROW"], "move_grow_ms_fp32_search": msx.value / kt_steps,
                  "speedup": timers["MOVE_GROW"] / (msx.value / kt_steps) if msx.value > 0 else None,
                  "accuracy": "branch found in FP32, closest points and forces in FP64; tests/test_gpu_mechanics.py "
                              "holds 1e-10 against the oracle"}
    except Exception as e:      # reported, not required
        pair32 = {"error": str(e)}
    k_mean_measured = mean_neighbours(lib, ctx)
    n_now = ctypes.c_int()
    lib.bcg_num_cells(ctx, ctypes.byref(n_now))
    colony = colony_sweep_bench(lib, ctx) if world == 1 else None
    field_update = None
    if world == 1 and not args.no_field_update:
        field_update = field_update_bench(lib, ctx, p, timers, rebuild_ms, n_now.value)
    lib.bcg_sim_destroy(sim)

    # end to end through the C ABI with host buffers: upload of the colony
    # from pinned host memory, the steps (each reads two counters back and
    # uploads the division draws), download of the final colony
    # one untimed pass (2 steps) first: first-touch costs of a new context
    for e2e_pass, e2e_steps in ((0, 2), (1, args.steps)):
        sim2 = ctypes.c_void_p()
        _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(hostbuf), 0, 12345 + rank, 0, ctypes.byref(sim2)), "sim2")
        _abi.check(lib.bcg_sim_set_step_mode(sim2, 0, args.vcycles), "mode2")
        ctx2 = lib.bcg_sim_ctx(sim2)
        apply_shapes(lib, ctx2, tuned)
        g = np.full(p.box_x * p.box_z, 0.9)
        lib.bcg_set_field(ctx2, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size)
        out_pinned = torch.empty((n0 + n0 // 4) * 208, dtype=torch.uint8, pin_memory=True)
        outbuf = out_pinned.numpy().view(_abi.CELL_DTYPE)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        _abi.check(lib.bcg_upload_cells(ctx2, _abi.ptr(hostbuf), n0), "upload")
        _abi.check(lib.bcg_update_density(ctx2), "density")
        set_depleted_wall(lib, ctx2, p, wall_rows)
        _abi.check(lib.bcg_sim_run(sim2, e2e_steps), "e2e steps")
        got = ctypes.c_int()
        _abi.check(lib.bcg_download_cells(ctx2, _abi.ptr(outbuf), len(outbuf), ctypes.byref(got)), "download")
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - w0
        e2e_s += (e2e_steps / every - sim_rebuilds(lib, sim2)) * rebuild_ms / 1e3
        t2 = ctypes.c_double(); n2 = ctypes.c_int(); d2 = ctypes.c_int64()
        lib.bcg_sim_time(sim2, ctypes.byref(t2), ctypes.byref(n2), ctypes.byref(d2))
        lib.bcg_sim_destroy(sim2)
        h2d = (n0 * 208 + 3 * 8 * p.box_x + 9 * 4 * d2.value) / e2e_steps
        d2h = (got.value * 208 + 16 * e2e_steps + 8 * d2.value) / e2e_steps
        e2e_value = 0.5 * (n0 + got.value) * e2e_steps / e2e_s

    # the agar solve to a 1e-8 relative defect: plain FP64 V-cycles vs FP32
    # V-cycles with FP64 defect checks and FP64 refinement, from the same state
    mg_tol = None
    if not args.no_mg_tol:
        from baccolonygrowth_b200.colony import Colony
        res = {}
        sols = {}
        for prec in (64, 32):
            col = Colony(p, cells)
            col.update_density()
            col.deplete_wall()
            col.mg_solve_tol(1e-8, prec, 2)        # warm-up (pages in)
            col.close()
            col = Colony(p, cells)
            col.update_density()
            col.deplete_wall()
            col.enable_timers(True)
            it, rel = col.mg_solve_tol(1e-8, prec, 100)
            msx, _ = col.timer("MG_SOLVE")
            res["fp64" if prec == 64 else "mixed"] = {"iters": it, "ms": msx, "rel_defect": rel}
            sols[prec] = [col.field("MG_SOL_" + sp, 0) for sp in ("CARBON", "OXYGEN", "ACETATE")]
            col.close()
        diff = max(float(np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)) for a, b in zip(sols[64], sols[32]))
        mg_tol = {"rel_tol": 1e-8, "fp64": res["fp64"], "mixed": res["mixed"],
                  "speedup": res["fp64"]["ms"] / res["mixed"]["ms"] if res["mixed"]["ms"] > 0 else None,
                  "max_rel_diff_level0": diff, "dof": mg_dof(p)}

    # ensemble of independent colonies (log-uniform 1k-100k cells, each on a
    # grid sized to it), stepped together vs one after another
    ens = None
    if not args.no_ensemble and world == 1:
        ens = ensemble_bench(lib, args)

    dense = None
    if world == 1 and not args.no_dense:
        dense = dense_mechanics_bench(lib, p, min(args.steps, 20), args.warmup)

    # an output step through the asynchronous writer, last so that its
    # file traffic does not disturb the measurements above
    out_step = None
    if not args.no_output and world == 1:
        sim3 = ctypes.c_void_p()
        _abi.check(lib.bcg_sim_create(ctypes.byref(p), _abi.ptr(hostbuf), n0, 12345 + rank, 0, ctypes.byref(sim3)), "sim3")
        _abi.check(lib.bcg_sim_set_step_mode(sim3, 0, args.vcycles), "mode3")
        ctx3 = lib.bcg_sim_ctx(sim3)
        apply_shapes(lib, ctx3, tuned)
        g = np.full(p.box_x * p.box_z, 0.9)
        lib.bcg_set_field(ctx3, _abi.FIELDS["ENV_GROWTH1"], 0, _abi.ptr(g, ctypes.c_double), g.size)
        _abi.check(lib.bcg_update_density(ctx3), "density3")
        set_depleted_wall(lib, ctx3, p, wall_rows)
        _abi.check(lib.bcg_sim_run(sim3, 2), "warmup3")
        out_step = output_step_bench(lib, sim3, ctx3, p, torch.cuda.ExternalStream(lib.bcg_stream(ctx3)))
        lib.bcg_sim_destroy(sim3)

    # max over ranks (time) and sum over ranks (work); no other collective
    from baccolonygrowth_b200 import replicas
    (ms_max, e2e_max), (work, work_e2e) = replicas.aggregate(
        [ms, e2e_s], [cells_mean * args.steps, 0.5 * (n0 + got.value) * args.steps],
        device="cuda" if world > 1 else "cpu")

    value = work / (ms_max / 1e3)
    e2e_value = work_e2e / e2e_max

    # roofline of the dominant kernel group
    peak_gbs, peak_src = measured_peaks()
    dof = mg_dof(p)
    mg_ms = timers["MG_SOLVE"]
    mech_ms = timers["MOVE_GROW"]
    mg_bytes = mg_solve_bytes(p, args.vcycles)
    mech_bytes = (280.0 + 4.0 * k_mean_measured) * cells_mean
    mg_gbs = mg_bytes / (mg_ms / 1e3) / 1e9 if mg_ms > 0 else 0.0
    mech_gbs = mech_bytes / (mech_ms / 1e3) / 1e9 if mech_ms > 0 else 0.0
    roof_mg = {"kernel": "multigrid solve (Multigrid::solve, %d V-cycle)" % args.vcycles, "bound": "hbm",
               "achieved": mg_gbs, "peak": peak_gbs, "unit": "GB/s", "frac": mg_gbs / peak_gbs,
               "traffic": None, "peak_source": peak_src, "algorithmic_bytes_per_launch": mg_bytes,
               "launch_ms": mg_ms,
               "bytes_model": "per point and species: fused 3-sweep smoothing 24 B before and after, "
                              "restriction 12 B + 8 B per coarse point written, prolongation 16 B + 8 B per "
                              "coarse point read, on every level; setup's residual 16 B and reset's update "
                              "40 B on the composite levels, zeroing 16 B on the others"}
    # the dominant single kernel: the fused 3-sweep smoother on a finest
    # composite level, 24 B per point and species (R and E read, E2
    # written), timed with CUDA events by the autotuner
    sm_ms = tuned.get("smoother_launch_ms", 0.0)
    lvl0_pts = 3 * (p.box_x + 1) * (p.box_z_agar + 1)
    sm_bytes = 24.0 * lvl0_pts
    if mg_ms >= mech_ms and sm_ms > 0:
        sm_gbs = sm_bytes / (sm_ms / 1e3) / 1e9
        # the smoother form in use (bcg_set_relax_mode; the library's default is 3)
        tma = tuned.get("relax_mode", 3) == 3
        kname = "k_mg_smooth_tma" if tma else "k_mg_smooth"
        traffic, traffic_src = profiled_traffic(kname + "_" + args.workload + ".md", args.workload)
        roof = {"kernel": kname + "<double,3> (finest agar level, 3 fused zebra sweeps)", "bound": "hbm",
                "achieved": sm_gbs, "peak": peak_gbs, "unit": "GB/s", "frac": sm_gbs / peak_gbs,
                "traffic": traffic, "traffic_source": traffic_src,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": sm_bytes,
                "launch_ms": sm_ms, "unit_work": "%d points x 3 species, 24 B each" % (lvl0_pts // 3)}
    elif mg_ms >= mech_ms:
        roof = roof_mg
    else:
        roof = {"kernel": "k_move_grow (MoveCell+GrowCell)", "bound": "hbm", "achieved": mech_gbs,
                "peak": peak_gbs, "unit": "GB/s", "frac": mech_gbs / peak_gbs, "traffic": None,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": mech_bytes, "launch_ms": mech_ms}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            r = cpu_run(p, cells, args.cpu_sample_steps, os.cpu_count() or 1)
            cpu = {"value": r["cell_steps"], "unit": "cell-steps/s", "cores": r["threads"], "kind": r["kind"],
                   "sample": r["sample"], "mg_dof_per_s": r["mg_dof_s"]}
            if field_update is not None:
                try:
                    field_update["cpu"] = cpu_field_update(p, cells, os.cpu_count() or 1, mech=r)
                except Exception as e:      # reported, not required
                    field_update["cpu"] = {"error": str(e)}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "cell-steps/s", "cores": 0, "kind": "port", "sample": "failed: %s" % e}
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "cells": n0, "cells_end": n_end,
                   "box": [p.box_x, p.box_y, p.box_z], "box_z_agar": p.box_z_agar,
                   "agar_levels": p.max_levels_mg, "mg_levels": p.mg_levels, "mg_dof": dof,
                   "vcycles_per_step": args.vcycles, "neighbour_rebuild_every": every,
                   "neighbour_rebuild": {"ms": rebuild_ms, "in_timed_steps": rebuilds_timed,
                                         "accounting": "timed steps minus the rebuilds inside them, "
                                                       "plus 1/%d of one rebuild per step" % every},
                   "autotuned": tuned,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (cell records 2x%d MB + fields)" % (n0 * 128 // 2 ** 20)},
        "mg_dof_per_s": dof * args.vcycles / (mg_ms / 1e3) if mg_ms > 0 else None,
        "mg_tolerance_solve": mg_tol,
        "ensemble": ens,
        "output_step": out_step,
        "colony_sweeps": colony,
        "field_update": field_update,
        "pair_geometry_fp32": pair32,
        "mean_neighbours": k_mean_measured,
        "dense_mechanics": dense,
        "kernel_ms_per_step": timers,
        "step_timeline": step_timeline,
        "divisions": d_.value,
        "roofline": roof,
        "roofline_mg_solve": roof_mg,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    a = parse()
    sys.exit(reference_arm(a) if a.impl == "reference" else b200_arm(a))
