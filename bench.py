"""Benchmark of the cell-mechanics step on B200.

Default workload (N=1): the batched ensemble of 512 independent synthetic
tissues (membrane side in {16,24,32,48,64}, 2-8 jittered cell layers, per-tissue
spring / LJ / bending constants scaled log-uniform in [0.5, 2]), FP32 forces
with FP64 sums and positions, one CUDA graph replaying the whole batch per
step. A step is one full mechanics step of every tissue: interaction + commit +
periodic wrap + re-binning + neighbour lists (the reference's cell_dynamics
without cell_state_renew). value = particles (membrane + mobile, all tissues,
all ranks) x steps / device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ensemble|c2|c3|c1] [--precision mixed|fp64]

Under torchrun (N > 1) the ensemble scales weakly: the job is N x 512
tissues of the same generator (the first 512 are the 1-GPU batch), balanced
over the ranks so each holds about 512, with no collective on the data path;
the timed region is bracketed by barriers and the max over ranks is
reported. A single-tissue workload (c1-c3) runs as N replicas, one per
rank (one tissue is not split).

--impl reference times the reference's own CPU implementation (epi5_MT built
by oracle/build_ref.py, OpenMP TBB stand-in, all host threads) on a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from epi_b200 import tissue as T  # noqa: E402
from epi_b200.ensemble import shard_tissues  # noqa: E402

METRIC = "cell-updates/s: FP32/batched vs plain FP64 GPU @≤1e-5 rel pos err; grad err"
UNIT = "cell-updates/s"


def workload(name: str, tissues: int = 512):
    if name == "ensemble":
        if tissues != 512:
            return (T.config4()[:tissues],
                    f"first {tissues} tissues of the batched ensemble (config 4)")
        return T.config4(), "batched ensemble: 512 tissues, side {16..64}, 2-8 layers (config 4)"
    if name == "tri_ensemble":
        return (T.config4_tri()[:tissues],
                f"batched ensemble of {tissues} tissues with triangular membranes (config 4 "
                f"shapes, TRI_MEMB)")
    if name == "c2":
        return [T.config2()], "single tissue 64x64 membrane + 32,768 cells (config 2)"
    if name == "c3":
        return [T.config3()], "single tissue 256x256 membrane + 1,048,576 cells (config 3)"
    if name == "c1":
        return [T.config1()], "single tissue 16x16 membrane + 512 cells (config 1)"
    raise SystemExit(f"unknown workload {name}")


def rank_workload(name: str, tissues: int, world: int, rank: int):
    """This rank's tissues of the job: (mine, particles of the whole job,
    tissues of the whole job, description, the whole tissue list or None).

    Ensemble, N > 1: weak scaling. The job is N x `tissues` tissues of the
    same generator (the first `tissues` are the 1-GPU batch), balanced over
    the ranks by shard_tissues; each rank generates only its own. Single
    tissue, N > 1: one replica per rank. N = 1: the workload itself."""
    if name == "ensemble" and world > 1:
        nt = tissues * world
        specs = T.config4_specs(n_tissues=nt)
        sizes = [side * side * (1 + layers) for side, layers, _ in specs]
        shards = shard_tissues(sizes, world)
        mine = T.config4(n_tissues=nt, indices=shards[rank])
        desc = (f"batched ensemble, {tissues} tissues per GPU: {nt} tissues, "
                f"side {{16..64}}, 2-8 layers (config 4)")
        return mine, sum(sizes), nt, desc, None
    every, desc = workload(name, tissues)
    if world > 1:
        return (every, world * sum(t.n for t in every), world * len(every),
                f"{desc}, one replica per GPU", every)
    return every, sum(t.n for t in every), len(every), desc, every


def rank_tissue_ids(name: str, tissues: int, world: int, rank: int):
    """Job ids of this rank's tissues, in the order rank_workload returns
    them: the ensemble's shard, or the rank's own replica of a single-tissue
    workload (job id = rank; the replicas are ordered by rank)."""
    if name == "ensemble" and world > 1:
        specs = T.config4_specs(n_tissues=tissues * world)
        sizes = [side * side * (1 + layers) for side, layers, _ in specs]
        return shard_tissues(sizes, world)[rank]
    if world > 1:
        return [rank]
    every, _ = workload(name, tissues)
    return list(range(len(every)))


def gather_positions(ctx, mine, ids, dist):
    """The job's final positions on rank 0 in job order (bench.py's result
    gather, after the timed region): (tissues, particles, checksum) there,
    None elsewhere. Single-tissue replicas count once per rank."""
    from epi_b200.ensemble import gather_results, split_by_tissue
    per = split_by_tissue(ctx.positions(), [t.n for t in mine])
    if dist is None:
        allr = per
    else:
        allr = gather_results(ids if len(ids) == len(per) else list(range(len(per))), per, dist)
    if allr is None:
        return None
    total = sum(len(r[0]) for r in allr)
    checksum = float(sum(np.sum(a) for r in allr for a in r))
    return {"tissues": len(allr), "particles": total, "sum_of_coordinates": checksum,
            "order": "job order (tissue ids of the whole job)"}


# --------------------------------------------------------------------------
# clocks during the timed region (NVML)
# --------------------------------------------------------------------------
class ClockSampler:
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int, period: float = 0.02):
        self.samples = []
        self.reasons = 0
        self.period = period
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None

    def _sample(self):
        nv = self._nv
        self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
        try:
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        except Exception:
            r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
        self.reasons |= int(r) & ~0x1

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self._t.join()
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "samples": len(self.samples),
                "reasons": [n for b, n in self.REASONS.items() if self.reasons & b]}


# --------------------------------------------------------------------------
# CPU baseline / reference arm: compiled epi5_MT (OpenMP) on a sample
# --------------------------------------------------------------------------
def reference_sample(tissues, target_particles: int):
    """Deterministic bounded sample: every k-th tissue, k = total / target."""
    total = sum(t.n for t in tissues)
    step = max(1, total // max(target_particles, 1))
    return list(tissues[::step])


def time_reference_cpu(tissues, warmup: int, steps: int, threads=None):
    """Runs the compiled reference on each sampled tissue; returns
    (cell-updates/s over the sample, details). The sample is advanced
    `steps` timed steps; time per step = sum over tissues of the median."""
    from oracle import oracle as O
    per = []
    for t in tissues:
        r = O.time_reference(t, warmup, steps, threads)
        per.append((t.n, r["median_s"], r["threads"]))
    cells = sum(n for n, _, _ in per)
    sec = sum(s for _, s, _ in per)
    return cells / sec, dict(tissues=len(per), particles=cells, step_s=sec,
                             threads=per[0][2] if per else 0)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tissues, desc = workload(args.workload, args.tissues)
    sample = reference_sample(tissues, args.ref_particles)
    try:
        v, d = time_reference_cpu(sample, max(1, args.warmup), max(1, args.steps))
    except FileNotFoundError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return 0
    sample_desc = (f"{d['tissues']} of {len(tissues)} tissues ({d['particles']} particles), "
                   f"median of {max(1, args.steps)} steps each after {max(1, args.warmup)} warm-up")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * d["step_s"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "sample": sample_desc},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": d["threads"], "kind": "reference",
                         "sample": sample_desc},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def load_traffic(kernel: str, workload_name: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(workload_name, {}).get(kernel)
    except Exception:
        return None


def min_image_err(t, a, b):
    """max over particles of the minimum-image |a - b| / L_x."""
    d = [a[k] - b[k] for k in range(3)]
    for k, L in ((0, t.lx), (1, t.ly)):
        d[k] = np.where(d[k] > 0.5 * L, d[k] - L, np.where(d[k] <= -0.5 * L, d[k] + L, d[k]))
    return float(np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2).max() / t.lx)


def mean_sq_loss(t, pos, target):
    d = [pos[k] - target[k] for k in range(3)]
    for k, L in ((0, t.lx), (1, t.ly)):
        d[k] = np.where(d[k] > 0.5 * L, d[k] - L, np.where(d[k] <= -0.5 * L, d[k] + L, d[k]))
    m = slice(t.nmemb, t.n)
    return float(np.mean(d[0][m] ** 2 + d[1][m] ** 2 + d[2][m] ** 2))


def accuracy_check(capi, device: int, steps: int):
    """Mixed (FP32 forces) against FP64 positions on the 64x64, 32,768-cell
    tissue after `steps` steps (the FP64 path is pinned to the oracle by the
    parity tests)."""
    t = T.config2()
    pos = {}
    for name, prec in (("fp64", capi.EPI_PREC_FP64), ("mixed", capi.EPI_PREC_MIXED)):
        with capi.Context(precision=prec, device=device) as c:
            c.upload([t])
            c.step(steps, "graph")
            pos[name] = c.positions()
    return {"workload": "64x64 membrane + 32,768 cells (seed 1)", "steps": steps,
            "max_rel_pos_err_mixed_vs_fp64": min_image_err(t, pos["mixed"], pos["fp64"]),
            "bar": 1e-5}


def adjoint_check(capi, device: int, steps: int, every: int = 20, h: float = 1e-4):
    """The adjoint workload: 64x64 membrane + 32,768 cells, loss = mean squared
    distance of the final cell positions to a run with every force constant
    +10%; gradient w.r.t. the spring / LJ-epsilon / bending multipliers by
    epi_adjoint (FP64, checkpoint every `every` steps), against central
    differences of the FP64 step (h relative)."""
    import torch
    t = T.config5()

    def run(params):
        with capi.Context(precision=capi.EPI_PREC_FP64, device=device) as c:
            c.upload([t], [params])
            c.step(steps, "graph")
            return c.positions()

    target = run(t.params.scaled(1.1, 1.1, 1.1))
    with capi.Context(precision=capi.EPI_PREC_FP64, device=device) as c:
        c.upload([t])
        c.adjoint(steps, target, checkpoint_every=every)  # warm-up
        c.upload([t])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss, grad = c.adjoint(steps, target, checkpoint_every=every)
        adj_s = time.perf_counter() - t0
    fd = []
    for k in range(3):
        e = [1.0, 1.0, 1.0]
        e[k] = 1.0 + h
        lp = mean_sq_loss(t, run(t.params.scaled(*e)), target)
        e[k] = 1.0 - h
        lm = mean_sq_loss(t, run(t.params.scaled(*e)), target)
        fd.append((lp - lm) / (2 * h))
    rel = [abs(grad[0, k] - fd[k]) / abs(fd[k]) for k in range(3)]
    return {"workload": "64x64 membrane + 32,768 cells (seed 4), target from +10% constants",
            "steps": steps, "checkpoint_every": every, "loss": float(loss[0]),
            "grad": [float(g) for g in grad[0]], "fd": fd, "fd_h": h,
            "max_rel_err_vs_fd": max(rel), "bar": 1e-4, "seconds": adj_s,
            "grad_order": ["s_spring", "s_eps", "s_bend"]}


def field_check(capi, device: int, steps: int, with_cpu: bool):
    """The field part of the reference's step (zzmax, cell maps, external-
    stimulus update; epi_field_step) on the 64x64, 32,768-cell tissue with a
    129 x 129 x 65 grid (the reference's 0.5 spacing), timed with CUDA events;
    beside it the reference's own OpenMP build on the same tissue."""
    import torch
    t = T.config2()
    grid = (128, 128, 64)
    with capi.Context(precision=capi.EPI_PREC_MIXED, device=device) as c:
        c.upload([t])
        c.field_init(*grid)
        c.field_step(3)
        s = torch.cuda.ExternalStream(c.stream_handle())
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        c.field_step(steps)
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
    out = {"workload": "64x64 membrane + 32,768 cells, grid 129 x 129 x 65",
           "gpu_ms_per_step": ms, "steps": steps}
    if with_cpu:
        try:
            from oracle import oracle as O
            d = O.time_reference_field(t, 2, 5, threads=os.cpu_count())
            out["cpu_reference_ms_per_step"] = d["median_s"] * 1e3
            out["cpu_cores"] = d["threads"]
            out["speedup_vs_cpu_reference"] = d["median_s"] * 1e3 / ms
        except Exception as e:  # reference build missing on this host
            out["cpu_reference"] = f"unavailable: {e}"
    return out


def dropin_check(workloads, steps: int, warmup: int):
    """The drop-in inside the reference's own step loop: epi5_MT's harness
    (cell_interaction -> pos_copy -> cell_pos_periodic_fix -> connect_cell,
    proc.cpp:22-32) built with epi_b200/shim in place of its two mechanics
    files, against the same harness built with the reference's own mechanics;
    both OpenMP builds on all host threads, steady_clock median per step. The
    drop-in's step includes every host<->device copy and the write-back of
    connected_cell, the gap-junction maps and dermis."""
    from oracle import oracle as O
    out = {}
    for name, t in workloads:
        try:
            ref = O.time_reference(t, warmup, steps, threads=os.cpu_count())
            gpu = O.time_reference(t, warmup, steps, threads=os.cpu_count(),
                                   variant="dropin_omp")
            out[name] = {"particles": t.n, "steps": steps, "warmup": warmup,
                         "reference_ms_per_step": ref["median_s"] * 1e3,
                         "dropin_ms_per_step": gpu["median_s"] * 1e3,
                         "host_threads": ref["threads"],
                         "speedup": ref["median_s"] / gpu["median_s"]}
        except Exception as e:  # harness builds missing on this host
            out[name] = {"unavailable": str(e)[:200]}
    return out


def cfg_skin(tuned, args):
    """The candidate skin the headline run used."""
    if tuned:
        return tuned["skin"]
    return args.skin if args.skin is not None else 0.1


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ensemble",
                    choices=["ensemble", "tri_ensemble", "c1", "c2", "c3"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--skin", type=float, default=None,
                    help="candidate skin (default: chosen by the autotuner)")
    ap.add_argument("--tissues", type=int, default=512, help="ensemble size (profiling)")
    ap.add_argument("--variant", type=int, default=None, help="step-kernel tuning variant")
    ap.add_argument("--mode", default="graph", choices=["graph", "eager"])
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default skin / variant instead of epi_autotune's choice")
    ap.add_argument("--tune-steps", type=int, default=128, help="timed steps per autotuner trial")
    ap.add_argument("--retune", action="store_true",
                    help="run the autotuner even when its choice for this batch is cached")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--fp64-batched-steps", type=int, default=None,
                    help="timed steps of the FP64-forces batched run (default: --steps; 0: skip)")
    ap.add_argument("--ref-particles", type=int, default=120000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="timed region only (profiling)")
    ap.add_argument("--adjoint-steps", type=int, default=200,
                    help="steps of the adjoint workload (0: skip)")
    ap.add_argument("--field-steps", type=int, default=50,
                    help="timed steps of the cell-map / stimulus part (0: skip)")
    ap.add_argument("--dropin-steps", type=int, default=10,
                    help="timed steps of the drop-in inside the reference's loop (0: skip)")
    ap.add_argument("--dropin-c3", action="store_true",
                    help="also time the drop-in on the 1.1M-particle tissue")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 position error check (0: skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)
    if args.fp64_batched_steps is None:
        args.fp64_batched_steps = args.steps

    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    from epi_b200 import capi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    mine, n_all, n_tissues_all, desc, tissues = rank_workload(args.workload, args.tissues,
                                                               world, rank)
    n_mine = sum(t.n for t in mine)
    prec = capi.EPI_PREC_MIXED if args.precision == "mixed" else capi.EPI_PREC_FP64

    ctx = capi.Context(precision=prec, max_conn=64, device=local, skin=args.skin,
                       variant=args.variant)
    ctx.upload(mine)
    tuned = None
    if args.skin is None and args.variant is None and not args.no_autotune:
        # tune on the state the timed region starts from (after the warm-up's
        # relaxation of the jittered start), then warm up again below; a
        # choice cached for this batch shape is reused (epi_b200/autotune.py)
        if args.warmup:
            ctx.step(args.warmup, args.mode)
        from epi_b200.autotune import tuned as autotuned
        tuned = autotuned(ctx, mine, args.tune_steps, device=local, retune=args.retune)
        tuned["grid"] = ("skin {0.05,0.08,0.1,0.15,0.2,0.3} x step-kernel variant 1..4, "
                         "then rebuild node {conditional, always launched}, "
                         "then search switch {8192,16384,49152,131072}")
    off, _ = ctx.connections()
    kbar = float(off[-1]) / max(n_mine, 1)  # mean connected_cell length incl. lattice links
    nmemb_mine = sum(t.nmemb for t in mine)
    kbar_searched = (float(off[-1]) - 4 * nmemb_mine) / max(n_mine, 1)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    def barrier():
        if dist is not None:
            dist.barrier()

    # the positions the warm-up starts from: the per-kernel split below
    # replays the warm-up and the timed steps from them
    start_pos = None if args.no_extras else tuple(a.copy() for a in ctx.positions())
    # warm-up (also captures the graph)
    if args.warmup:
        ctx.step(args.warmup, args.mode)
    rebuilds0 = ctx.rebuild_count()
    launches0 = ctx.launch_count()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        ctx.step(args.steps, args.mode)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    rebuilds_timed = ctx.rebuild_count() - rebuilds0
    launches_timed = ctx.launch_count() - launches0
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = n_all * args.steps / (ms * 1e-3)

    extras = {}
    # every rank's final positions, assembled on rank 0 in job order
    gathered = gather_positions(ctx, mine,
                                rank_tissue_ids(args.workload, args.tissues, world, rank), dist)
    if gathered is not None:
        extras["gathered"] = gathered
    if not args.no_extras:
        # Per-kernel device time over a replay of the timed steps: the
        # positions the warm-up started from, every tissue's candidates
        # rebuilt from them (as after the autotuner's last restore, or the
        # upload), the warm-up, then the timed number of steps with events
        # around each kernel class (launched one by one, not from the graph).
        # The replay should reproduce the timed steps' positions bit for bit
        # (checked below).
        end_pos = tuple(a.copy() for a in ctx.positions())
        ctx.set_positions(*start_pos)
        cfg_now = ctx.config()
        ctx.set_tuning(cfg_now["skin"], cfg_now["variant"], cfg_now["search_switch"],
                       cfg_now["rebuild_gate"])
        if args.warmup:
            ctx.step(args.warmup, args.mode)
        tk = ctx.time_kernels(args.steps)
        replay_pos = ctx.positions()
        extras["kernel_split"] = {
            "window": f"replay of the {args.warmup} warm-up and {args.steps} timed steps",
            "replay_bit_identical": bool(all(np.array_equal(a, b)
                                             for a, b in zip(end_pos, replay_pos))),
        }
        # The roofline is the step kernel's: it does the whole per-step work
        # of the reference (exact predicate = connect, forces, commit). In
        # eager timing the rebuild classes also carry their launches on steps
        # with nothing to rebuild, so the largest class is not always it.
        dom = "step"
        dom_ms = tk[dom][0] / max(tk[dom][1], 1)
        hbm, peak_kind = measured_peaks()
        # Algorithmic bytes per particle of each kernel class. Step:
        # B = 52 + 8 k (24 B xyz read, 24 B xyz write, 4 B state, 4k B list
        # write + 4k B list read).
        per_particle = {
            "step": 52 + 8 * kbar,
            "prepass": 32 * 3 + 64,
            "rebuild_bin": 32 + 4 + 8,
            "rebuild_scan": 0,
            "rebuild_sort": 4 + 32 + 4 + 32,
            "rebuild_search": 32 + 4 + 4 * 2 * kbar + 4,
            "gate": 0,
        }
        alg = per_particle[dom] * n_mine
        achieved = alg / (dom_ms * 1e-3) / 1e9
        traffic = load_traffic(dom, args.workload)
        extras["roofline"] = {
            "bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback",
            "traffic": traffic, "alg_bytes_per_launch": alg,
            "launch_ms": dom_ms,
            "step_alg_bytes_per_particle": 52 + 8 * kbar,
            "step_frac": (52 + 8 * kbar) * value / max(world, 1) / 1e9 / hbm,
        }
        extras["kernel_ms_per_step"] = {k: v[0] / max(v[1], 1) for k, v in tk.items()}

        # e2e through the C ABI with host buffers: every step takes the
        # positions from pinned host memory and returns the new ones there.
        # epi_step_host_async queues each step (its copies of tissue groups
        # overlap other groups' kernels and the neighbouring steps' copies)
        # and epi_sync ends the run; epi_step_host waits for every step; the
        # three-call path (epi_upload_positions, epi_interact_commit,
        # epi_download_positions: the drop-in's data flow) runs its copies
        # and kernels one after another.
        pin = [torch.empty(n_mine, dtype=torch.float64, pin_memory=True) for _ in range(3)]
        host = tuple(p.numpy() for p in pin)
        ctx.positions(host)

        def timed_e2e(one_step):
            torch.cuda.synchronize()
            barrier()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            for _ in range(args.e2e_steps):
                one_step()
            ctx.sync()  # every queued step's copies are done
            f1.record(stream)
            f1.synchronize()
            barrier()
            e_ms = f0.elapsed_time(f1)
            if dist is not None:
                t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                e_ms = float(t.item())
            return n_all * args.e2e_steps / (e_ms * 1e-3)

        def three_calls():
            ctx.set_positions(*host)
            ctx.interact_commit()
            ctx.positions(host)

        ctx.step_host(host, host)  # first call sets up its streams and staging
        e2e_async = timed_e2e(lambda: ctx.step_host(host, host, wait=False))
        e2e_sync = timed_e2e(lambda: ctx.step_host(host, host))
        e2e_serial = timed_e2e(three_calls)
        extras["e2e"] = {"value": e2e_async, "unit": UNIT,
                         "h2d_bytes_per_step": 24 * n_mine, "d2h_bytes_per_step": 24 * n_mine,
                         "steps": args.e2e_steps,
                         "path": "epi_step_host_async per step, epi_sync after the last "
                                 "(positions in and out of pinned host arrays every step; copies "
                                 "of tissue groups overlap kernels and the neighbouring steps' "
                                 "copies)",
                         "sync_call_path": {"value": e2e_sync, "unit": UNIT,
                                            "path": "epi_step_host per step (returns with the "
                                                    "step's positions in host memory)"},
                         "three_call_path": {"value": e2e_serial, "unit": UNIT,
                                             "path": "epi_upload_positions + epi_interact_commit"
                                                     " + epi_download_positions per step"}}

        # plain FP64 GPU step: same kernels in FP64, one launch sequence per
        # tissue, no graph (the denominator of the >= 3x target)
        if args.plain_steps > 0:
            with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=64, device=local) as pc:
                pc.upload(mine)
                pc.step(1, "per_tissue")
                ps = torch.cuda.ExternalStream(pc.stream_handle())
                torch.cuda.synchronize()
                barrier()
                g0 = torch.cuda.Event(enable_timing=True)
                g1 = torch.cuda.Event(enable_timing=True)
                g0.record(ps)
                pc.step(args.plain_steps, "per_tissue")
                g1.record(ps)
                g1.synchronize()
                barrier()
                pms = g0.elapsed_time(g1)
            if dist is not None:
                t = torch.tensor([pms], device="cuda", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                pms = float(t.item())
            plain = n_all * args.plain_steps / (pms * 1e-3)
            extras["fp64_plain"] = {"value": plain, "unit": UNIT, "steps": args.plain_steps,
                                    "path": "FP64 forces, one launch sequence per tissue, "
                                            "no graph",
                                    "speedup": value / plain}

        # FP64 forces on the same batch, graph and step count as the headline:
        # what the precision pattern alone buys (batching and launch
        # amortisation are the same on both sides)
        if args.fp64_batched_steps > 0 and args.precision == "mixed":
            with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=64, device=local,
                              skin=cfg_skin(tuned, args)) as bc:
                bc.upload(mine)
                if args.warmup:
                    bc.step(args.warmup, args.mode)
                bs = torch.cuda.ExternalStream(bc.stream_handle())
                torch.cuda.synchronize()
                barrier()
                h0 = torch.cuda.Event(enable_timing=True)
                h1 = torch.cuda.Event(enable_timing=True)
                h0.record(bs)
                bc.step(args.fp64_batched_steps, args.mode)
                h1.record(bs)
                h1.synchronize()
                barrier()
                bms = h0.elapsed_time(h1)
            if dist is not None:
                t = torch.tensor([bms], device="cuda", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                bms = float(t.item())
            batched = n_all * args.fp64_batched_steps / (bms * 1e-3)
            extras["fp64_batched"] = {
                "value": batched, "unit": UNIT, "steps": args.fp64_batched_steps,
                "warmup": args.warmup,
                "path": "FP64 forces, same batch, graph and skin as the headline",
                "speedup": value / batched}

    if world == 1 and not args.no_extras:
        if args.accuracy_steps > 0:
            extras["accuracy"] = accuracy_check(capi, local, args.accuracy_steps)
        if args.adjoint_steps > 0:
            extras["adjoint"] = adjoint_check(capi, local, args.adjoint_steps)
        if args.field_steps > 0:
            extras["field"] = field_check(capi, local, args.field_steps,
                                          not args.no_cpu_baseline)
        if args.dropin_steps > 0 and not args.no_cpu_baseline:
            wl = [("c2", T.config2())]
            if args.dropin_c3:
                wl.append(("c3", T.config3()))
            extras["dropin"] = dropin_check(wl, args.dropin_steps, 2)

    if rank == 0:
        cfg = {"workload": desc, "tissues": n_tissues_all, "particles": n_all,
               "mean_connections": kbar, "precision": args.precision,
               "skin": cfg_skin(tuned, args),
               "variant": tuned["variant"] if tuned else (args.variant or 3),
               "search_switch": ctx.config()["search_switch"] or 49152,
               "autotune": tuned,
               "tissues_rebuilt_per_step": rebuilds_timed / max(args.steps, 1),
               "rebuilt_fraction_per_step": rebuilds_timed / max(args.steps, 1) / len(mine),
               "launch": "one graph launch per run (device WHILE loop over a 2-step body)",
               "l2": "inputs larger than L2 (working set >> 126 MB)"
               if n_all * 200 > 126e6 else "working set fits in L2 (no flush)",
               "parallelism": ("1 GPU" if world == 1 else
                               f"{world} GPUs, tissue shards of the {world}x ensemble (weak)"
                               if args.workload == "ensemble" else
                               f"{world} GPUs, one replica each (weak)")}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32-force/f64-sum" if args.precision == "mixed" else "f64",
                "data": "synthetic (seeded splitmix64 jittered lattices)", "config": cfg,
                "gpu_launches": launches_timed,
                "clocks": clk.summary()}
        line.update(extras)
        if world == 1 and not args.no_cpu_baseline and not args.no_extras:
            sample = reference_sample(tissues, args.ref_particles // 4)
            try:
                v, d = time_reference_cpu(sample, 2, 5)
                line["cpu_baseline"] = {
                    "value": v, "unit": UNIT, "cores": d["threads"], "kind": "reference",
                    "sample": f"{d['tissues']} tissues, {d['particles']} particles, "
                              f"median of 5 steps after 2 warm-up (epi5_MT, OpenMP TBB stand-in)"}
            except Exception as e:  # reference build missing on this host
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0,
                                        "kind": "reference", "sample": f"unavailable: {e}"}
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
