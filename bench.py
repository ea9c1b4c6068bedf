#!/usr/bin/env python
"""Benchmark of the FARRSIGHT hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload two_stream|landau|bump_on_tail|landau_batch|serve]
                    [--field direct32c|direct64|treecode32c|treecode64]

A step is one AMRSimulation::step of the workload (RK4 with three field
evaluations, then either the fourth field evaluation or the remesh + reduced
grid field every 5 steps), device resident.  Default workload: the two-stream
precision form -- 256 x 512 panels (525,825 points), eps 0.02, dt 0.2, FP32
compensated direct sum -- with synthetic inputs generated from the deck.

value     pair interactions per second over the timed steps (whole job: all
          ranks' pairs / max-over-ranks device time), CUDA events on the
          simulation's stream; L2 flushed (256 MiB write) between timed steps.
accuracy  FP32c against the plain FP64 path on the same workload: relative L2
          error of E on the final state, and the field-energy drift over an
          FP32c and an FP64 session stepped side by side from t = 0.
plain_fp64_gpu  the FP64 session's rate (k_direct64, the reference arithmetic
          bit for bit), with its FP64-pipe roofline; speedup_vs_plain_fp64_gpu
          is value over it.
batch     64 seeded Landau instances stepped together: rate, p50/p99 step
          latency, speed-up over the plain FP64 path.
e2e       same metric through the reference-facing plugin call
          (E_MQ_DirectSum_B200.__call__, i.e. fs_field_eval with HOST arrays)
          driving a host-side RK4 step like AMRSimulation::rk4_step: every
          field call copies sources and weights host->device and E back.
roofline  the dominant pair kernel: achieved pair rate per launch time against
          its FP32-pipe bound (and the one-MUFU-plus-8-FP32 convention).
cpu_baseline  the reference's own E_MQ_DirectSum (oracle/_ref, compiled from
          the reference sources) on all host cores, on a bounded target sample.

Multi-GPU: replicas only (one independent simulation per rank, no data-path
collective); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MUFU_PER_CLK_PER_SM = 16          # MUFU (rsqrt / rcp) lanes per clock per SM
FP32_LANES_PER_CLK_PER_SM = 128    # FP32 FMA-pipe lanes per clock per SM
# FP32 lane-operations per far pair in k_pairs32 (FFMA2 difference, FFMA2
# square, FFMA2 accumulate over two targets = 6, plus the scalar FMULs for
# r_a r_b and q W = 8 per two pairs); its MUFU use is 0.5 per pair, so the FP32
# datapath (128 / 4 = 32 pairs/clk/SM) and MUFU (16 x 2 = 32) bound it alike.
PAIR32_FP32_OPS = 4.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="two_stream",
                    choices=["two_stream", "landau", "bump_on_tail", "landau_batch", "serve"])
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serve: arrival window")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: mean arrivals per second")
    ap.add_argument("--batch", type=int, default=64, help="instances of the landau_batch workload")
    ap.add_argument("--field", default=None, choices=["direct32c", "direct64", "treecode32c", "treecode64"],
                    help="default: direct32c, treecode32c for bump_on_tail")
    ap.add_argument("--h", type=int, default=None, help="override the mesh height (small cases for profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP64 shadow run (accuracy, plain FP64 rate)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-instance batch record")
    ap.add_argument("--no-treecode", action="store_true",
                    help="skip the full-size treecode record (also skipped with --no-accuracy)")
    ap.add_argument("--drift-steps", type=int, default=None,
                    help="steps of the FP32c-vs-FP64 field-energy comparison (default: warmup + steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    return ap.parse_args()


def workload_deck(a):
    from multi_species_b200 import decks
    if a.workload == "two_stream":
        d = decks.two_stream(h=a.h or 8, ph=1, steps=100, remesh_period=5)
        name = "two_stream_precision_form"
    elif a.workload == "bump_on_tail":
        d = decks.bump_on_tail(h=a.h or 9, ph=1, steps=50)
        name = "bump_on_tail_treecode"
    elif a.workload == "landau_batch":
        # the batch's largest instance stands in for it where one deck is needed
        ds = decks.landau_batch(count=a.batch, seed=0)
        d = max(ds, key=decks.deck_points)
        name = f"landau_batch{a.batch}"
    else:
        d = decks.landau_two_species(h=a.h or 5, ph=1)
        name = "landau_two_species"
    return name, d


class ClockSampler:
    """nvidia-smi samples during the timed region (clock, throttle reasons)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def traffic_per_pair(kernel: str):
    """DRAM bytes per pair of a pair kernel, from the `dram_bytes_per_pair:` line
    of its committed ncu summary (profiles/<kernel>_*.md)."""
    import glob
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_*.md"))):
        with open(p) as f:
            lines = f.read().splitlines()
        if f"kernel: {kernel}" not in lines:
            continue
        for line in lines:
            if line.startswith("dram_bytes_per_pair:"):
                return {"dram_bytes_per_pair": float(line.split(":")[1]), "source": os.path.basename(p)}
    return None


def _lattice(deck, h_drop=0):
    """All species' mesh points and weights of a deck (optionally h reduced),
    from the oracle's mesh restatement: the CPU legs load no product code."""
    import oracle as O
    xs, qs = [], []
    for sp in deck["species_list"]:
        m = O.Mesh(max(1, sp["initial_height"] - h_drop), sp["p_height"], deck["xmin"], deck["xmax"], sp["pmin"],
                   sp["pmax"])
        xs.append(m.xs + 0.2 * m.ps)
        qs.append(m.base_weights(sp["q"], deck["quadrature"]))
    return np.concatenate(xs), np.concatenate(qs)


def workload_config(name, deck, n, world):
    """The workload, the same dict on both arms; how an arm computes it (field
    kind, L2 handling) goes in top-level keys."""
    return {"workload": name, "points": int(n), "eps": deck["greens_epsilon"], "dt": deck["dt"],
            "remesh_period": deck["remesh_period"], "parallelism": f"replicas{world}"}


def cpu_baseline(deck, seconds: float, treecode: bool = False):
    """The reference's own field code (oracle/_ref) on the host cores: the
    OpenMP direct sum over a sample of targets, or for treecode decks the
    reference treecode (serial as shipped) on a reduced copy of the deck."""
    import oracle as O
    L = deck["xmax"] - deck["xmin"]
    cores = os.cpu_count() or 1
    if treecode:
        for drop in (4, 3, 2):
            x, q = _lattice(deck, drop)
            t0 = time.perf_counter()
            O.ref_treecode(L, deck["greens_epsilon"], deck["mac"], deck["degree"], deck["max_source"], x, q)
            dt = time.perf_counter() - t0
            if dt > seconds / 4:
                break
        return {"value": len(x) ** 2 / dt, "unit": "pair-interactions/s (direct-equivalent)", "cores": 1,
                "kind": "reference",
                "sample": f"reference E_MQ_Treecode (serial far/near loops as shipped) on the deck with mesh height "
                          f"reduced by {drop}: {len(x)} points, one evaluation ({dt:.1f} s)"}
    x, q = _lattice(deck)
    nt = 256
    while True:
        t0 = time.perf_counter()
        O.ref_direct_sum(L, deck["greens_epsilon"], x[:nt], x, q, threads=cores)
        dt = time.perf_counter() - t0
        if dt > 0.5 or nt >= len(x):
            break
        nt = min(len(x), nt * 4)
    nt = int(min(len(x), max(nt, nt * seconds / max(dt, 1e-9) / 2)))
    t0 = time.perf_counter()
    O.ref_direct_sum(L, deck["greens_epsilon"], x[:nt], x, q, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": nt * len(x) / dt, "unit": "pair-interactions/s", "cores": cores, "kind": "reference",
            "sample": f"{nt} targets x {len(x)} sources of the workload's point set, one field evaluation "
                      f"({dt:.1f} s)"}


def run_reference(a, rank, world):
    """--impl reference: the reference's CPU direct sum on the host cores."""
    name, deck = workload_deck(a)
    if rank != 0:
        return None
    vals = []
    per = max(1.0, a.cpu_seconds / max(1, a.steps + a.warmup))
    tree = int(deck.get("use_treecode", 0)) > 0
    for _ in range(a.warmup):
        cpu_baseline(deck, per, tree)
    for _ in range(a.steps):
        vals.append(cpu_baseline(deck, per, tree))
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[-1])
    cb["value"] = v
    from multi_species_b200 import decks
    n = decks.deck_points(deck)
    return {"metric": "pair-interactions/s", "value": v, "unit": "pair-interactions/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (deck-generated point set)",
            "impl": "reference",
            # one RK4 step is four evaluations of n x n pairs; each timed step here
            # is a bounded sample of one evaluation, so the step time is extrapolated
            "ms_per_step": 4.0 * n * n / v * 1e3,
            "config": workload_config(name, deck, n, world),
            "field": ("reference E_MQ_Treecode (CPU, serial as shipped)" if tree
                      else "reference E_MQ_DirectSum (CPU, OpenMP)"),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "pair-interactions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


KERNEL_OF_FIELD = {"direct32c": "k_pairs32", "direct64": "k_direct64", "treecode32c": "k_near32",
                   "treecode64": "k_far_near64"}


def roofline(a, kern, kl, kms, kwork, total_ms, sm, peaks, peak_src, band_fraction=None):
    """Roofline object for the dominant kernel of the field kind.  For the
    FP32c pair kernels the band pairs (evaluated in FP64) come from the
    profile (one simulation) or from `band_fraction` (a batch)."""
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    clk_hz = mhz * 1e6
    mufu_peak = sm * MUFU_PER_CLK_PER_SM * clk_hz        # one MUFU op per pair
    fp32_peak = sm * FP32_LANES_PER_CLK_PER_SM * clk_hz / PAIR32_FP32_OPS
    achieved = kwork / (kms / 1e3) if kms > 0 else 0.0
    tr = traffic_per_pair(kern)
    roof = {"kernel": kern, "bound": "fp32-pipe", "unit": "Gpair/s", "achieved": achieved / 1e9,
            "peak": fp32_peak / 1e9, "frac": achieved / fp32_peak,
            "peak_source": f"{sm} SMs x {FP32_LANES_PER_CLK_PER_SM} FP32 lanes/clk x sm_max_mhz {mhz:.0f} "
                           f"({peak_src} MEASURED_PEAKS.json clock) / {PAIR32_FP32_OPS} FP32 lane-ops per far "
                           f"pair (packed FP32x2, one MUFU.RCP per two pairs)",
            "mufu_convention": {"peak": mufu_peak / 1e9, "frac": achieved / mufu_peak,
                                "note": "one MUFU op + 8 FP32 ops per pair: min(FP32/8, MUFU) = 16 pairs/clk/SM"},
            "launches": kl, "avg_launch_ms": kms / kl if kl else None,
            "pairs_per_launch": kwork / kl if kl else None,
            "traffic": (tr["dram_bytes_per_pair"] * (kwork / kl)) if (tr and kl) else None,
            "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum per pair from profiles/"
                               f"{tr['source']}, scaled by this run's pairs per launch") if tr else None,
            "kernel_share_of_step_time": kms / total_ms if total_ms else None}
    if a.field == "direct32c" and kern in ("k_pairs32", "k_pairs32_batched"):
        # far pairs on the FP32 pipe and MUFU, band pairs (|d| <= 16 eps) on
        # the FP64 pipe: the kernel's bound is the time of both at their peaks
        import multi_species_b200 as M
        band = kwork * band_fraction if band_fraction is not None else M.profile_read("pairs32_band_pairs")[2]
        if band > 0 and kms > 0:
            fp64_band_peak = sm * FP64_LANES_PER_CLK_PER_SM * clk_hz / BAND64_FP64_INSTR_PER_PAIR
            t_bound = (kwork - band) / fp32_peak + band / fp64_band_peak
            roof.update({"bound": "fp32-pipe (far pairs) + fp64-pipe (band pairs)",
                         "frac": t_bound / (kms / 1e3), "band_pairs_per_launch": band / kl,
                         "band_fraction": band / kwork, "fp64_band_peak_gpairs": fp64_band_peak / 1e9,
                         "frac_note": "frac = (far pairs / FP32-pipe peak + band pairs / FP64-pipe peak) / kernel "
                                      "time; achieved and peak are the direct-equivalent rate against the FP32 "
                                      "bound alone"})
    if a.field == "direct64":
        # two IEEE divisions + one square root + ~11 FP64 ops per pair, no MUFU shortcut
        roof.update({"bound": "fp64-pipe", "peak": None, "frac": None, "mufu_convention": None,
                     "peak_source": "FP64 pipe (reference arithmetic, bit-exact); not a speed-of-light kernel"})
    elif a.field.startswith("treecode"):
        # actual near-field pairs (counted on the device while profiling) per
        # near-kernel time, against one MUFU rsqrt per pair
        import multi_species_b200 as M
        near_pairs = M.profile_read("treecode_near_pairs")[2]
        ach = near_pairs / (kms / 1e3) if kms > 0 else 0.0
        roof.update({"bound": "mufu", "peak": mufu_peak / 1e9, "unit": "Gpair/s (near-field pairs)",
                     "achieved": ach / 1e9, "frac": ach / mufu_peak if a.field == "treecode32c" else None,
                     "mufu_convention": None, "pairs_per_launch": near_pairs / kl if kl else None,
                     "traffic": None,
                     "peak_source": f"{sm} SMs x {MUFU_PER_CLK_PER_SM} MUFU/clk x sm_max_mhz {mhz:.0f}: each "
                                    "near-field band pair needs one MUFU rsqrt",
                     "direct_equivalent_per_s": achieved / 1e9})
    return roof


def combine_ranks(total_ms, work):
    """Replicas: the job's device time is the slowest rank's, its work the sum
    over ranks (host scalars over the process group; no data-path collective)."""
    import torch
    import torch.distributed as D
    t = torch.tensor([float(total_ms)], dtype=torch.float64)
    D.all_reduce(t, op=D.ReduceOp.MAX)
    w = torch.tensor([float(x) for x in work], dtype=torch.float64)
    D.all_reduce(w, op=D.ReduceOp.SUM)
    return float(t.item()), [float(x) for x in w.tolist()]


def run_ours(a, rank, world, local_rank):
    import multi_species_b200 as M
    import torch
    name, deck = workload_deck(a)
    torch.cuda.set_device(local_rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
    sim = M.Simulation(deck, field_backend=a.field, device=local_rank)
    n = sim.n
    for _ in range(a.warmup):
        sim.step(1)
    M.profile_reset()
    M.profile_enable(True)
    launches0 = M.kernel_launches()
    pairs0, evals0 = sim.work()
    step_ms = []
    dist = world > 1
    if dist:
        import torch.distributed as D
        D.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            sim.step(1)
            step_ms.extend(sim.step_times().tolist())
    torch.cuda.synchronize()
    if dist:
        D.barrier()
    M.profile_enable(False)
    launches = M.kernel_launches() - launches0
    pairs1, evals1 = sim.work()
    pairs, evals = pairs1 - pairs0, evals1 - evals0
    total_ms = float(np.sum(step_ms))
    kern = KERNEL_OF_FIELD[a.field]
    kl, kms, kwork = M.profile_read(kern)
    rl, rms, _ = M.profile_read("remesh")
    sim.close()
    t_max = total_ms
    if dist:
        t_max, (pairs, evals) = combine_ranks(total_ms, [pairs, evals])
    value = pairs / (t_max / 1e3)
    res = None
    if rank == 0:
        peaks, peak_src = measured_peaks()
        sm = torch.cuda.get_device_properties(local_rank).multi_processor_count
        res = {"metric": "pair-interactions/s", "value": value, "unit": "pair-interactions/s", "n_gpus": world,
               "steps": a.steps, "warmup": a.warmup, "ms_per_step": t_max / a.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if a.field.endswith("32c") else "f64",
               "data": "synthetic (deck-generated, no dataset)",
               "config": workload_config(name, deck, n, world),
               "field": a.field, "l2": "flushed (256 MiB write) between timed steps",
               "value_note": VALUE_NOTE.get(a.field, ""),
               "rk4_steps_per_s": a.steps / (t_max / 1e3) * world,
               "kernel_evals_per_s": evals / (t_max / 1e3),
               "remesh_ms_per_remesh": (rms / rl) if rl else None,
               "gpu_launches": int(launches),
               "roofline": roofline(a, kern, kl, kms, kwork, total_ms, sm, peaks, peak_src),
               "clocks": clk.summary()}
        if not a.no_accuracy:
            acc = accuracy_vs_fp64(a, deck, local_rank, a.drift_steps or (a.warmup + a.steps), sm, peaks)
            res["accuracy"] = acc["accuracy"]
            res["plain_fp64_gpu"] = acc["plain_fp64_gpu"]
            res["speedup_vs_plain_fp64_gpu"] = value / acc["plain_fp64_gpu"]["value"]
        if not a.no_batch and a.workload == "two_stream":
            res["batch"] = batch_summary(local_rank, a.batch, 2, 4)
        if not a.no_treecode and not a.no_accuracy and a.workload == "two_stream":
            res["treecode"] = treecode_summary(local_rank, 1, 3)
        if not a.no_e2e:
            res["e2e"] = e2e_plugin(deck, a.field, n, local_rank, a.steps)
        if not a.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(deck, a.cpu_seconds, a.field.startswith("treecode"))
    return res


VALUE_NOTE = {
    "direct32c": "pairs are direct-equivalent: N^2 per full evaluation (and U^2 per reduced-grid evaluation) at the "
                 "accuracy stated in `accuracy`; far pairs (|d| > 16 eps) are summed as an exact FP64 sign part plus a "
                 "one-term series of analytic error <= v^2/16 (v = eps^2/(d^2+eps^2)) accumulated in FP32, band pairs "
                 "(|d| <= 16 eps) in FP64",
    "direct64": "pairs evaluated one by one with the reference's FP64 arithmetic (bit-identical)",
    "treecode32c": "pairs are direct-equivalent N^2 per evaluation; the treecode evaluates near-field pairs and "
                   "far-field cluster terms (kernel_evals_per_s)",
    "treecode64": "pairs are direct-equivalent N^2 per evaluation; the treecode evaluates near-field pairs and "
                  "far-field cluster terms (kernel_evals_per_s)",
}

# FP64 pipe: 64 FP64 lanes per clock per SM on B200 (half the FP32 lanes).
FP64_LANES_PER_CLK_PER_SM = 64
# FP64 thread instructions per pair of k_direct64 (its two IEEE divisions,
# square root, round, compares and the term: 17.1 DFMA + 12.0 DMUL + 8.0 DADD
# + 3.1 others), counted by ncu (sm__sass_thread_inst_executed_op_fp64_pred_on
# over the launch's pairs) on the two-stream deck at 33,153 points; the count
# per pair does not depend on the size.
DIRECT64_FP64_INSTR_PER_PAIR = 40.2
# FP64 instructions per band pair of k_pairs32: d (DADD), d^2 + eps^2 (DFMA),
# (q/4) d y (two DMUL), y^2 (DMUL), 3 - r y^2 (DFMA) and the accumulation
# (DFMA), the Newton step's 1/2 folded into q/4; plus one MUFU op.
BAND64_FP64_INSTR_PER_PAIR = 7.0


def accuracy_vs_fp64(a, deck, local_rank, steps, sm, peaks):
    """FP32c against the plain FP64 path on the same workload, from t = 0:

    * field_energy_drift = max_t |W32(t) - W64(t)| / max_t W64(t) over `steps`
      steps of an FP32c session and an FP64 session (W = 1/2 sum dx E^2 at the
      unique x in [0, L), the reference's diagnostic);
    * e_rel_l2 = ||E32 - E64|| / ||E64||: E32 the FP32c session's own field at
      the end of its last step (a full evaluation, as in the timed steps), E64
      the plain FP64 sum on the same positions and weights (all N targets and
      sources);
    * plain_fp64_gpu: pair-interactions/s of the FP64 session (k_direct64, the
      reference arithmetic bit for bit; k_far_near64 for the treecode), CUDA
      events, with its kernel's FP64-pipe fraction."""
    import multi_species_b200 as M
    L = deck["xmax"] - deck["xmin"]
    tree = a.field.startswith("treecode")
    k64 = "treecode64" if tree else "direct64"
    s32 = M.Simulation(deck, field_backend=a.field, device=local_rank)
    s64 = M.Simulation(deck, field_backend=k64, device=local_rank)
    w32, w64 = [M.field_energy(s32.state()["xs"], s32.state()["es"], L)], []
    w64.append(M.field_energy(s64.state()["xs"], s64.state()["es"], L))
    M.profile_reset()
    M.profile_enable(True)
    t64, p64 = 0.0, 0.0
    for _ in range(steps):
        s32.step(1)
        q0, _ = s64.work()
        s64.step(1)
        t64 += float(np.sum(s64.step_times()))
        p64 += s64.work()[0] - q0
        st32, st64 = s32.state(), s64.state()
        w32.append(M.field_energy(st32["xs"], st32["es"], L))
        w64.append(M.field_energy(st64["xs"], st64["es"], L))
    M.profile_enable(False)
    kern64 = KERNEL_OF_FIELD[k64]
    kl, kms, kwork = M.profile_read(kern64)
    if s32.iteration()[0] % int(deck["remesh_period"]) == 0:
        s32.step(1)  # end on a full evaluation, not a remesh's reduced grid
    st32 = s32.state()
    s32.close()
    s64.close()
    w32, w64 = np.array(w32), np.array(w64)
    if tree:
        f32 = M.E_MQ_Treecode_B200(L, deck["greens_epsilon"], deck["mac"], deck["degree"], deck["max_source"],
                                   precision="fp32c", device=local_rank)
        f64 = M.E_MQ_Treecode_B200(L, deck["greens_epsilon"], deck["mac"], deck["degree"], deck["max_source"],
                                   precision="fp64", device=local_rank)
    else:
        f32 = M.E_MQ_DirectSum_B200(L, deck["greens_epsilon"], "fp32c", device=local_rank)
        f64 = M.E_MQ_DirectSum_B200(L, deck["greens_epsilon"], "fp64", device=local_rank)
    x, q = st32["xs"], st32["q_ws"]
    e32, e64 = st32["es"], f64.evaluate(x, x, q)
    if tree:
        e32p = f32.evaluate(x, x, q)
    f32.close()
    f64.close()
    acc = {"e_rel_l2": float(np.linalg.norm(e32 - e64) / np.linalg.norm(e64)),
           "e_reference": f"{k64} at the session's final positions and weights (all {len(x)} targets)",
           "field_energy_drift": float(np.max(np.abs(w32 - w64)) / np.max(w64)),
           "drift_steps": steps,
           "target": "e_rel_l2 <= 1e-6, field_energy_drift <= 1e-5"}
    if tree:
        # the treecode's own approximation error, against the plain FP64 direct
        # sum (rescaled by the treecode kernel's sqrt(L^2 + 4 eps^2) / L) on
        # 4096 evenly spaced targets
        idx = np.linspace(0, len(x) - 1, 4096).astype(np.int64)
        fd = M.E_MQ_DirectSum_B200(L, deck["greens_epsilon"], "fp64", device=local_rank)
        ed = fd.evaluate(x[idx], x, q) * np.sqrt(L * L + 4 * deck["greens_epsilon"] ** 2) / L
        fd.close()
        acc["tree_vs_direct64_sampled"] = {"fp32c": float(np.linalg.norm(e32p[idx] - ed) / np.linalg.norm(ed)),
                                           "fp64": float(np.linalg.norm(e64[idx] - ed) / np.linalg.norm(ed)),
                                           "targets": len(idx)}
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    plain = {"value": p64 / (t64 / 1e3), "unit": "pair-interactions/s", "path": f"{k64} Simulation, same deck",
             "steps": steps, "ms_per_step": t64 / steps}
    if not tree and kms > 0 and DIRECT64_FP64_INSTR_PER_PAIR:
        rate = kwork / (kms / 1e3)
        peak = sm * FP64_LANES_PER_CLK_PER_SM * mhz * 1e6 / DIRECT64_FP64_INSTR_PER_PAIR
        plain["roofline"] = {"kernel": kern64, "bound": "fp64-pipe", "unit": "Gpair/s", "achieved": rate / 1e9,
                             "peak": peak / 1e9, "frac": rate / peak,
                             "peak_source": f"{sm} SMs x {FP64_LANES_PER_CLK_PER_SM} FP64 lanes/clk x {mhz:.0f} MHz / "
                                            f"{DIRECT64_FP64_INSTR_PER_PAIR} FP64-pipe instructions per pair "
                                            "(ncu count, profiles/k_direct64_two_stream.md)"}
    return {"accuracy": acc, "plain_fp64_gpu": plain}


def treecode_summary(local_rank, warmup, steps):
    """Compact record of the treecode workload at full size (three species x
    2,100,225 points, FP32c treecode, degree 8, theta 0.7, leaf 2000): step
    time and pair rate over `steps` steps, and the final state's field
    against the FP64 treecode (all targets) and against the plain FP64 direct
    sum on 4096 evenly spaced targets (the treecode's own approximation)."""
    import multi_species_b200 as M
    from multi_species_b200 import decks
    d = decks.bump_on_tail()
    L = d["xmax"] - d["xmin"]
    sim = M.Simulation(d, field_backend="treecode32c", device=local_rank)
    sim.step(warmup)
    p0, _ = sim.work()
    ms = []
    for _ in range(steps):
        sim.step(1)
        ms.extend(sim.step_times().tolist())
    pairs = sim.work()[0] - p0
    if sim.iteration()[0] % int(d["remesh_period"]) == 0:
        sim.step(1)  # end on a full evaluation, not a remesh's reduced grid
    st = sim.state()
    sim.close()
    x, q, e32 = st["xs"], st["q_ws"], st["es"]
    f64 = M.E_MQ_Treecode_B200(L, d["greens_epsilon"], d["mac"], d["degree"], d["max_source"], precision="fp64",
                               device=local_rank)
    e64 = f64.evaluate(x, x, q)
    f64.close()
    idx = np.linspace(0, len(x) - 1, 4096).astype(np.int64)
    fd = M.E_MQ_DirectSum_B200(L, d["greens_epsilon"], "fp64", device=local_rank)
    ed = fd.evaluate(x[idx], x, q) * np.sqrt(L * L + 4 * d["greens_epsilon"] ** 2) / L
    fd.close()
    rel = lambda a_, b_: float(np.linalg.norm(a_ - b_) / np.linalg.norm(b_))
    return {"workload": "bump_on_tail_treecode", "points": int(len(x)), "field": "treecode32c",
            "steps": steps, "warmup": warmup, "ms_per_step": float(np.mean(ms)),
            "value": pairs / (float(np.sum(ms)) / 1e3), "unit": "pair-interactions/s (direct-equivalent)",
            "e_rel_l2_vs_fp64_treecode": rel(e32, e64),
            "e_rel_l2_vs_fp64_direct_sampled": rel(e32[idx], ed),
            "fp64_treecode_vs_fp64_direct_sampled": rel(e64[idx], ed),
            "note": "all targets against the FP64 treecode; 4096 sampled targets against the FP64 direct sum "
                    "(rescaled by the treecode kernel's sqrt(L^2 + 4 eps^2) / L), which measures the treecode's "
                    "own approximation at theta 0.7, degree 8"}


def batch_summary(local_rank, count, warmup, steps):
    """Compact C4 record: `count` seeded Landau instances stepped together
    (one persistent pair launch per field evaluation, autotuned, graph-replayed
    steps), p50/p99 step latency and the rate against the plain FP64 path on
    the batch's largest instance."""
    import multi_species_b200 as M
    from multi_species_b200 import decks
    ds = decks.landau_batch(count=count, seed=0)
    b = M.Batch(device=local_rank)
    for d in ds:
        b.add(d)
    b.step(warmup)
    p0 = b.pair_count()
    ms = []
    for _ in range(steps):
        b.step(1)
        ms.extend(b.step_times().tolist())
    pairs = b.pair_count() - p0
    st = b.stats()
    b.close()
    big = max(ds, key=decks.deck_points)
    sim = M.Simulation(big, field_backend="direct64", device=local_rank)
    sim.step(1)
    w0, _ = sim.work()
    sim.step(1)
    plain = (sim.work()[0] - w0) / (float(np.sum(sim.step_times())) / 1e3)
    sim.close()
    value = pairs / (float(np.sum(ms)) / 1e3)
    return {"workload": f"landau_batch{count}", "instances": len(ds),
            "points_total": int(sum(decks.deck_points(d) for d in ds)), "steps": steps, "warmup": warmup,
            "value": value, "unit": "pair-interactions/s", "step_ms_p50": float(np.percentile(ms, 50)),
            "step_ms_p99": float(np.percentile(ms, 99)), "plain_fp64_gpu": plain,
            "speedup_vs_plain_fp64_gpu": value / plain,
            "tuning": {k: st[k] for k in ("targets_per_thread", "tiles_per_item")},
            "graph_steps": st["graph_steps"]}


def run_batch(a, rank, world, local_rank):
    """landau_batch: independent Landau instances of 2k-200k points stepped
    together (fs_batch_*: one persistent pair launch per field evaluation,
    autotuned items, graph-replayed steps).  Next to it, the plain FP64 GPU
    path (direct64, one simulation at a time) on the batch's largest instance."""
    import multi_species_b200 as M
    import torch
    from multi_species_b200 import decks
    torch.cuda.set_device(local_rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
    ds = decks.landau_batch(count=a.batch, seed=0)
    b = M.Batch(device=local_rank)
    ids = [b.add(d) for d in ds]
    npts = [b.info(i)["n"] for i in ids]
    for _ in range(a.warmup):
        b.step(1)
    M.profile_reset()
    M.profile_enable(True)
    launches0 = M.kernel_launches()
    pairs0 = b.pair_count()
    step_ms = []
    dist = world > 1
    if dist:
        import torch.distributed as D
        D.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            b.step(1)
            step_ms.extend(b.step_times().tolist())
    torch.cuda.synchronize()
    if dist:
        D.barrier()
    M.profile_enable(False)
    launches = M.kernel_launches() - launches0
    pairs = b.pair_count() - pairs0
    kl, kms, kwork = M.profile_read("k_pairs32_batched")
    breakdown = {k: M.profile_read(k)[1] / a.steps for k in ("k_pairs32_batched", "batch_prepare", "batch_finalize",
                                                             "remesh")}
    stats = b.stats()
    band, last = b.band_pairs()  # the last evaluation's band share stands for the timed ones
    b.close()
    total_ms = float(np.sum(step_ms))
    t_max = total_ms
    if dist:
        t_max, (pairs,) = combine_ranks(total_ms, [pairs])
    value = pairs / (t_max / 1e3)
    if rank != 0:
        return None
    # plain FP64 GPU path on the largest instance, same device
    big = max(ds, key=decks.deck_points)
    sim = M.Simulation(big, field_backend="direct64", device=local_rank)
    sim.step(1)
    w0, _ = sim.work()
    sim.step(2)
    w1, _ = sim.work()
    plain = (w1 - w0) / (float(np.sum(sim.step_times())) / 1e3)
    sim.close()
    peaks, peak_src = measured_peaks()
    sm = torch.cuda.get_device_properties(local_rank).multi_processor_count
    a.field = "direct32c"
    roof = roofline(a, "k_pairs32_batched", kl, kms, kwork, total_ms, sm, peaks, peak_src,
                    band_fraction=band / last if last > 0 else None)
    res = {"metric": "pair-interactions/s", "value": value, "unit": "pair-interactions/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": t_max / a.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (deck-generated, no dataset)",
           "config": {"workload": f"landau_batch{a.batch}", "instances": len(ds), "points_total": int(sum(npts)),
                      "points_min": int(min(npts)), "points_max": int(max(npts)),
                      "eps": 0.05, "dt": 0.25, "remesh_period": 5, "parallelism": f"replicas{world}"},
           "field": "direct32c", "l2": "flushed (256 MiB write) between timed steps",
           "tuning": {k: stats[k] for k in ("targets_per_thread", "tiles_per_item")},
           "graph_steps": stats["graph_steps"], "plain_steps": stats["plain_steps"],
           "rk4_steps_per_s": a.steps * len(ds) / (t_max / 1e3) * world,
           "plain_fp64_gpu": {"value": plain, "unit": "pair-interactions/s",
                              "path": "direct64 Simulation (reference arithmetic), largest instance alone",
                              "points": decks.deck_points(big)},
           "speedup_vs_plain_fp64_gpu": value / plain,
           "step_ms_p50": float(np.percentile(step_ms, 50)), "step_ms_p99": float(np.percentile(step_ms, 99)),
           "ms_per_step_by_phase": breakdown,
           "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary()}
    if not a.no_e2e:
        res["e2e"] = e2e_plugin(big, "direct32c", decks.deck_points(big), local_rank, a.steps)
        res["e2e"]["note"] = "plugin path on the batch's largest instance"
    if not a.no_cpu_baseline:
        res["cpu_baseline"] = cpu_baseline(big, a.cpu_seconds, False)
    return res


def run_serve(a, rank, world, local_rank):
    """serve: Poisson arrivals (rate/s over serve-seconds) of Landau, two-stream
    and bump-on-tail requests (10k-2M points, 10-100 steps) into fs_pool with a
    150 GB HBM budget.  Requests arriving while others run are admitted as
    memory and slots free up and stepped together.  value = pair interactions
    completed inside the arrival window / window; latencies are per (request,
    step).  What is still queued at the end of the window is cancelled."""
    import multi_species_b200 as M
    import torch
    from multi_species_b200 import decks
    torch.cuda.set_device(local_rank)
    reqs = decks.serving_requests(rate=a.rate, seconds=a.serve_seconds, seed=rank)
    pool = M.Pool(device=local_rank, hbm_budget=150e9, max_live=64)
    ids, kinds = [], {}
    launches0 = M.kernel_launches()
    h2d = 0
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        for (t_arr, kind, deck, steps) in reqs:
            now = time.perf_counter() - t0
            if t_arr > now:
                time.sleep(t_arr - now)
            rid = pool.submit(deck, steps)
            ids.append(rid)
            kinds[rid] = kind
            h2d += 4 * 8 * decks.deck_points(deck)  # x, p, f, q_w uploaded at set-up
        rest = a.serve_seconds - (time.perf_counter() - t0)
        if rest > 0:
            time.sleep(rest)
        window = time.perf_counter() - t0
        st = pool.stats()
    infos = [pool.poll(r) for r in ids]
    launches = M.kernel_launches() - launches0
    pool.close()
    done = [i for i in infos if i["state"] == "done"]
    steps_total = sum(i["steps_done"] for i in infos)
    d2h = sum(5 * 8 * i["npoints"] for i in done)
    turn = [i["total_ms"] for i in done]
    value = st["pairs"] / window
    if rank != 0:
        return None
    by_kind = {}
    for r, i in zip(ids, infos):
        k = by_kind.setdefault(kinds[r], {"submitted": 0, "completed": 0, "steps": 0, "pairs": 0.0})
        k["submitted"] += 1
        k["completed"] += i["state"] == "done"
        k["steps"] += i["steps_done"]
        k["pairs"] += i["pairs"]
    return {"metric": "pair-interactions/s", "value": value, "unit": "pair-interactions/s", "n_gpus": world,
            "steps": int(steps_total), "warmup": 0, "ms_per_step": st["step_ms_p50"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Poisson request stream of deck-generated simulations)",
            "config": {"workload": "serve", "rate_per_s": a.rate, "window_s": a.serve_seconds,
                       "requests": len(reqs), "points": "log-normal median 100k (log-sd 1), clipped 10k-2M",
                       "steps_per_request": "10-100", "hbm_budget_gb": 150, "max_live": 64,
                       "fields": {"landau": "direct32c", "two_stream": "direct32c", "bump_on_tail": "treecode32c"}},
            "value_note": "pairs of treecode (bump_on_tail) requests are direct-equivalent N^2 per field "
                          "evaluation; by_kind gives the split",
            "step_ms_p50": st["step_ms_p50"], "step_ms_p99": st["step_ms_p99"],
            "requests": {"submitted": int(st["submitted"]), "admitted": int(st["admitted"]),
                         "completed_in_window": int(st["completed"]), "queued_at_end": int(st["queued"]),
                         "live_at_end": int(st["live"]), "by_kind": by_kind},
            "turnaround_ms_p50": float(np.percentile(turn, 50)) if turn else None,
            "turnaround_ms_p99": float(np.percentile(turn, 99)) if turn else None,
            "busy_fraction": st["busy_ms"] / (1e3 * window),
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "e2e": {"value": value, "unit": "pair-interactions/s",
                    "h2d_bytes_per_step": h2d / max(steps_total, 1), "d2h_bytes_per_step": d2h / max(steps_total, 1),
                    "path": "fs_pool_submit (host deck) -> fs_pool_result (host arrays); the served metric is "
                            "end to end by construction"}}


def host_rk4_step(field, xs, ps, es, qw, qm, dt, work=None):
    """AMRSimulation::rk4_step + end-of-step field on the host, each field
    evaluation through the plugin call with host arrays (qm per point).  The
    caller's arithmetic is the reference's, in its order, written in place
    into preallocated buffers (`work`, nine arrays of len(xs)) the way the
    reference's C++ loops write into its vectors."""
    n = len(xs)
    if work is None:
        work = [np.empty(n) for _ in range(9)]
    ef1, ef2, ef3, ef4, p2, p3, p4, xk, tmp = work
    mul, add = np.multiply, np.add
    mul(es, qm, out=ef1)
    mul(0.5 * dt, ef1, out=p2)
    add(ps, p2, out=p2)
    mul(0.5 * dt, ps, out=xk)
    add(xs, xk, out=xk)
    field(ef2, xk, n, xk, qw, n)
    mul(ef2, qm, out=ef2)
    mul(0.5 * dt, ef2, out=p3)
    add(ps, p3, out=p3)
    mul(0.5 * dt, p2, out=xk)
    add(xs, xk, out=xk)
    field(ef3, xk, n, xk, qw, n)
    mul(ef3, qm, out=ef3)
    mul(dt, ef3, out=p4)
    add(ps, p4, out=p4)
    mul(dt, p3, out=xk)
    add(xs, xk, out=xk)
    field(ef4, xk, n, xk, qw, n)
    mul(ef4, qm, out=ef4)
    # xs + dt/6 (p1 + 2 p2 + 2 p3 + p4) and ps + dt/6 (ef1 + 2 ef2 + 2 ef3 + ef4), left to right
    mul(2, p2, out=tmp)
    add(ps, tmp, out=tmp)
    mul(2, p3, out=xk)
    add(tmp, xk, out=tmp)
    add(tmp, p4, out=tmp)
    mul(dt / 6.0, tmp, out=tmp)
    xs = xs + tmp
    mul(2, ef2, out=tmp)
    add(ef1, tmp, out=tmp)
    mul(2, ef3, out=xk)
    add(tmp, xk, out=tmp)
    add(tmp, ef4, out=tmp)
    mul(dt / 6.0, tmp, out=tmp)
    ps = ps + tmp
    es = np.empty(n)
    field(es, xs, n, xs, qw, n)
    return xs, ps, es


def e2e_plugin(deck, field_kind, n, device, steps=2):
    """The metric through the reference-facing plugin call with HOST arrays:
    E_MQ_DirectSum_B200 / E_MQ_Treecode_B200 (es, targets, nt, sources, q_ws, ns)
    driving the caller's host RK4 step, `steps` steps after one warm-up step.
    Bytes are counted from the arrays each call hands over: sources and
    weights host->device (targets too when they are a different array) and E
    device->host."""
    import multi_species_b200 as M
    sim = M.Simulation(deck, field_backend=field_kind, device=device)
    st = sim.state()
    counts = sim.species_points
    sim.close()
    L = deck["xmax"] - deck["xmin"]
    prec = "fp32c" if field_kind.endswith("32c") else "fp64"
    if field_kind.startswith("treecode"):
        f = M.E_MQ_Treecode_B200(L, deck["greens_epsilon"], deck["mac"], deck["degree"], deck["max_source"],
                                 precision=prec, device=device)
    else:
        f = M.E_MQ_DirectSum_B200(L, deck["greens_epsilon"], prec, device=device)
    qm = np.concatenate([np.full(c, sp["q"] / sp["m"]) for c, sp in zip(counts, deck["species_list"])])
    xs, ps, es, qw = st["xs"], st["ps"], st["es"], st["q_ws"]
    in_calls = [0.0]
    moved = [0, 0]

    def timed_field(es_, targets, nt, sources, q_ws, ns):
        c0 = time.perf_counter()
        f(es_, targets, nt, sources, q_ws, ns)
        in_calls[0] += time.perf_counter() - c0
        moved[0] += sources[:ns].nbytes + q_ws[:ns].nbytes + (0 if targets is sources else targets[:nt].nbytes)
        moved[1] += es_[:nt].nbytes

    work = [np.empty(len(xs)) for _ in range(9)]
    xs, ps, es = host_rk4_step(timed_field, xs, ps, es, qw, qm, deck["dt"], work)  # warm-up
    in_calls[0] = 0.0
    moved[0] = moved[1] = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        xs, ps, es = host_rk4_step(timed_field, xs, ps, es, qw, qm, deck["dt"], work)
    dt = time.perf_counter() - t0
    f.close()
    pairs = 4.0 * n * n * steps
    return {"value": pairs / dt, "unit": "pair-interactions/s", "h2d_bytes_per_step": moved[0] / steps,
            "d2h_bytes_per_step": moved[1] / steps, "steps": steps,
            "ms_per_plugin_call": 1e3 * in_calls[0] / (4 * steps),
            "host_rk4_ms_per_step": 1e3 * (dt - in_calls[0]) / steps,
            "path": f"{type(f).__name__}(es, targets, nt, sources, q_ws, ns) with host arrays, host RK4"}


def main():
    a = parse()
    if a.field is None:
        a.field = "treecode32c" if a.workload == "bump_on_tail" else "direct32c"
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as D
        D.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    try:
        if a.impl == "reference":
            res = run_reference(a, rank, world)
        elif a.workload == "landau_batch":
            res = run_batch(a, rank, world, local_rank)
        elif a.workload == "serve":
            res = run_serve(a, rank, world, local_rank)
        else:
            res = run_ours(a, rank, world, local_rank)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as D
            D.destroy_process_group()


if __name__ == "__main__":
    main()
