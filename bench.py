#!/usr/bin/env python
"""Benchmark of the interpolation-grid build (path a) on the charged synthetic framework (three 133 x 133 x 89 grids).

Workload (one "step"): the three tricubic grids of the charged synthetic framework — C_co2 Lennard-Jones, O_co2
Lennard-Jones and the unit-charge real-space Ewald grid — 133 x 133 x 89 = 1,574,321 points each (0.15 Angstrom
spacing over the 20.0 x 19.9 x 13.4 Angstrom cell, 96 T + 192 O atoms, rc = 12 Angstrom, alpha = 0.265), computed in
FP32 with compensated accumulation (FP32C). Metric: grid points per second over the whole job.

* value: device-resident output buffers, CUDA events on the launching stream, an L2 flush (a 256 MiB write) between
  timed steps (the per-step output of 302 MB also exceeds the 126 MB L2), max over ranks.
* e2e: the same steps through the C-ABI with host buffers: the framework upload and the 302 MB device-to-host copy of
  the grids are inside the timed region.
* roofline: the dominant kernel's achieved FP32 throughput (in-cutoff pairs x FLOPs per pair / launch time) against
  the FP32 FMA throughput measured by rg_probe_fma_peak in the same run.
* cpu_baseline: the FP64 CPU oracle (the reference's grid loop restated) on a sample of points, all host cores.

--impl reference times the CPU oracle alone on the same workload (rank 0 only).
Multi-GPU: the grid build is replicated (independent frameworks per rank, no collective), so scaling is weak.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid pts/s"
UNIT = "grid points/s"
# FLOPs per in-cutoff pair of the restated formulas (add/mul = 1, FMA = 2, reciprocal/sqrt/erfc/exp = 1 each).
FLOPS_PER_PAIR = {"lj": 55, "ewald": 65}
# DRAM bytes (read + write) per launch of the grid kernels in their ncu capture (the grid-build summary in profiles/)
NCU_DRAM_BYTES = {"LJ C_co2+O_co2 (two-probe kernel)": 0.29e6 + 143e6, "Ewald-real": 0.17e6 + 44e6}
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gcmc", action="store_true", help="skip the GCMC steps/s section")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-uniform proposal section")
    ap.add_argument("--no-alkane", action="store_true", help="skip the batched flexible-chain CBMC section")
    ap.add_argument("--no-mixture", action="store_true", help="skip the large two-component system section")
    ap.add_argument("--no-paths", action="store_true", help="skip the trial-energy and Ewald C-ABI section")
    ap.add_argument("--no-triquintic", action="store_true", help="skip the triquintic grid section")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the cpu_baseline sample")
    return ap.parse_args()


def workload():
    from raspa3_b200.synthetic import spacing_grid_dims, synthetic_forcefield, synthetic_framework

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=8)
    cell, atoms = synthetic_framework(ff, seed=42)
    dims = spacing_grid_dims(cell)
    grids = [("C_co2-LJ", 0, ff.index("C_co2")), ("O_co2-LJ", 0, ff.index("O_co2")), ("Ewald-real", 1, 0)]
    return ff, cell, atoms, dims, grids


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def max_over_ranks(seconds: float, world: int, dist, device: str = "cuda") -> float:
    """The slowest rank's time of a timed region (every rank makes this call at the same point, so the collective
    sequence is the same on all ranks); the time itself with one rank."""
    if world <= 1:
        return seconds
    import torch

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Units per second of the whole job: every rank processed units_per_rank in at most `seconds` (weak scaling)."""
    return world * units_per_rank / seconds


def cpu_oracle_rate(ff, cell, atoms, dims, grids, target_seconds, threads=0, seed=5):
    """FP64 oracle on a random sample of grid points of every grid; returns (points/s, points, seconds, threads)."""
    import oracle

    nx, ny, nz = dims
    total = nx * ny * nz
    rng = np.random.default_rng(seed)
    threads = threads or os.cpu_count() or 1

    def run(n):
        pts = np.sort(rng.choice(total, size=min(n, total), replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        for _, gt, probe in grids:
            oracle.make_grid(gt, ff, cell, atoms, probe, 12.0, dims, points=pts, threads=threads)
        return len(pts) * len(grids), time.perf_counter() - t0

    n0 = 64 * threads
    pts0, t0 = run(n0)
    n1 = int(n0 * max(1.0, target_seconds / max(t0, 1e-3)))
    pts1, t1 = run(n1)
    return pts1 / t1, pts1, t1, threads


def run_methane_grid_fp64(args, ctx, world, rank, dist, torch):
    """The plain small FP64 case: the methane Lennard-Jones tricubic grid of the uncharged synthetic
    framework, 133 x 133 x 89 points, FP64 pair terms and sums: grid points/s, the FP64-pipe roofline, end to end
    through rg_grid_build with a pinned host output, and the FP64 oracle on the host cores."""
    from raspa3_b200 import native
    from raspa3_b200.synthetic import spacing_grid_dims, synthetic_forcefield, synthetic_framework

    ff = synthetic_forcefield(charges=False)
    cell, atoms = synthetic_framework(ff, seed=42)
    dims = spacing_grid_dims(cell)
    npts = dims[0] * dims[1] * dims[2]
    probe = ff.index("CH4")
    stream = torch.cuda.current_stream()
    out = torch.empty(8 * npts, dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    _, st = ctx.grid_build(0, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64, out_device=out.data_ptr(),
                           host=False, count_pairs=True)
    peak64 = ctx.probe_fma_peak(native.PRECISION_FP64)
    for _ in range(args.warmup):
        ctx.grid_build(0, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64, out_device=out.data_ptr(),
                       host=False)
    steps = max(1, min(args.steps, 40))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        ctx.grid_build(0, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64, out_device=out.data_ptr(),
                       host=False)
        e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    total_s = max_over_ranks(sum(ms) / 1e3, world, dist)
    value = whole_job_rate(npts * steps, world, total_s)
    achieved = st["pair_count"] * FLOPS_PER_PAIR["lj"] / (statistics.mean(ms) * 1e-3) / 1e12
    # end to end: rg_grid_build with a pinned host output (upload of the images and the 100.75 MB download inside)
    host = torch.empty(8 * npts, dtype=torch.float64, pin_memory=True).numpy()
    ctx.grid_build(0, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64, out_host=host)
    torch.cuda.synchronize()
    e2e_steps = 5
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.grid_build(0, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64, out_host=host)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, dist)
    res = {"workload": "CH4 Lennard-Jones tricubic grid of the uncharged synthetic framework (96 T + 192 O, "
                       "20.0 x 19.9 x 13.4 A), 133 x 133 x 89 points, rc 12 A, FP64",
           "value": value, "unit": UNIT, "ms_per_step": 1e3 * total_s / steps, "steps": steps, "dtype": "f64",
           "pairs": st["pair_count"], "images": st["n_images"],
           "roofline": {"kernel": "gridKernel<double> (Lennard-Jones)", "bound": "fp64", "achieved": achieved,
                        "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                        "flops_per_pair": FLOPS_PER_PAIR["lj"],
                        "peak_source": "rg_probe_fma_peak(FP64): FP64 FMA chains on all SMs, measured in this run"},
           "e2e": {"value": whole_job_rate(npts * e2e_steps, world, e2e_s), "unit": UNIT,
                   "h2d_bytes_per_step": st["h2d_bytes"], "d2h_bytes_per_step": 8 * 8 * npts,
                   "path": "rg_grid_build with a pinned host output"},
           "clocks": clocks, "l2": "256 MiB flush between timed steps"}
    del flush
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, pts, secs, threads = cpu_oracle_rate(ff, cell, atoms, dims, [("CH4-LJ", 0, probe)],
                                                   min(args.cpu_seconds, 8.0))
        res["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{pts} random grid points in {secs:.1f} s (FP64 oracle of "
                                         f"makeFrameworkInterpolationGrid, release flags, OpenMP over points)"}
    return res


GCMC_CHAINS_PER_SM = 8
GCMC_MOVES = 2000
GCMC_EQUIL = 500


def gcmc_setup(ff, cell, atoms):
    from raspa3_b200.synthetic import replicate

    scell, sfw = replicate(cell, atoms, (2, 2, 3))
    return scell, sfw


def run_gcmc(args, ctx, ff, cell, atoms, dims, grids, outs, world, rank, dist, torch):
    """Device-resident GCMC of CO2 at 300 K and 1e5 Pa in the charged 2x2x3 box: move attempts per second over all chains."""
    from raspa3_b200 import native
    from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of

    scell, sfw = gcmc_setup(ff, cell, atoms)
    sysg = native.System(ctx, ff, scell, sfw)
    for (name, gt, probe), out in zip(grids, outs):
        idx = probe if gt == 0 else ff.n_types
        sysg.set_grid(idx, cell, dims, out.data_ptr(), on_device=True)
    ew = native.Ewald(ctx, ff, scell)
    ew.set_framework(sfw)
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    chains = GCMC_CHAINS_PER_SM * sms
    g = native.Gcmc(sysg, ew, co2_component(), beta_of(300.0), fugacity_of(1e5), n_chains=chains, seed=1 + rank)
    g.run(GCMC_EQUIL, record=False)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    e0.record(stream)
    g.run(GCMC_MOVES, record=True)
    e1.record(stream)
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    secs = max_over_ranks(secs, world, dist)
    # e2e: the same run call plus the read-back of every chain's statistics through the C-ABI
    t0 = time.perf_counter()
    g.run(GCMC_MOVES, record=True)
    res = g.results()
    e2e_secs = time.perf_counter() - t0
    moves = world * chains * GCMC_MOVES
    mean_n = float(np.mean([r["sum_n"] / max(1, r["samples"]) for r in res]))
    out = {"metric": "GCMC steps/s", "value": moves / secs, "unit": "MC move attempts/s", "chains": chains,
           "moves_per_chain": GCMC_MOVES, "ms": secs * 1e3,
           "workload": "CO2 (rigid 3-site), 300 K, 1e5 Pa, 2x2x3 box of the charged framework, FP32C grids, "
                       "Ewald alpha 0.265 kmax 8 (1152 k), translation/rotation/CBMC swap 1:1:1, 10+10 trials",
           "mean_loading": mean_n, "n_kvectors": ew.n_kvectors,
           "e2e": {"value": world * chains * GCMC_MOVES / e2e_secs, "unit": "MC move attempts/s",
                   "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": chains * 8 * 24 + chains * 12}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_gcmc_rate(ff, cell, scell, sfw, dims, grids, outs, args.cpu_seconds)
    g.close()
    ew.close()
    sysg.close()
    return out


ALKANE_SYSTEMS = 64
ALKANE_EQUIL = 2000
ALKANE_MOVES = 1000
# FLOPs per in-cutoff pair of the FP32 Lennard-Jones trial term: displacement scaling and r^2 (8), sigma^2/r^2 (1),
# t^3 (2), 4 eps t^3 (t^3 - 1) - shift (4), accumulation (1), counted as in the grid kernels (reciprocal = 1)
ALKANE_FLOPS_PER_PAIR = 16


def run_alkane(args, ctx, peak_fp32, world, rank, dist, torch):
    """Batched CBMC of flexible alkanes: 64 independent systems of uneven size (cells 12-40 A,
    96-1536 framework atoms, 4-8 bead chains) in one graph replay of persistent cluster kernels, GCMC at 300 K and
    1e5 Pa with translation and CBMC swap moves. Metric: move attempts per second over all systems, after
    equilibration, with the launch plan chosen by the autotuner."""
    from raspa3_b200 import native
    from raspa3_b200.alkane import alkane_forcefield, alkane_batch_systems

    ff = alkane_forcefield()
    systems = alkane_batch_systems(ff, n_systems=ALKANE_SYSTEMS, seed=1234, max_molecules=128)
    stream = torch.cuda.current_stream()
    w_ig = {}
    for q in systems:
        nb = q.chain.n_beads
        if nb not in w_ig:
            w_ig[nb] = native.alkane_grow_vacuum(ctx, ff, q.chain, q.beta, 200000, seed=17)
        q.w_ig = w_ig[nb]
    a = native.Alkane(ctx, ff, systems, seed=5 + rank)
    a.run(ALKANE_EQUIL, record=False)
    plan = a.autotune(moves_per_candidate=16)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    pairs0 = a.pair_count()
    launches0 = a.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    a.run(ALKANE_MOVES, record=True)
    e1.record(stream)
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    pairs = a.pair_count() - pairs0
    launches = a.launch_count() - launches0
    secs = max_over_ranks(secs, world, dist)
    res = a.results()
    # e2e: the run call plus the read-back of every system's statistics through the C-ABI
    t0 = time.perf_counter()
    a.run(ALKANE_MOVES, record=True)
    a.results()
    e2e_secs = time.perf_counter() - t0
    achieved = pairs * ALKANE_FLOPS_PER_PAIR / secs / 1e12
    loading = [r["n_molecules"] for r in res]
    out = {"metric": "batched CBMC steps/s", "value": world * ALKANE_SYSTEMS * ALKANE_MOVES / secs,
           "unit": "MC move attempts/s", "systems": ALKANE_SYSTEMS, "moves_per_system": ALKANE_MOVES,
           "ms": secs * 1e3, "plan": plan, "w_ig": {str(k): v for k, v in sorted(w_ig.items())},
           "workload": "64 synthetic cells (lengths U[12,40] A, 0.025 atoms/A^3 clipped to 96-1536 atoms, replicated "
                       "for rc = 12 A), one 4-8 bead TraPPE-UA alkane per system, 300 K, 1e5 Pa, translation : CBMC "
                       "swap 1 : 1, 10 first-bead trials, 10 directions x 100 torsion spins per bead",
           "loading_min_mean_max": [min(loading), float(np.mean(loading)), max(loading)],
           "pairs_per_move": pairs / (ALKANE_SYSTEMS * ALKANE_MOVES),
           "gpu_launches": launches, "kernel_launches_before_timed": launches0,
           "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_fp32, "unit": "TFLOP/s",
                        "frac": achieved / peak_fp32, "flops_per_pair": ALKANE_FLOPS_PER_PAIR},
           "e2e": {"value": world * ALKANE_SYSTEMS * ALKANE_MOVES / e2e_secs, "unit": "MC move attempts/s",
                   "h2d_bytes_per_step": 16, "d2h_bytes_per_step": ALKANE_SYSTEMS * (8 * 24 + 12)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        start = [a.positions(s) for s in range(ALKANE_SYSTEMS)]
        threads = os.cpu_count() or 1
        _, _, t_probe = oracle.alkane_run(ff, systems, steps=20, seed=3, threads=threads, initial=start)
        steps = int(max(20, 20 * args.cpu_seconds / max(t_probe, 1e-3)))
        _, _, t_cpu = oracle.alkane_run(ff, systems, steps=steps, seed=4, threads=threads, initial=start)
        out["cpu_baseline"] = {"value": ALKANE_SYSTEMS * steps / t_cpu, "unit": "MC move attempts/s",
                               "cores": threads, "kind": "port",
                               "sample": f"64 systems x {steps} moves from the device's equilibrated state in "
                                         f"{t_cpu:.1f} s (FP64 oracle restating the flexible CBMC, one system per "
                                         f"thread)"}
    a.close()
    return out


MIXTURE_EQUIL = 2000
MIXTURE_MOVES = 20000
MIXTURE_BLOCKS_PER_SYSTEM = 4  # CTAs per system in the many-systems run: 37 systems on 148 SMs


def run_mixture(args, ctx, world, rank, dist, torch):
    """The large mixture: 2,000 CO2 + 2,000 N2 in the 18,432-atom framework, Ewald kmax 12
    (8,124 k-vectors), translation : rotation : CBMC swap : identity change = 1 : 1 : 1 : 1 with the learned first-bead
    proposal of each component, one system advanced by all SMs. Metric: move attempts per second."""
    from raspa3_b200 import native
    from raspa3_b200.gcmc import beta_of, fugacity_of
    from raspa3_b200.mixture import large_mixture, total_energy

    d = large_mixture(ctx, torch)
    ff, comps = d["ff"], d["components"]
    beta = beta_of(300.0)
    e0 = total_energy(d["system"], d["ewald"], ff, comps, d["xyz"], d["comp"])
    sk0 = d["ewald"].structure_factors(0)
    # learned first-bead proposals (C of CO2, N of N2), trained on the unit-cell grids
    t0 = time.perf_counter()
    props, mlps = [], []
    for c, comp in enumerate(comps):
        sb = comp.starting_bead
        n = 1 << 20
        ds = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        dt = torch.empty(n, dtype=torch.float32, device="cuda")
        native.sample_targets(d["system"], int(comp.types(ff)[sb]), float(comp.charges(ff)[sb]), beta, -15.0,
                              d["unit_cell"], n, 11 + c, ds.data_ptr(), dt.data_ptr())
        m = native.Mlp(ctx, seed=1 + c)
        m.train(ds.data_ptr(), dt.data_ptr(), n, steps=1500, batch=4096, lr=2e-3)
        props.append(native.Proposal(m, cells_per_axis=48, eps_uniform=0.05))
        mlps.append(m)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    mx = native.Mixture(d["system"], d["ewald"], comps, beta, [fugacity_of(1e5), fugacity_of(1e5)], d["xyz"],
                        d["comp"], max_molecules=6000, seed=3 + rank)
    mx.set_state(e0, sk0)
    for c, pr in enumerate(props):
        mx.set_proposal(c, pr, d["unit_cell"])
    mx.run(MIXTURE_EQUIL, record=False)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0_.record(stream)
    mx.run(MIXTURE_MOVES, record=True)
    e1_.record(stream)
    torch.cuda.synchronize()
    secs = e0_.elapsed_time(e1_) / 1e3
    secs = max_over_ranks(secs, world, dist)
    r = mx.results()
    # e2e: the run call plus the read-back of the statistics
    t1 = time.perf_counter()
    mx.run(MIXTURE_MOVES // 4, record=True)
    r_end = mx.results()
    e2e_secs = time.perf_counter() - t1
    # drift: the running energy after every move so far against a recomputation of the final configuration
    xyz, comp = mx.positions()
    e_check = total_energy(d["system"], d["ewald"], ff, comps, xyz, comp)
    info = mx.info()
    nk = info["n_kvectors"]
    # structure-factor traffic of one move: every CTA reads its S(k) range once per phase and, on acceptance, reads and
    # writes it again (16 bytes each per k-vector); S(k) and temp(k) (8 B) stay in L2
    phases = 1.0 + r["attempted"][2] / max(1, sum(r["attempted"]))  # a second phase for insertions
    acc_frac = sum(r["accepted"]) / max(1, sum(r["attempted"]))
    sk_bytes = nk * (phases * (16 + 8) + acc_frac * 32)
    moves_per_s = world * MIXTURE_MOVES / secs
    hbm = None
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        hbm = None
    out = {"metric": "mixture GCMC steps/s", "value": moves_per_s, "unit": "MC move attempts/s",
           "moves": MIXTURE_MOVES, "ms": secs * 1e3, "blocks": info["blocks"], "n_kvectors": nk,
           "workload": "2,000 CO2 + 2,000 N2 (12,000 sites) in the 4x4x4 replica (18,432 atoms) of the synthetic "
                       "charged cell at 1.5x the 20.0 x 19.9 x 13.4 A lengths, Ewald alpha 0.265 kmax 12, 300 K, 1e5 Pa "
                       "each, translation : rotation : CBMC swap : identity change 1:1:1:1, 10 + 10 trials, learned "
                       "first-bead proposal per component",
           "n_molecules": r["n_molecules"][:2], "attempted": r["attempted"], "accepted": r["accepted"],
           "proposal_training_s": t_train, "status": r["status"],
           "drift_relative": abs(r_end["energy"] - e_check) / max(1.0, abs(e_check)),
           "structure_factor_update": {"bytes_per_move": sk_bytes, "achieved_gbs": sk_bytes * moves_per_s / 1e9,
                                       "hbm_peak_gbs": hbm,
                                       "frac_of_hbm": (sk_bytes * moves_per_s / 1e9 / hbm) if hbm else None,
                                       "note": "the per-move S(k) traffic is L2-resident; the move is latency-bound "
                                               "by its grid barriers, not by memory"},
           "e2e": {"value": world * (MIXTURE_MOVES // 4) / e2e_secs, "unit": "MC move attempts/s",
                   "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 176}}
    # many independent copies of the system at once: one cooperative launch, each copy on MIXTURE_BLOCKS_PER_SYSTEM
    # SMs (rg_mixture_run_many), the way the GPU is used for a batch of systems rather than a single chain
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    n_sys = sms // MIXTURE_BLOCKS_PER_SYSTEM
    many = []
    for s in range(n_sys):
        m = native.Mixture(d["system"], d["ewald"], comps, beta, [fugacity_of(1e5), fugacity_of(1e5)], d["xyz"],
                           d["comp"], max_molecules=6000, seed=100 + 10 * rank + s, n_blocks=MIXTURE_BLOCKS_PER_SYSTEM)
        m.set_state(e0, sk0)
        for c, pr in enumerate(props):
            m.set_proposal(c, pr, d["unit_cell"])
        many.append(m)
    native.Mixture.run_many(many, MIXTURE_EQUIL, record=False)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2_, e3_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2_.record(stream)
    native.Mixture.run_many(many, MIXTURE_MOVES, record=True)
    e3_.record(stream)
    torch.cuda.synchronize()
    secs_many = max_over_ranks(e2_.elapsed_time(e3_) / 1e3, world, dist)
    rm = [m.results() for m in many]
    # e2e: the run_many call plus the read-back of every system's statistics, timed on the host
    t2 = time.perf_counter()
    native.Mixture.run_many(many, MIXTURE_MOVES // 4, record=True)
    rm_end = [m.results() for m in many]
    e2e_many = max_over_ranks(time.perf_counter() - t2, world, dist)
    xyz_m, comp_m = many[0].positions()
    e_many = total_energy(d["system"], d["ewald"], ff, comps, xyz_m, comp_m)
    out["several_systems"] = {
        "systems": n_sys, "blocks_per_system": MIXTURE_BLOCKS_PER_SYSTEM, "moves_per_system": MIXTURE_MOVES,
        "value": world * n_sys * MIXTURE_MOVES / secs_many, "unit": "MC move attempts/s (all systems)",
        "ms": secs_many * 1e3, "status": [r_["status"] for r_ in rm],
        "drift_relative_first_system": abs(rm_end[0]["energy"] - e_many) / max(1.0, abs(e_many)),
        "e2e": {"value": world * n_sys * (MIXTURE_MOVES // 4) / e2e_many, "unit": "MC move attempts/s (all systems)",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 176 * n_sys},
        "path": "rg_mixture_run_many: one cooperative launch, CTAs [s B, (s + 1) B) run system s"}
    for m in many:
        m.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        from concurrent.futures import ThreadPoolExecutor

        host_grids = [None] * (ff.n_types + 1)
        ctx.synchronize()
        for idx, buf in zip(d["grid_types"], d["grids"]):
            host_grids[idx] = buf.cpu().numpy()
        s_fw = d["ewald"].structure_factors(2)
        threads = os.cpu_count() or 1

        def one(seed, steps):
            rr, _, _, s_ = oracle.mixture_run(ff, d["cell"], comps, beta, [fugacity_of(1e5), fugacity_of(1e5)],
                                             d["xyz"], d["comp"], steps, seed=seed, grids=host_grids,
                                             grid_dims=d["dims"], grid_cell=d["unit_cell"], s_framework=s_fw,
                                             max_molecules=6000)
            return s_

        t_probe = one(1, 20)
        steps = int(max(20, 20 * args.cpu_seconds / max(t_probe, 1e-3)))
        with ThreadPoolExecutor(threads) as pool:
            secs_cpu = list(pool.map(lambda s: one(s + 2, steps), range(threads)))
        out["cpu_baseline"] = {"value": threads * steps / max(secs_cpu), "unit": "MC move attempts/s",
                               "cores": threads, "kind": "port",
                               "sample": f"{threads} independent copies x {steps} moves from the same starting "
                                         f"configuration (FP64 oracle mixture GCMC, one copy per thread, uniform "
                                         f"first beads) in {max(secs_cpu):.1f} s"}
    mx.close()
    for pr in props:
        pr.close()
    for m in mlps:
        m.close()
    return out


LEARNED_SAMPLES = 1 << 22
LEARNED_TRAIN_STEPS = 3000
LEARNED_EQUIL = 4000
LEARNED_MOVES = 40000


def run_learned(args, ctx, world, rank, dist, torch):
    """Learned vs uniform first-bead proposal: CO2 at 300 K and 1e6 Pa in the 2x2x3 box of the
    synthetic framework, with the framework charges set to zero (with them the binding wells of about -1e4 K make the
    system non-ergodic for every sampler); CO2 keeps its charges, Ewald on. The MLP is trained on 2^22 grid-sampled
    Boltzmann factors of the C atom. Both arms run the same number of chains and moves; the statistical error of the
    loading is the standard error over independent chains. GPU-seconds to reach the uniform run's error:
    t_train + t_learned * (se_learned / se_uniform)^2, against t_uniform."""
    from raspa3_b200 import native
    from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of
    from raspa3_b200.synthetic import spacing_grid_dims, replicate, synthetic_forcefield, synthetic_framework

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=8)
    for pa in ff.pseudo_atoms[:2]:
        pa.charge = 0.0
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = spacing_grid_dims(ucell)
    stream = torch.cuda.current_stream()
    sysg = native.System(ctx, ff, scell, sfw)
    keep = []
    for idx, gt in ((ff.index("C_co2"), 0), (ff.index("O_co2"), 0), (ff.n_types, 1)):
        buf = torch.empty(8 * dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
        ctx.grid_build(gt, ff, ucell, ufw, idx if gt == 0 else 0, 12.0, dims, native.PRECISION_FP32C,
                       out_device=buf.data_ptr(), host=False)
        sysg.set_grid(idx, ucell, dims, buf.data_ptr(), on_device=True)
        keep.append(buf)
    ew = native.Ewald(ctx, ff, scell)
    ew.set_framework(sfw)
    beta = beta_of(300.0)
    comp = co2_component()
    c_atom = comp.starting_bead
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    chains = GCMC_CHAINS_PER_SM * sms

    def timed(fn, host=False):
        # device time between two events on the stream; host=True: wall time of a call that mixes host and device work
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, (time.perf_counter() - t0) if host else e0.elapsed_time(e1) / 1e3

    # training: target sampling from the grids, MLP training, tabulation of the proposal density
    n = LEARNED_SAMPLES
    ds = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    dt = torch.empty(n, dtype=torch.float32, device="cuda")
    # untimed warm-up of the four kernels (their first launch in a process loads them)
    w = native.Mlp(ctx, seed=2)
    native.sample_targets(sysg, int(comp.types(ff)[c_atom]), float(comp.charges(ff)[c_atom]), beta, -15.0, ucell,
                          4096, 9, ds.data_ptr(), dt.data_ptr())
    w.train(ds.data_ptr(), dt.data_ptr(), 4096, steps=2, batch=4096, lr=2e-3)
    native.Proposal(w, cells_per_axis=4, eps_uniform=0.05).close()
    w.close()
    m = native.Mlp(ctx, seed=1)
    _, t_sample = timed(lambda: native.sample_targets(sysg, int(comp.types(ff)[c_atom]), float(comp.charges(ff)[c_atom]),
                                                      beta, -15.0, ucell, n, 9, ds.data_ptr(), dt.data_ptr()))
    loss, t_fit = timed(lambda: m.train(ds.data_ptr(), dt.data_ptr(), n, steps=LEARNED_TRAIN_STEPS, batch=4096,
                                        lr=2e-3))
    prop, t_table = timed(lambda: native.Proposal(m, cells_per_axis=48, eps_uniform=0.05), host=True)
    t_train = t_sample + t_fit + t_table

    arms = {}
    for name, use in (("uniform", False), ("learned", True)):
        g = native.Gcmc(sysg, ew, comp, beta, fugacity_of(1e6), n_chains=chains, seed=(31 if use else 32) + 100 * rank)
        if use:
            g.set_proposal(prop, ucell)
        g.run(LEARNED_EQUIL, record=False)
        _, secs = timed(lambda: g.run(LEARNED_MOVES, record=True))
        res = g.results()
        g.close()
        means = np.array([r["sum_n"] / r["samples"] for r in res])
        emeans = np.array([r["sum_energy"] / r["samples"] for r in res])
        blocks = np.array([r["block_n"] for r in res], dtype=np.float64)
        acc = np.sum([r["accepted"] for r in res], axis=0)
        att = np.sum([r["attempted"] for r in res], axis=0)
        arms[name] = {"gpu_seconds": secs, "loading": float(means.mean()),
                      "loading_se": float(means.std(ddof=1) / np.sqrt(len(means))),
                      "loading_block_se": float(blocks.mean(axis=0).std(ddof=1) / np.sqrt(blocks.shape[1])),
                      "energy_K": float(emeans.mean()), "energy_se_K": float(emeans.std(ddof=1) / np.sqrt(len(means))),
                      "swap_acceptance": float((acc[2] + acc[3]) / max(1, att[2] + att[3])),
                      "moves_per_s": chains * LEARNED_MOVES / secs}
    u, l = arms["uniform"], arms["learned"]
    var_ratio = (l["loading_se"] / u["loading_se"]) ** 2
    t_equal = t_train + l["gpu_seconds"] * var_ratio
    out = {"metric": "GPU-seconds to equal loading error, learned vs uniform first-bead proposal",
           "workload": "CO2 (charged, Ewald alpha 0.265 kmax 8) at 300 K and 1e6 Pa in the 2x2x3 box of the synthetic "
                       "framework with framework charges off, 133x133x89 FP32C grids; MLP 96-64-64-1 SiLU trained on "
                       f"2^22 grid Boltzmann factors, proposal tabulated on 48^3 cells with 5% uniform mixing; "
                       f"{chains} chains x {LEARNED_MOVES} moves after {LEARNED_EQUIL} equilibration moves per arm",
           "train": {"sample_s": t_sample, "fit_s": t_fit, "table_s": t_table, "total_s": t_train,
                     "final_loss": loss, "steps": LEARNED_TRAIN_STEPS, "batch": 4096},
           "uniform": u, "learned": l,
           "loading_difference_sigmas": abs(l["loading"] - u["loading"]) / float(np.hypot(u["loading_se"],
                                                                                           l["loading_se"])),
           "sampling_efficiency_ratio": u["gpu_seconds"] / (l["gpu_seconds"] * var_ratio),
           "learned_seconds_to_uniform_error": t_equal,
           "speedup_at_equal_error_incl_training": u["gpu_seconds"] / t_equal}
    prop.close()
    m.close()
    ew.close()
    sysg.close()
    return out


VALIDATION_POINTS = 100000  # the reference's default NumberOfGridTestPoints (forcefield.ixx:172)


def run_grid_validation(args, ctx, ff, cell, atoms, dims, outs, rank, world, native):
    """The grid test that System::createFrameworkInterpolationGrids runs after each build, on the device: the C_co2
    grid just built (FP32C) and its charge term (+0.70 e x the unit-charge Ewald grid) at 100,000 points of the 2x2x3
    box, weighted as at 300 K. CPU baseline: the oracle of the same test on a sample of points, one core (the reference's
    test is serial)."""
    import torch

    scell, _ = gcmc_setup(ff, cell, atoms)
    probe = ff.index("C_co2")
    kw = dict(probe_charge=0.70, weight_beta=1.0 / 300.0, n_points=VALIDATION_POINTS)
    ctx.grid_validate(ff, cell, atoms, scell, probe, dims, outs[0].data_ptr(), outs[2].data_ptr(), seed=1, **kw)
    reps = 5
    t0 = time.perf_counter()
    for r in range(reps):
        res = ctx.grid_validate(ff, cell, atoms, scell, probe, dims, outs[0].data_ptr(), outs[2].data_ptr(), seed=2 + r,
                                **kw)
    secs = (time.perf_counter() - t0) / reps
    out = {"metric": "grid test points/s through rg_grid_validate", "value": VALIDATION_POINTS / secs,
           "unit": "points/s", "ms": 1e3 * secs, "points": VALIDATION_POINTS,
           "energy_relative_error": res["energy_relative_error"],
           "charge_energy_relative_error": res["charge_energy_relative_error"],
           "gradient_relative_error": res["gradient_relative_error"],
           "workload": "C_co2 FP32C grid of the charged synthetic framework with its charge term, 2x2x3 box, weights at 300 K"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        torch.cuda.synchronize()
        ctx.synchronize()
        host = [outs[0].cpu().numpy(), outs[2].cpu().numpy()]
        pts = np.random.default_rng(5).random((200, 3))
        t0 = time.perf_counter()
        oracle.grid_validate(ff, cell, atoms, scell, probe, dims, host[0], host[1], 0.70, 1.0 / 300.0, pts[:20])
        one = (time.perf_counter() - t0) / 20
        n = int(max(20, min(20000, args.cpu_seconds / 2 / max(one, 1e-6))))
        pts = np.random.default_rng(5).random((n, 3))
        t0 = time.perf_counter()
        oracle.grid_validate(ff, cell, atoms, scell, probe, dims, host[0], host[1], 0.70, 1.0 / 300.0, pts)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / t, "unit": "points/s", "cores": 1, "kind": "port",
                               "sample": f"{n} points in {t:.1f} s (FP64 oracle of the reference's grid test, one core)"}
    return out


TRIQUINTIC_STEPS = 5
# FP64 FLOPs per in-cutoff pair of the rectangular Lennard-Jones triquintic formula as evaluated (add/mul = 1,
# FMA = 2, reciprocal = 1): distance 8, radial factors F0..F6 45, axis powers 6, the 20 non-trivial monomials 20,
# factor-monomial products 50, and 64 channel terms as FMAs 128
TRIQUINTIC_FLOPS_PER_PAIR = 257


def run_triquintic(args, ctx, ff, cell, atoms, dims, world, rank, dist, torch):
    """Triquintic grid (27 values per point, FP64) of the C_co2 Lennard-Jones probe on the charged synthetic framework and
    grid (133 x 133 x 89 points, 340 MB): grid points/s with the output on the device (CUDA events; each output is
    larger than L2), end to end with a pinned host output, and the FP64 roofline of the kernel. CPU baseline: the
    oracle of the reference's triquintic branch on a sample of points, all host cores."""
    from raspa3_b200 import native

    probe = ff.index("C_co2")
    npts = dims[0] * dims[1] * dims[2]
    out = torch.empty(27 * npts, dtype=torch.float64, device="cuda")
    _, st = ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                                      out_device=out.data_ptr(), host=False, count_pairs=True)
    stream = torch.cuda.current_stream()
    for _ in range(2):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                                  out_device=out.data_ptr(), host=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(TRIQUINTIC_STEPS):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                                  out_device=out.data_ptr(), host=False)
    e1.record(stream)
    e1.synchronize()
    secs = max_over_ranks(e0.elapsed_time(e1) / 1e3 / TRIQUINTIC_STEPS, world, dist)
    # the same grid with FP32 pair terms and compensated sums (RG_TRIQUINTIC_FP32C)
    for _ in range(2):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                                  out_device=out.data_ptr(), host=False, fp32c=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(TRIQUINTIC_STEPS):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                                  out_device=out.data_ptr(), host=False, fp32c=True)
    e1.record(stream)
    e1.synchronize()
    secs32 = max_over_ranks(e0.elapsed_time(e1) / 1e3 / TRIQUINTIC_STEPS, world, dist)
    host = torch.empty(27 * npts, dtype=torch.float64, pin_memory=True).numpy()
    # untimed warm-up of the end-to-end call (first copies into freshly pinned pages)
    ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                              out_device=out.data_ptr(), out_host=host)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(2):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims,
                                  out_device=out.data_ptr(), out_host=host)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / 2, world, dist)
    peak64 = ctx.probe_fma_peak(native.PRECISION_FP64)
    tflops = st["pair_count"] * TRIQUINTIC_FLOPS_PER_PAIR / secs / 1e12
    res = {"metric": "triquintic grid pts/s through rg_grid_build_triquintic", "unit": "grid points/s",
           "value": whole_job_rate(npts, world, secs), "ms": 1e3 * secs,
           "workload": "C_co2 Lennard-Jones triquintic grid (27 channels, FP64) of the charged synthetic framework, 133 x 133 x 89 "
                       "points, 340 MB",
           "pairs": st["pair_count"], "pairs_per_s": st["pair_count"] / secs,
           "roofline": {"bound": "fp64", "achieved": tflops, "peak": peak64, "unit": "TFLOP/s",
                        "frac": tflops / peak64 if peak64 else None, "flops_per_pair": TRIQUINTIC_FLOPS_PER_PAIR,
                        "peak_source": "rg_probe_fma_peak FP64, measured in this run"},
           "fp32c": {"value": whole_job_rate(npts, world, secs32), "ms": 1e3 * secs32,
                     "note": "RG_TRIQUINTIC_FP32C: FP32 pair terms, compensated FP32 sums, FP64 epilogue"},
           "e2e": {"value": whole_job_rate(npts, world, e2e_s), "unit": "grid points/s",
                   "h2d_bytes_per_step": st["h2d_bytes"], "d2h_bytes_per_step": 27 * 8 * npts}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        threads = os.cpu_count() or 1
        rng = np.random.default_rng(6)
        n = 16 * threads
        pts = np.sort(rng.choice(npts, size=n, replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        oracle.make_grid_triquintic(0, ff, cell, atoms, probe, 12.0, dims, points=pts, threads=threads)
        t = time.perf_counter() - t0
        n = int(min(npts, n * max(1.0, args.cpu_seconds / 2 / max(t, 1e-3))))
        pts = np.sort(rng.choice(npts, size=n, replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        oracle.make_grid_triquintic(0, ff, cell, atoms, probe, 12.0, dims, points=pts, threads=threads)
        t = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": n / t, "unit": "grid points/s", "cores": threads, "kind": "port",
                               "sample": f"{n} random grid points in {t:.1f} s (FP64 oracle of the triquintic branch "
                                         f"of makeFrameworkInterpolationGrid, OpenMP over points)"}
    return res


PATH_INSERTIONS = 200   # CBMC insertions whose trial sets go through rg_cbmc_external_energies, per precision
PATH_DELTAS = 1000      # Ewald Fourier differences through rg_ewald_delta, per box
PATH_FULL = 20          # full structure-factor recomputes through rg_ewald_full
EWALD_FLOPS_PER_TERM = 16  # one (atom, k) term of the full recompute: two complex products + a complex multiply-add


EWALD_BATCH_SYSTEMS = 1184
EWALD_BATCH_STEPS = 20


def run_ewald_batch(args, ctx, world, rank, dist, torch):
    """Path (c) batched: the Fourier energy difference of one CO2 translation in each of 1,184 systems that share the
    large-mixture box and k-vectors (kmax 12, the full half-box, 8,124 k-vectors), one rg_ewald_batch_delta call per
    step: every system's S(k) read and its trial S(k) written (32 bytes per k-vector and system), the HBM roofline of
    the structure-factor update."""
    from raspa3_b200 import native
    from raspa3_b200.mixture import MIXTURE_CELL
    from raspa3_b200.synthetic import random_molecules, synthetic_forcefield

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=12, sphere=False)
    cell = np.diag([4 * MIXTURE_CELL[0], 4 * MIXTURE_CELL[1], 4 * MIXTURE_CELL[2]])
    ew = native.Ewald(ctx, ff, cell)
    nk = ew.n_kvectors
    n_sys = EWALD_BATCH_SYSTEMS
    batch = native.EwaldBatch(ew, n_sys)
    mols = random_molecules(ff, cell, 200, seed=5)
    ew.full(mols, [3] * 200)
    for sy in range(n_sys):
        batch.set(sy)
    rng = np.random.default_rng(8)

    def moves():
        out = []
        for sy in range(n_sys):
            m = int(rng.integers(200))
            old = mols[3 * m:3 * m + 3]
            new = old.copy()
            d = rng.normal(size=3) * 0.5
            for i, k in enumerate("xyz"):
                new[k] += d[i]
            out.append(np.concatenate([new, old]))
        return np.concatenate(out)

    steps_atoms = [moves() for _ in range(4)]
    previous = ctx.stream
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    for w in range(max(3, args.warmup)):
        batch.delta(steps_atoms[w % 4], 6, [3] * n_sys, [3] * n_sys)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(EWALD_BATCH_STEPS)]
    kernel_ms, upload_ms = [], []
    t0 = time.perf_counter()
    for i, (a, b) in enumerate(ev):
        with torch.cuda.stream(stream):
            a.record(stream)
            batch.delta(steps_atoms[i % 4], 6, [3] * n_sys, [3] * n_sys)
            b.record(stream)
        up, kern = batch.timing()  # CUDA events around the upload and the kernel, on the same stream
        upload_ms.append(up)
        kernel_ms.append(kern)
    torch.cuda.synchronize()
    host_s = time.perf_counter() - t0
    call_ms = statistics.mean(x.elapsed_time(y) for x, y in ev)
    dev_ms = statistics.mean(kernel_ms)
    ctx.set_stream(previous or None)
    host_s = max_over_ranks(host_s, world, dist)
    sk_bytes = n_sys * nk * 32
    atom_bytes = n_sys * 6 * 48
    hbm = None
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        hbm = None
    gbs = sk_bytes / (dev_ms * 1e-3) / 1e9
    out = {"workload": f"{n_sys} systems x one CO2 translation, {nk} k-vectors (kmax 12, the full half-box), "
                       "large-mixture box, one rg_ewald_batch_delta call per step",
           "value": world * n_sys / (dev_ms * 1e-3), "unit": "Fourier differences/s",
           "ms_per_step": dev_ms, "steps": EWALD_BATCH_STEPS,
           "value_note": "the update kernel's device time with the moved atoms already on the device (CUDA events "
                         "around the kernel inside rg_ewald_batch_delta, read by rg_ewald_batch_timing)",
           "upload_ms": statistics.mean(upload_ms), "call_ms": call_ms,
           "roofline": {"kernel": "ewaldBatchDeltaKernel", "bound": "hbm", "achieved": gbs, "peak": hbm,
                        "unit": "GB/s", "frac": (gbs / hbm) if hbm else None,
                        "bytes_per_step": sk_bytes, "bytes_note": "32 B per k-vector and system: read S(k), write the "
                        "trial S(k), over the kernel's own duration",
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
           "e2e": {"value": world * n_sys * EWALD_BATCH_STEPS / host_s, "unit": "Fourier differences/s",
                   "h2d_bytes_per_step": atom_bytes, "d2h_bytes_per_step": 8 * n_sys,
                   "path": "rg_ewald_batch_delta with host atoms and host results"}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        from concurrent.futures import ThreadPoolExecutor

        _, stored = oracle.ewald_fourier_energy(ff, cell, mols, [3] * 200)
        threads = os.cpu_count() or 1
        atoms = steps_atoms[0]
        per = max(1, int(8 * args.cpu_seconds / 12.0))

        def one(t):
            for j in range(per):
                sy = (t * per + j) % n_sys
                a = atoms[6 * sy:6 * sy + 6]
                oracle.ewald_delta(ff, cell, stored, a[:3], a[3:])

        one(0)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as pool:
            list(pool.map(one, range(threads)))
        secs = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": threads * per / secs, "unit": "Fourier differences/s", "cores": threads,
                               "kind": "port", "sample": f"{threads * per} differences, one system per thread "
                                                         f"(FP64 oracle of energyDifferenceEwaldFourier) in {secs:.1f} s"}
    batch.close()
    ew.close()
    return out


def run_paths(args, ctx, world, rank, dist, torch):
    """Paths (b) and (c) on their own, through their C-ABI entry points with host buffers, on the large-mixture
    system (18,432 framework atoms, 2,000 CO2 + 2,000 N2, Ewald kmax 12: 8,124 k-vectors):
    (b) the trial sets of one CBMC insertion of CO2 (10 first-bead C positions, then 10 orientations whose two O atoms
        are the trial atoms), each trial atom against the grids and the 12,000 adsorbate sites, in FP64 and FP32C;
    (c) the Ewald Fourier difference of a CO2 translation (3 new + 3 old atoms) at the large-mixture box (8,124 k-vectors) and at the
        charged 2x2x3 box (1,152 k-vectors), and the full recompute of the large mixture's structure factors."""
    from raspa3_b200 import native
    from raspa3_b200.forcefield import make_atoms
    from raspa3_b200.mixture import large_mixture, molecules_as_atoms
    from raspa3_b200.synthetic import (CO2_NAMES, CO2_OFFSETS, random_molecules, random_rotation, replicate,
                                       rigid_molecule, synthetic_forcefield, synthetic_framework)

    d = large_mixture(ctx, torch)
    ff, comps, sysg, ew = d["ff"], d["components"], d["system"], d["ewald"]
    atoms = molecules_as_atoms(ff, comps, d["xyz"], d["comp"])
    n_mol = len(d["comp"])
    sysg.set_molecules(atoms)
    rng = np.random.default_rng(17)
    q_c = float(ff.pseudo_atoms[ff.index("C_co2")].charge)
    inserts = []
    for _ in range(PATH_INSERTIONS):
        first = make_atoms(rng.random((10, 3)) @ d["cell"], ff.index("C_co2"), q_c, molecule_ids=np.full(10, n_mol))
        centre = first[int(rng.integers(10))]
        c = np.array([centre["x"], centre["y"], centre["z"]])
        orient = np.concatenate([rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, c, random_rotation(rng), n_mol)
                                 for _ in range(10)])
        inserts.append((first, orient))
    trial_atoms = 10 + 10 * 2
    stream = torch.cuda.current_stream()
    out = {"workload": "large mixture: 18,432 framework atoms, 12,000 adsorbate sites, grids for every adsorbate "
                       "type, Ewald alpha 0.265 kmax 12 (8,124 k)"}

    def time_trials():
        for first, orient in inserts[:3]:
            sysg.external_energies(first, 1)
            sysg.external_energies(orient, 3, skip=1)
        dev = 0.0
        t0 = time.perf_counter()
        for first, orient in inserts:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sysg.external_energies(first, 1)
            sysg.external_energies(orient, 3, skip=1)
            e1.record(stream)
            e1.synchronize()
            dev += e0.elapsed_time(e1) / 1e3
        return time.perf_counter() - t0, dev

    trials = {}
    for name, prec in (("fp64", native.PRECISION_FP64), ("fp32c", native.PRECISION_FP32C)):
        sysg.set_precision(prec)
        wall, dev = time_trials()
        tests = PATH_INSERTIONS * trial_atoms * len(atoms)
        trials[name] = {"insertions_per_s": PATH_INSERTIONS / wall, "pair_tests_per_s": tests / wall,
                        "device_pair_tests_per_s": tests / dev, "ms_per_insertion": 1e3 * wall / PATH_INSERTIONS}
    sysg.set_precision(native.PRECISION_FP64)
    out["trial_energies"] = {
        "metric": "CBMC trial-atom x partner pair tests/s through rg_cbmc_external_energies", "unit": "pair tests/s",
        "value": trials["fp32c"]["pair_tests_per_s"], "per_precision": trials,
        "per_insertion": "10 first-bead sets of 1 atom + 10 orientation sets of 2 atoms, 12,000 partners each, two "
                         "calls with host buffers",
        "e2e": {"value": trials["fp32c"]["pair_tests_per_s"], "unit": "pair tests/s",
                "h2d_bytes_per_step": trial_atoms * 64 + 20 * 64, "d2h_bytes_per_step": 20 * 104}}

    # (c) Fourier differences: the large-mixture box and the charged 2x2x3 box
    ew.full(atoms, np.full(n_mol, 3, dtype=np.int32))
    ff2 = synthetic_forcefield(charges=True, alpha=0.265, kmax=8)
    ucell2, ufw2 = synthetic_framework(ff2, seed=42)
    cell2, fw2 = replicate(ucell2, ufw2, (2, 2, 3))
    ew2 = native.Ewald(ctx, ff2, cell2)
    ew2.set_framework(fw2)
    ads2 = random_molecules(ff2, cell2, 30, seed=8)
    ew2.full(ads2, np.full(30, 3, dtype=np.int32))

    def moves(a, n, count):
        mv = []
        for _ in range(count):
            m = int(rng.integers(n))
            old = a[3 * m:3 * m + 3].copy()
            new = old.copy()
            step = (rng.random(3) - 0.5) * 2.0
            new["x"] += step[0]
            new["y"] += step[1]
            new["z"] += step[2]
            mv.append((new, old))
        return mv

    deltas = {}
    for name, e_, a_, n_ in (("large_mixture_8124k", ew, atoms, n_mol), ("charged_box_1152k", ew2, ads2, 30)):
        mv = moves(a_, n_, PATH_DELTAS)
        for new, old in mv[:10]:
            e_.delta(new, old)
        t0 = time.perf_counter()
        for new, old in mv:
            e_.delta(new, old)
        wall = time.perf_counter() - t0
        # the C-ABI call alone, as a C++ caller makes it: its atom arrays and result struct exist before the loop, so
        # the timed loop holds only rg_ewald_delta (atom packing, launch, kernel, synchronisation, host terms)
        fn = native.lib().rg_ewald_delta
        res = native.EwaldEnergy()
        ref = ctypes.byref(res)
        prepared = [(ctypes.c_void_p(n_.ctypes.data), len(n_), ctypes.c_void_p(o_.ctypes.data), len(o_))
                    for n_, o_ in mv]
        handle = e_.handle
        for pn, nn, po, no in prepared[:10]:
            fn(handle, pn, nn, po, no, 0.0, None, ref)
        status = 0
        t0 = time.perf_counter()
        for pn, nn, po, no in prepared:
            status |= fn(handle, pn, nn, po, no, 0.0, None, ref)
        direct = time.perf_counter() - t0
        if status:
            raise RuntimeError("rg_ewald_delta failed in the timed loop")
        nk = e_.n_kvectors
        deltas[name] = {"n_kvectors": nk, "deltas_per_s": PATH_DELTAS / direct, "us_per_delta": 1e6 * direct / PATH_DELTAS,
                        "python_wrapper_us_per_delta": 1e6 * wall / PATH_DELTAS,
                        "algorithmic_bytes_per_delta": 40 * nk,
                        "achieved_gbs": 40 * nk * PATH_DELTAS / direct / 1e9}
    # full recompute of the large mixture (adsorbates on top of the rigid framework structure factor)
    sizes = np.full(n_mol, 3, dtype=np.int32)
    for _ in range(2):
        ew.full(atoms, sizes)
    t0 = time.perf_counter()
    for _ in range(PATH_FULL):
        ew.full(atoms, sizes)
    full_s = (time.perf_counter() - t0) / PATH_FULL
    terms = len(atoms) * ew.n_kvectors
    peak64 = ctx.probe_fma_peak(native.PRECISION_FP64)
    full_tf = terms * EWALD_FLOPS_PER_TERM / full_s / 1e12
    out["ewald"] = {
        "metric": "Ewald Fourier differences/s through rg_ewald_delta", "unit": "differences/s",
        "value": deltas["large_mixture_8124k"]["deltas_per_s"], "per_box": deltas,
        "full_recompute": {"atoms": len(atoms), "n_kvectors": ew.n_kvectors, "ms": 1e3 * full_s,
                           "terms_per_s": terms / full_s, "tflops": full_tf, "fp64_peak_tflops": peak64,
                           "frac_of_fp64_peak": full_tf / peak64 if peak64 else None,
                           "flops_per_term": EWALD_FLOPS_PER_TERM,
                           "includes": "host packing of the atoms, their upload, both kernels and the host self / "
                                       "exclusion sums"},
        "note": "one difference reads S(k) and temp(k) and writes the trial S(k): 40 B per k, L2-resident at both "
                "sizes (130 KB at 8,124 k), so a single difference is latency-bound and its GB/s is far below HBM"}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        from concurrent.futures import ThreadPoolExecutor

        threads = os.cpu_count() or 1
        host_grids = [None] * (ff.n_types + 1)
        ctx.synchronize()
        for idx, buf in zip(d["grid_types"], d["grids"]):
            host_grids[idx] = buf.cpu().numpy()

        def cpu_insertion(k):
            first, orient = inserts[k % len(inserts)]
            for t in range(10):
                oracle.cbmc_framework_molecule(ff, d["cell"], np.zeros(0, dtype=atoms.dtype), first[t:t + 1],
                                               ff.cutoff_framework_vdw, ff.cutoff_coulomb, grids=host_grids,
                                               grid_dims=d["dims"], grid_cell=d["unit_cell"])
                oracle.cbmc_intermolecular(ff, d["cell"], atoms, first[t:t + 1], ff.cutoff_molecule_vdw,
                                           ff.cutoff_coulomb)
            for t in range(10):
                s3 = orient[3 * t:3 * t + 3]
                oracle.cbmc_framework_molecule(ff, d["cell"], np.zeros(0, dtype=atoms.dtype), s3,
                                               ff.cutoff_framework_vdw, ff.cutoff_coulomb, grids=host_grids,
                                               grid_dims=d["dims"], grid_cell=d["unit_cell"], skip=1)
                oracle.cbmc_intermolecular(ff, d["cell"], atoms, s3, ff.cutoff_molecule_vdw, ff.cutoff_coulomb,
                                           skip=1)

        t0 = time.perf_counter()
        cpu_insertion(0)
        one = time.perf_counter() - t0
        per_thread = max(1, int(args.cpu_seconds / 2 / max(one, 1e-3)))
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as pool:
            list(pool.map(cpu_insertion, range(threads * per_thread)))
        secs = time.perf_counter() - t0
        tests = threads * per_thread * trial_atoms * len(atoms)
        out["trial_energies"]["cpu_baseline"] = {
            "value": tests / secs, "unit": "pair tests/s", "cores": threads, "kind": "port",
            "sample": f"{threads * per_thread} insertions' trial sets in {secs:.1f} s (FP64 oracle of "
                      f"computeFrameworkMoleculeEnergy + computeInterMolecularEnergy, one insertion per thread)"}
        # the oracle's Fourier difference: (i) one core, the reference's serial k loop (a single system's move is serial
        # there); (ii) all host cores, the same loop parallelised over k by us (OpenMP over a precomputed k table)
        cpu_d, cpu_all = {}, {}
        for name, ff_, cell_, a_, n_, fw_ in (("large_mixture_8124k", ff, d["cell"], atoms, n_mol, d["framework"]),
                                              ("charged_box_1152k", ff2, cell2, ads2, 30, fw2)):
            s_rig = oracle.ewald_rigid(ff_, cell_, fw_)
            _, stored = oracle.ewald_fourier_energy(ff_, cell_, a_, np.full(n_, 3, dtype=np.int32), s_rigid=s_rig)
            mv = moves(a_, n_, 1000)
            par = oracle.EwaldDeltaParallel(ff_, cell_, threads)
            for target, fn in ((cpu_d, lambda new, old: oracle.ewald_delta(ff_, cell_, stored, new, old)),
                               (cpu_all, lambda new, old: par(stored, new, old))):
                count = 0
                t0 = time.perf_counter()
                while time.perf_counter() - t0 < args.cpu_seconds / 8:
                    new, old = mv[count % len(mv)]
                    fn(new, old)
                    count += 1
                target[name] = count / (time.perf_counter() - t0)
        out["ewald"]["cpu_baseline"] = {
            "value": cpu_d["large_mixture_8124k"], "unit": "differences/s", "cores": 1, "kind": "port",
            "per_box": cpu_d, "sample": "FP64 oracle of energyDifferenceEwaldFourier on one core, same moves",
            "all_cores": {"cores": threads, "per_box": cpu_all,
                          "sample": "the same k loop parallelised over k with OpenMP (restated reference loop, "
                                    "parallelised by us), same moves"}}
    ew2.close()
    return out


def cpu_gcmc_rate(ff, cell, scell, sfw, dims, grids, outs, target_seconds):
    """The oracle GCMC (the reference's moves restated) on all host cores, one chain per core, same grids."""
    import oracle
    from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of

    threads = os.cpu_count() or 1
    host_grids = [None] * (ff.n_types + 1)
    for (name, gt, probe), out in zip(grids, outs):
        host_grids[probe if gt == 0 else ff.n_types] = out.cpu().numpy()
    s_fw = oracle.ewald_rigid(ff, scell, sfw)
    kw = dict(grids=host_grids, grid_dims=dims, grid_cell=cell, s_framework=s_fw, threads=threads)
    _, t0 = oracle.gcmc_run(ff, scell, co2_component(), beta_of(300.0), fugacity_of(1e5), n_chains=threads,
                            steps=200, equilibration=0, seed=3, **kw)
    steps = int(max(200, 200 * target_seconds / max(t0, 1e-3)))
    _, t1 = oracle.gcmc_run(ff, scell, co2_component(), beta_of(300.0), fugacity_of(1e5), n_chains=threads,
                            steps=steps, equilibration=0, seed=4, **kw)
    return {"value": threads * steps / t1, "unit": "MC move attempts/s", "cores": threads, "kind": "port",
            "sample": f"{threads} chains x {steps} moves from an empty box in {t1:.1f} s (FP64 oracle GCMC, one chain "
                      f"per thread)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle

    # the reference's release flags (-O3 -ffast-math) and -march=native, compiled here for this host's CPU
    oracle.use_release_build()
    ff, cell, atoms, dims, grids = workload()
    threads = os.cpu_count() or 1
    # size one step so that W + K steps take a few minutes at most
    per_step = max(2.0, min(8.0, 150.0 / max(1, args.steps + args.warmup)))
    rate0, _, _, _ = cpu_oracle_rate(ff, cell, atoms, dims, grids, 1.0, threads)
    n_pts = max(256, int(rate0 * per_step / len(grids)))
    rng = np.random.default_rng(99)
    total = dims[0] * dims[1] * dims[2]
    done, secs = 0, 0.0
    for s in range(args.warmup + args.steps):
        pts = np.sort(rng.choice(total, size=min(n_pts, total), replace=False)).astype(np.int64)
        t0 = time.perf_counter()
        for _, gt, probe in grids:
            oracle.make_grid(gt, ff, cell, atoms, probe, 12.0, dims, points=pts, threads=threads)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            done += len(pts) * len(grids)
            secs += dt
    value = done / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "grid build: C_co2-LJ + O_co2-LJ + unit-charge Ewald-real tricubic grids, "
                               "133x133x89 points each", "grid_points_per_step_full": 3 * total,
                   "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n_pts} random grid points x 3 grids per step (FP64 oracle restating "
                                   f"makeFrameworkInterpolationGrid, release flags -O3 -ffast-math -march=native, "
                                   f"OpenMP over points)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    from raspa3_b200 import native

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # every CPU baseline below runs the oracle built with the reference's release flags (-O3 -ffast-math) and
        # -march=native for this host; the strict build stays the parity oracle of the tests
        import oracle

        oracle.use_release_build()
    ff, cell, atoms, dims, grids = workload()
    npts = dims[0] * dims[1] * dims[2]
    ctx = native.Context(local)
    # a created stream (not the legacy NULL stream) shared by the library and the timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    outs = [torch.empty(8 * npts, dtype=torch.float64, device="cuda") for _ in grids]
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    # one step = two calls of the grid-set entry point: the two Lennard-Jones grids (one two-probe kernel) and the
    # unit-charge Ewald grid
    calls = [[0, 1], [2]]
    call_names = ["LJ C_co2+O_co2 (two-probe kernel)", "Ewald-real"]

    def build_call(ci, out_host=None, count=False):
        idx = calls[ci]
        return ctx.grid_build_set(ff, cell, atoms, 12.0, dims, native.PRECISION_FP32C, [grids[g][1] for g in idx],
                                  [grids[g][2] for g in idx], [outs[g].data_ptr() for g in idx], count_pairs=count,
                                  out_host=None if out_host is None else [out_host[g] for g in idx])

    # work per grid (pair counts) outside the timed region
    stats = [None] * len(grids)
    for ci, idx in enumerate(calls):
        for g, st in zip(idx, build_call(ci, count=True)):
            stats[g] = st
    peak_fp32 = ctx.probe_fma_peak(native.PRECISION_FP32C)

    for _ in range(args.warmup):
        for ci in range(len(calls)):
            build_call(ci)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(calls) + 1)] for _ in range(args.steps)]
    for s in range(args.steps):
        flush.zero_()
        ev[s][0].record(stream)
        for ci in range(len(calls)):
            build_call(ci)
            ev[s][ci + 1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = [ev[s][0].elapsed_time(ev[s][-1]) for s in range(args.steps)]
    kern_ms = [[ev[s][c].elapsed_time(ev[s][c + 1]) for s in range(args.steps)] for c in range(len(calls))]
    total_s = sum(step_ms) / 1e3
    total_s = max_over_ranks(total_s, world, dist)
    value = whole_job_rate(len(grids) * npts * args.steps, world, total_s)

    # e2e through the C-ABI with pinned host output buffers (framework upload + grid download inside the region)
    e2e_steps = max(1, min(args.steps, 5))
    host_bufs = [torch.empty(8 * npts, dtype=torch.float64, pin_memory=True) for _ in grids]
    host_np = [b.numpy() for b in host_bufs]
    # untimed warm-up of the same call: the first copies into freshly pinned pages are several times slower
    for _ in range(max(1, min(args.warmup, 2))):
        ctx.grid_build_set(ff, cell, atoms, 12.0, dims, native.PRECISION_FP32C, [g[1] for g in grids],
                           [g[2] for g in grids], [outs[g].data_ptr() for g in range(len(grids))], out_host=host_np)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    # per step: the framework images uploaded by each call (as counted above) and every grid downloaded
    h2d = sum(stats[g]["h2d_bytes"] for g in range(len(grids)))
    d2h = sum(b.numel() * b.element_size() for b in host_bufs)
    all_idx = list(range(len(grids)))
    e2e_step_ms = []
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        ts = time.perf_counter()
        ctx.grid_build_set(ff, cell, atoms, 12.0, dims, native.PRECISION_FP32C, [g[1] for g in grids],
                           [g[2] for g in grids], [outs[g].data_ptr() for g in all_idx], out_host=host_np)
        e2e_step_ms.append(1e3 * (time.perf_counter() - ts))
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world, dist)
    e2e_value = whole_job_rate(len(grids) * npts * e2e_steps, world, e2e_s)

    # the reference's grid test after the build (rg_grid_validate): 100,000 points on the C_co2 grid and its charge term
    validation = run_grid_validation(args, ctx, ff, cell, atoms, dims, outs, rank, world, native)

    # roofline of the dominant kernel: algorithmic FLOPs = in-cutoff pairs x FLOPs per pair, per grid built
    mean_ms = [statistics.mean(k) for k in kern_ms]
    call_flops = [sum(stats[g]["pair_count"] * FLOPS_PER_PAIR["ewald" if grids[g][1] == 1 else "lj"] for g in idx)
                  for idx in calls]
    dom = int(np.argmax(mean_ms))
    achieved = call_flops[dom] / (mean_ms[dom] * 1e-3) / 1e12
    # DRAM traffic per launch from the ncu capture of the same kernels (dram__bytes_read.sum + dram__bytes_write.sum,
    # the grid-build summary in profiles/): the images are L2-resident, and part of the 100.75 MB a grid kernel writes is
    # still in the 126 MB L2 when the kernel ends, so the counters see less than the output
    traffic = NCU_DRAM_BYTES.get(call_names[dom])

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "grid build: C_co2-LJ + O_co2-LJ + unit-charge Ewald-real tricubic grids, "
                               "133x133x89 points each, FP32C", "grid_points_per_step": len(grids) * npts,
                   "framework_atoms": int(len(atoms)), "cutoff": 12.0, "precision": "FP32 pairs, compensated FP32 "
                   "accumulation, FP64 epilogue", "l2": "256 MiB flush between timed steps; 302 MB output per step",
                   "parallelism": f"replicas x{world}"},
        "kernels": {call_names[c]: {"ms": mean_ms[c], "grids": [grids[g][0] for g in calls[c]],
                                    "pairs_per_grid": stats[calls[c][0]]["pair_count"],
                                    "images": stats[calls[c][0]]["n_images"],
                                    "tflops": call_flops[c] / (mean_ms[c] * 1e-3) / 1e12}
                    for c in range(len(calls))},
        "roofline": {"kernel": f"gridKernelPacked ({call_names[dom]})", "bound": "fp32", "achieved": achieved,
                     "peak": peak_fp32, "unit": "TFLOP/s", "frac": achieved / peak_fp32, "traffic": traffic,
                     "peak_source": "rg_probe_fma_peak: FP32 FMA chains on all SMs, measured in this run",
                     "flops_per_pair": FLOPS_PER_PAIR,
                     "traffic_note": "bytes per launch from one ncu capture of the kernel (the grid-build summary in profiles/):"
                                     " DRAM read + write; the output (100.75 MB per grid) is partly still in L2 when the "
                                     "kernel ends, so the counters see less than it"},
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "step_ms": e2e_step_ms, "path": "rg_grid_build_set with pinned host outputs"},
        "gpu_launches": len(calls) * args.steps,
        "grid_validation": validation,
    }
    # ---- the methane grid in FP64 (FP64-pipe roofline) ----
    line["methane_grid_fp64"] = run_methane_grid_fp64(args, ctx, world, rank, dist, torch)
    # ---- GCMC steps/s on the same workload: CO2 in the 2x2x3 simulation box, the FP32C grids just built ----
    if not args.no_gcmc:
        line["gcmc"] = run_gcmc(args, ctx, ff, cell, atoms, dims, grids, outs, world, rank, dist, torch)
    # ---- batched CBMC of flexible chains in 64 uneven systems ----
    if not args.no_alkane:
        line["batched_cbmc"] = run_alkane(args, ctx, peak_fp32, world, rank, dist, torch)
    # ---- one large two-component system on the whole GPU ----
    if not args.no_mixture:
        line["mixture"] = run_mixture(args, ctx, world, rank, dist, torch)
    # ---- triquintic grid of the charged synthetic framework (27 channels, FP64) ----
    if not args.no_triquintic:
        line["triquintic"] = run_triquintic(args, ctx, ff, cell, atoms, dims, world, rank, dist, torch)
    # ---- paths (b) and (c) on their own through the C-ABI (large mixture, and the charged 2x2x3 box for the Ewald) ----
    if not args.no_paths:
        line["paths"] = run_paths(args, ctx, world, rank, dist, torch)
        line["paths"]["ewald_batch"] = run_ewald_batch(args, ctx, world, rank, dist, torch)
    # ---- learned vs uniform first-bead proposal at equal loading error ----
    if not args.no_learned:
        del flush
        line["learned_proposal"] = run_learned(args, ctx, world, rank, dist, torch)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, pts, secs, threads = cpu_oracle_rate(ff, cell, atoms, dims, grids, args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{pts // len(grids)} random grid points x {len(grids)} grids in {secs:.1f} s "
                                          f"(FP64 oracle of makeFrameworkInterpolationGrid, release flags, OpenMP over points)"}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
