#!/usr/bin/env python
"""Throughput of the fixed-charge nonbonded energy + force evaluation (TIP3P water boxes).

A step is one energy + force evaluation of one periodic water box: cluster-pair
neighbour build, fused real-space LJ + erfc-Coulomb with exclusion correction, PME
(spread, FFT, influence function, FFT, gather), forces back in caller order.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload water3000|water216|water100k] [--precision mixed|fp64]

Multi-GPU (torchrun, one rank per GPU): each rank evaluates its own replica box (seeded
per rank); no data-path collective exists for one system, so the run is weak scaling
over independent replicas. `--impl reference` times the CPU restatement of the
reference's pure-torch algorithm (O(N^2) neighbour list, pair terms, PME) on the host
cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(REPO, "torchff-lib_b200"), REPO):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "3000-water PME energy+force evals/s"
WORKLOAD_TEXT = {
    "water3000": "3000 rigid TIP3P waters (9000 atoms), cubic L=4.482 nm, rc=1.0 nm, Ewald alpha 2.628 nm^-1, "
                 "PME 48^3 order 6, LJ on O, intramolecular pairs excluded",
    "water216": "216 rigid TIP3P waters (648 atoms), cubic L=1.8662 nm, rc=0.9 nm, Ewald alpha 2.920 nm^-1, "
                "PME 20^3 order 6",
    "water100k": "100,000 rigid TIP3P waters (300,000 atoms), cubic L=14.42 nm, rc=1.0 nm, PME 144^3 order 6",
    "serving": "4096 requests, each a rigid TIP3P box of log-uniform [64, 4000] waters at 33.4 waters/nm^3, "
               "rc=0.9 nm, PME grid K=ceil(L/0.1 nm) order 6, mixed precision",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOAD_TEXT), default="water3000")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving section of the water3000 line")
    ap.add_argument("--no-large-box", action="store_true",
                    help="skip the 100,000-water section (large_box) of the water3000 line")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 timing of the water3000 line")
    ap.add_argument("--serving-requests", type=int, default=4096)
    ap.add_argument("--no-force-matching", action="store_true", help="skip the force-matching section")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference CUDA ops timing (reference_gpu) of the line")
    return ap.parse_args()


def water_box(name: str, seed: int):
    from torchff_b200 import water as W

    return {"water3000": W.water_box_3000, "water216": W.water_box_216, "water100k": W.water_box_100k}[name](seed)


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock/throttle samples every 50 ms; only samples whose own timestamp lies
    inside [begin(), end()] count, so the sampler's start-up time is not mistaken for load."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.t_begin = self.t_end = None

    def start(self, settle_s: float = 1.5):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(settle_s)
        except OSError:
            self.proc = None

    def begin(self):
        self.t_begin = datetime.datetime.now()

    def end(self):
        self.t_end = datetime.datetime.now()

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self, window=None) -> dict:
        """Median SM clock and the throttle reasons seen in [begin(), end()], or in
        window = (first, last) datetimes when given."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lo, hi = window if window is not None else (self.t_begin, self.t_end)
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                if lo is not None and not (lo <= ts <= hi):
                    continue
                sm.append(float(f[2]))
                smax = float(f[3])
            except ValueError:
                continue
            for name, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------------------

def count_pairs(wb, dtype, device, max_npairs: int | None = None):
    """In-cutoff half pairs (exclusions removed) of the frame: the algorithmic pair count (the
    cell list counts every pair it finds, also beyond a short max_npairs)."""
    import torch

    import torchff_b200  # noqa: F401
    from torchff_b200.nblist import convert_pairs_coo_to_csr

    rp, col = (t.to(device) for t in convert_pairs_coo_to_csr(torch.tensor(wb.nblist_exclusions), wb.natoms))
    x = torch.tensor(wb.coords, dtype=torch.float64, device=device)
    b = torch.tensor(wb.box, dtype=torch.float64, device=device)
    cap = int(wb.natoms * 4 / 3 * math.pi * wb.cutoff ** 3 * 100 / 2 * 1.5) if max_npairs is None else max_npairs
    _, n = torch.ops.torchff.build_neighbor_list_cell_list(x, b, wb.cutoff, cap, rp, col, False)
    return int(n.item())


def measured_peaks() -> dict:
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


PROFILED_SOURCES = ("pair_tile.cuh", "tile.cuh", "cluster.cuh", "tff_common.cuh", "fused.cu")


def kernel_source_hash() -> str:
    """sha256 (16 hex digits) of the real-space kernel sources, as the ncu summaries record
    it: a summary captured from other sources is stale for this build."""
    import hashlib

    h = hashlib.sha256()
    for name in PROFILED_SOURCES:
        with open(os.path.join(REPO, "torchff-lib_b200", "csrc", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def ncu_traffic(kernel: str, workload: str, name: str = "ncu_traffic.txt"):
    """A per-launch figure (DRAM bytes by default) from a committed ncu summary, with the
    date and source hash it records; the value is None when the summary is absent or was
    captured from other kernel sources than this build's."""
    path = os.path.join(REPO, "profiles", name)
    meta = {"file": f"profiles/{name}", "value": None}
    try:
        with open(path) as f:
            for ln in f:
                p = ln.split()
                if ln.startswith("# source-hash"):
                    meta["source_hash"] = p[2]
                elif ln.startswith("# captured"):
                    meta["captured"] = p[2]
                elif len(p) >= 3 and p[0] == kernel and p[1] == workload:
                    meta["value"] = float(p[2])
    except OSError:
        return meta
    current = kernel_source_hash()
    if meta.get("source_hash") != current:
        meta["stale"] = f"captured from sources {meta.get('source_hash')}, this build is {current}"
        meta["value"] = None
    return meta


def throughput_fields(npairs: int, evals_per_s: float, tile_ms: float, tile_dram_bytes) -> dict:
    """Pair throughput of the whole evaluation and the DRAM bandwidth the tile kernel draws.

    npairs: in-cutoff pairs of the box (each pair once); evals_per_s: the line's value;
    tile_ms: mean tile-kernel time per launch; tile_dram_bytes: dram__bytes_read.sum +
    dram__bytes_write.sum of one tile-kernel launch from the committed ncu summary (None if
    absent)."""
    out = {"pairs_per_s": round(npairs * evals_per_s), "unit": "in-cutoff pairs per second, each pair once"}
    if tile_dram_bytes is not None and tile_ms > 0:
        out["tile_kernel_dram_gbs"] = round(tile_dram_bytes / (tile_ms * 1e-3) / 1e9, 2)
        out["dram_note"] = ("DRAM bytes of one tile-kernel launch (ncu) / its mean CUDA-event time: positions "
                            "are re-read from L2, so the kernel draws little HBM bandwidth")
    return out


def cpu_baseline_sample(wb, evals: int = 2) -> tuple[dict, dict]:
    """The numpy oracle timed on one host core over `evals` evaluations of the box; also
    returns the oracle's FP64 result, which the accuracy figures of the line use."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    for _ in range(evals):
        ref = O.fixed_charge_energy(wb.coords, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                    wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                    138.935456)
    dt = time.perf_counter() - t0
    return ({"value": evals / dt, "unit": "evals/s", "cores": 1, "kind": "port",
             "sample": f"{evals} full evaluations of the same box by the numpy oracle (O(N^2) neighbour list, "
                       f"pair terms, PME with analytic forces), one thread"}, ref)


def accuracy_vs_oracle(energy: float, forces, ref: dict) -> dict:
    """Energy and force error of one result against the FP64 oracle on the same box."""
    import numpy as np

    f0 = -ref["grad_coords"]
    f = np.asarray(forces, dtype=np.float64)
    return {"energy_kj_mol": energy, "oracle_energy_kj_mol": float(ref["total"]),
            "energy_abs_err": float(f"{abs(energy - ref['total']):.3g}"),
            "energy_rel_err": float(f"{abs(energy - ref['total']) / abs(ref['total']):.3g}"),
            "force_rms_rel_err": float(f"{np.sqrt(np.mean((f - f0) ** 2)) / np.sqrt(np.mean(f0 ** 2)):.3g}"),
            "force_max_abs_err": float(f"{np.max(np.abs(f - f0)):.3g}"),
            "reference": "numpy FP64 oracle (restatement of the reference pure-torch path) on the same box"}


def time_graph_evals(wb, dtype, device, steps: int, warmup: int) -> dict:
    """evals/s of one system by CUDA-graph replays with an L2 flush in between."""
    import torch

    from torchff_b200.system import FixedChargeSystem

    system = FixedChargeSystem.from_water_box(wb, dtype=dtype, device=device)
    x = torch.tensor(wb.coords, dtype=dtype, device=device)
    b = torch.tensor(wb.box, dtype=dtype, device=device)
    energy = torch.empty(1, dtype=torch.float64, device=device)
    forces = torch.empty_like(x)
    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        for _ in range(2):
            system.evaluate_into(x, b, energy, forces)
    torch.cuda.current_stream(device).wait_stream(side)
    torch.cuda.synchronize(device)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        system.evaluate_into(x, b, energy, forces)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(warmup):
        flush.fill_(i & 0xff)
        graph.replay()
    total = 0.0
    for i in range(steps):
        flush.fill_(i & 0xff)
        start.record()
        graph.replay()
        end.record()
        end.synchronize()
        total += start.elapsed_time(end)
    del graph
    return {"value": round(steps / (total / 1e3), 2), "unit": "evals/s", "ms_per_step": round(total / steps, 5),
            "steps": steps, "warmup": warmup,
            "_result": (float(energy.item()), forces.double().cpu().numpy())}


def time_large_box(device, steps: int = 100, warmup: int = 5) -> dict:
    """The 100,000-water box (300,000 atoms, mixed precision) in the default line: evals/s by
    CUDA-graph replays with an L2 flush in between, the stage times, and the pair kernel's
    roofline at this size (its achieved FP32 rate over the mean pair-stage time)."""
    import torch

    from torchff_b200.system import FixedChargeSystem, StageTimer

    wb = water_box("water100k", 0)
    dtype = torch.float32
    system = FixedChargeSystem.from_water_box(wb, dtype=dtype, device=device)
    x = torch.tensor(wb.coords, dtype=dtype, device=device)
    b = torch.tensor(wb.box, dtype=dtype, device=device)
    energy = torch.empty(1, dtype=torch.float64, device=device)
    forces = torch.empty_like(x)
    timer = StageTimer()
    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        for _ in range(2):
            system.evaluate_timed_into(x, b, energy, forces, timer)
            system.evaluate_into(x, b, energy, forces)
    torch.cuda.current_stream(device).wait_stream(side)
    torch.cuda.synchronize(device)
    if system.status() != 0:
        raise RuntimeError("cluster neighbour list overflow")
    graph, tgraph = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        system.evaluate_into(x, b, energy, forces)
    with torch.cuda.graph(tgraph):
        system.evaluate_timed_into(x, b, energy, forces, timer)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(warmup):
        flush.fill_(i & 0xff)
        graph.replay()
    total = 0.0
    for i in range(steps):
        flush.fill_(i & 0xff)
        start.record()
        graph.replay()
        end.record()
        end.synchronize()
        total += start.elapsed_time(end)
    n_stage = min(steps, 50)
    acc = {k: 0.0 for k in StageTimer.STAGES}
    for i in range(n_stage):
        flush.fill_(i & 0xff)
        tgraph.replay()
        torch.cuda.synchronize(device)
        for k, v in timer.stages_ms().items():
            acc[k] += v
    del graph, tgraph
    stages = {k: round(v / n_stage * 1e3, 2) for k, v in acc.items()}
    npairs = count_pairs(wb, dtype, device, max_npairs=1)
    sm_max = float(measured_peaks().get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = 60.0 * npairs / (stages["tile_kernel"] * 1e-6) / 1e12
    traffic = ncu_traffic("pair_tile_kernel", "water100k")
    issue = ncu_traffic("pair_tile_kernel", "water100k", "ncu_issue.txt")
    return {"workload": f"water100k: {WORKLOAD_TEXT['water100k']}", "precision": "mixed",
            "value": round(steps / (total / 1e3), 2), "unit": "evals/s", "ms_per_step": round(total / steps, 4),
            "steps": steps, "warmup": warmup, "l2": "flushed between timed steps (256 MiB device write)",
            "stage_us_mean": stages,
            "roofline": {"kernel": "pair_tile_kernel<float>", "bound": "fp32", "achieved": round(achieved, 4),
                         "peak": round(fp32_peak, 2), "unit": "TFLOP/s", "frac": round(achieved / fp32_peak, 5),
                         "traffic": traffic["value"], "traffic_source": traffic, "issue_active": issue["value"],
                         "algorithmic": f"60 flop x {npairs} in-cutoff pairs per launch / mean pair-stage time "
                                        f"{stages['tile_kernel']:.1f} us (CUDA events in the graph)"},
            "throughput": {"pairs_per_s": round(npairs * steps / (total / 1e3)),
                           "unit": "in-cutoff pairs per second, each pair once"}}


def run_force_matching(device, dtype, rank: int, world: int, frames: int = 16, steps: int = 10,
                       warmup: int = 3) -> dict:
    """One force-matching training step = for each of `frames` perturbed frames of the
    3000-water box: energy, forces (create_graph) and the loss mean |F - F_target|^2; then
    backward to the per-atom charges, sigma and epsilon (double backward). Frames are split
    over the ranks; the parameter gradients are summed over ranks with one all-reduce."""
    import numpy as np
    import torch

    from torchff_b200.distributed import allreduce_sum_, frame_shard, max_over_ranks
    from torchff_b200.system import FixedChargeNonbonded, FixedChargeSystem
    from torchff_b200.water import force_matching_parameters, perturbed_frames, water_box_3000

    wb = water_box_3000()
    q0, s0, e0 = force_matching_parameters(wb, seed=0)
    xs = perturbed_frames(wb, frames, 0.005, seed=1)
    targets = np.random.default_rng(2).normal(0.0, 300.0, size=xs.shape)
    mine = frame_shard(frames, rank, world)
    sysm = FixedChargeSystem(q0, s0, e0, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid, dtype=dtype,
                             device=device)
    model = FixedChargeNonbonded(sysm)
    box = torch.tensor(wb.box, dtype=dtype, device=device)
    X = [torch.tensor(xs[f], dtype=dtype, device=device, requires_grad=True) for f in mine]
    T = [torch.tensor(targets[f], dtype=dtype, device=device) for f in mine]
    params = [torch.tensor(a, dtype=dtype, device=device, requires_grad=True) for a in (q0, s0, e0)]

    def step():
        for p in params:
            p.grad = None
        total = torch.zeros((), dtype=torch.float64, device=device)
        for x, t in zip(X, T):
            E = model(x, box, *params)
            (gx,) = torch.autograd.grad(E, x, create_graph=True)
            loss = torch.mean((-gx - t) ** 2) / frames
            loss.backward()
            total += loss.detach().double()
        allreduce_sum_([p.grad for p in params] + [total])
        return total

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(device)
    if world > 1:
        dist.barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        step()
    end.record()
    end.synchronize()
    ms = max_over_ranks(start.elapsed_time(end) / steps, device)
    return {"workload": "3000-water box, per-atom q (+-5% noise, neutral), sigma, eps leaves; "
                        f"{frames} frames with N(0, 0.005 nm) coordinate noise; loss mean |F - F_target|^2",
            "precision": "mixed" if dtype == torch.float32 else "fp64", "frames": frames, "ranks": world,
            "ms_per_step": round(ms, 3), "frames_per_s": round(frames / (ms / 1e3), 1),
            "per_frame": "forward with parameter gradients + one Hessian-vector product (double backward)",
            "gradient_allreduce": "NCCL sum of dE/d(q, sigma, eps) over ranks" if world > 1 else None}


def sequential_dropin_ops(boxes, device) -> float:
    """Seconds per system of the serving denominator: the reference's composition
    (examples/tip3p/model.py:100-133) through this library's drop-in modules, one request
    after another, in mixed precision (FP32 tensors); modules and parameters are prepared
    before the clock starts, and each request copies its host coordinates in and its forces
    and energy out."""
    import numpy as np
    import torch

    from torchff_b200 import PME, MultipolarInteraction, NeighborList, Vdw

    prepared = []
    for wb in boxes:
        n = wb.natoms
        dt = torch.float32
        nbl = NeighborList(n, exclusions=torch.tensor(wb.nblist_exclusions), algorithm="cell_list").to(device)
        cap = int(n * 4 / 3 * 3.1416 * wb.cutoff ** 3 * 100 / 2 * 1.2)
        prepared.append(dict(
            wb=wb, nbl=nbl, cap=cap,
            lj=Vdw("LennardJones", use_customized_ops=True, use_type_pairs=True).to(device),
            coul=MultipolarInteraction(0, wb.cutoff, wb.alpha, 138.935456).to(device),
            pme=PME(wb.alpha, wb.grid, 0, use_customized_ops=True).to(device),
            box=torch.tensor(wb.box, dtype=dt, device=device), q=torch.tensor(wb.charges, dtype=dt, device=device),
            sig=torch.tensor(wb.sigma_table, dtype=dt, device=device),
            eps=torch.tensor(wb.epsilon_table, dtype=dt, device=device),
            types=torch.tensor(wb.atom_types, dtype=torch.int64, device=device),
            excl=torch.tensor(wb.coulomb_exclusions, dtype=torch.int64, device=device),
            host=torch.tensor(np.ascontiguousarray(wb.coords), dtype=dt).pin_memory(),
            out=torch.empty((n, 3), dtype=dt).pin_memory()))

    def one(p):
        wb = p["wb"]
        x = p["host"].to(device, non_blocking=True).requires_grad_(True)
        pairs, _ = p["nbl"](x.detach(), p["box"], wb.cutoff, p["cap"], padding=True)
        e = (p["lj"](x, pairs, p["box"], p["sig"], p["eps"], wb.cutoff, atom_types=p["types"])
             + p["coul"](x, p["box"], pairs, p["q"], pairs_excl=p["excl"])
             + p["pme"](x, p["box"], p["q"]) * 138.935456)
        e.backward()
        p["out"].copy_(-x.grad, non_blocking=True)
        return float(e.item())

    for p in prepared:  # warm-up: cuFFT plans of every grid size, workspaces, allocator
        one(p)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for p in prepared:
        one(p)
    torch.cuda.synchronize(device)
    return (time.perf_counter() - t0) / len(prepared)


def run_serving(device, n_requests: int = 4096, seed: int = 0) -> dict:
    """Continuous-batching server on the serving workload: throughput at saturation, p50/p99
    latency under Poisson arrivals, and sequential single-system calls on the same requests."""
    import numpy as np
    import torch

    from torchff_b200.serving import Server, SystemSpec, autotune_atoms_per_cell
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import serving_water_box

    rng = np.random.default_rng(seed)
    n_waters = np.exp(rng.uniform(math.log(64), math.log(4000), n_requests)).astype(int)
    boxes = [serving_water_box(int(n), seed=seed * 100_003 + k) for k, n in enumerate(n_waters)]
    specs = [SystemSpec.from_water_box(w) for w in boxes]
    alpha, rc = boxes[0].alpha, 0.9
    atoms = np.array([s.natoms for s in specs])
    apc, tune_ms = autotune_atoms_per_cell(specs[:64], rc, alpha)
    # 4 lanes: 3 / 4 / 6 / 8 lanes of 256 systems served 71.4k / 73.6k / 74.3k / 73.3k systems/s
    lanes, per_batch, budget = 4, 256, 6 << 30
    srv = Server(rc, alpha, torch.float32, lanes=lanes, max_systems_per_batch=per_batch, hbm_budget_bytes=budget,
                 atoms_per_cell=apc, device=device)

    prepared = [srv.prepare(sp) for sp in specs]

    def run(rate):
        """rate None: every request queued while the server holds, then released at once
        (throughput from release to the last completion; latency from release). Otherwise
        Poisson arrivals at `rate` per second (latency from submission)."""
        reqs = []
        if rate is None:
            srv.hold(True)
            reqs = [srv.submit(pr) for pr in prepared]
            s0 = srv.now()
            srv.hold(False)
        else:
            arrivals = np.cumsum(np.random.default_rng(seed + 7).exponential(1.0 / rate, n_requests))
            s0 = srv.now()
            t0 = time.perf_counter()
            for k, pr in enumerate(prepared):
                while time.perf_counter() - t0 < arrivals[k]:
                    pass
                reqs.append(srv.submit(pr))
        srv.drain()
        times = np.array([r.times() for r in reqs])
        for r in reqs:
            r.release()
        lat = (times[:, 2] - np.maximum(times[:, 0], s0)) * 1e3
        span = times[:, 2].max() - s0
        return reqs, {"systems_per_s": round(n_requests / span, 1), "p50_ms": round(float(np.median(lat)), 3),
                      "p99_ms": round(float(np.percentile(lat, 99)), 3), "makespan_s": round(float(span), 4)}

    run(None)  # warm-up: cuFFT plans for every grid size and batch count that shows up
    b0 = srv.stats()["batches"]
    reqs, sat = run(None)
    st = srv.stats()
    sat.update({"batches": st["batches"] - b0, "max_batch_systems": st["max_batch_systems"],
                "max_lanes_in_flight": st["max_lanes_in_flight"]})
    poisson = []
    for frac in (0.25, 0.5, 0.8):
        rate = frac * sat["systems_per_s"]
        _, r = run(rate)
        r["offered_rate_per_s"] = round(rate, 1)
        poisson.append(r)
    # accuracy of served results against FP64 single-system evaluations
    errs = []
    for k in range(0, n_requests, max(1, n_requests // 16)):
        wb = boxes[k]
        ref = FixedChargeSystem.from_water_box(wb, dtype=torch.float64, device=device).evaluate(
            torch.tensor(wb.coords, dtype=torch.float64, device=device),
            torch.tensor(wb.box, dtype=torch.float64, device=device))["forces"].cpu().numpy()
        f = reqs[k].forces
        errs.append(float(np.sqrt(np.mean((f - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))))
    stats = srv.stats()
    srv.close()
    # sequential single-system calls: prebuilt systems (evaluation only), and plain calls
    # that set each system up per request (what a per-system API user does)
    nseq = min(128, n_requests)
    prebuilt = [FixedChargeSystem.from_water_box(boxes[k], dtype=torch.float32, device=device) for k in range(nseq)]
    host = [(np.ascontiguousarray(boxes[k].coords), np.ascontiguousarray(boxes[k].box),
             np.zeros_like(boxes[k].coords)) for k in range(nseq)]
    for sy, (x, b, f) in zip(prebuilt, host):
        sy.evaluate_host(x, b, f)
    t0 = time.perf_counter()
    for sy, (x, b, f) in zip(prebuilt, host):
        sy.evaluate_host(x, b, f)
    t_pre = (time.perf_counter() - t0) / nseq
    del prebuilt
    t_ops = sequential_dropin_ops(boxes[:nseq], device)
    nplain = min(64, n_requests)
    t0 = time.perf_counter()
    for k in range(nseq, nseq + nplain):
        wb = boxes[k % n_requests]
        sy = FixedChargeSystem.from_water_box(wb, dtype=torch.float32, device=device)
        sy.evaluate_host(np.ascontiguousarray(wb.coords), np.ascontiguousarray(wb.box), np.zeros_like(wb.coords))
        del sy
    t_plain = (time.perf_counter() - t0) / nplain
    # the sequential samples hold the same size distribution; scale by mean atoms
    return {
        "workload": WORKLOAD_TEXT["serving"],
        "requests": n_requests, "atoms_total": int(atoms.sum()), "atoms_mean": round(float(atoms.mean()), 1),
        "server": {"lanes": lanes, "max_systems_per_batch": per_batch, "hbm_budget_bytes": budget,
                   "lane_max_atoms": stats["lane_max_atoms"], "lane_device_bytes": stats["lane_device_bytes"],
                   "atoms_per_cell": apc, "autotune_ms": {str(k): round(v, 3) for k, v in tune_ms.items()}},
        "saturation": sat,
        "poisson": poisson,
        "sequential_prebuilt": {"us_per_system": round(t_pre * 1e6, 1), "systems_per_s": round(1.0 / t_pre, 1),
                                "sample": f"first {nseq} requests, FixedChargeSystem.evaluate_host on systems "
                                          "created beforehand (one CUDA-graph replay + copies per call)"},
        "sequential_plain_calls": {"us_per_system": round(t_plain * 1e6, 1),
                                   "systems_per_s": round(1.0 / t_plain, 1),
                                   "sample": f"{nplain} requests, FixedChargeSystem created, evaluated "
                                             "(evaluate_host) and freed per request"},
        "sequential_dropin_ops": {"us_per_system": round(t_ops * 1e6, 1), "systems_per_s": round(1.0 / t_ops, 1),
                                  "sample": f"first {nseq} requests through this library's drop-in ops "
                                            "(NeighborList cell list + Vdw + MultipolarInteraction + 138.935456 x PME, "
                                            "torch.ops.torchff, FP32), modules built beforehand; per request: "
                                            "host coords in, energy + backward, host forces and energy out"},
        "speedup_vs_dropin_ops": round(sat["systems_per_s"] * t_ops, 2),
        "speedup_vs_prebuilt": round(sat["systems_per_s"] * t_pre, 2),
        "speedup_vs_plain_calls": round(sat["systems_per_s"] * t_plain, 2),
        "accuracy": {"max_force_rms_rel_vs_fp64": float(f"{max(errs):.3g}"), "requests_checked": len(errs)},
        "precision": "mixed",
    }


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}; launch N>1 with torch.distributed.run")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    import torchff_b200  # noqa: F401
    from torchff_b200.system import FixedChargeSystem, StageTimer

    # one sampler for the whole run: the timed steps are the window [begin(), end()]
    clocks = ClockSampler(local)
    clocks.start()
    run_t0 = datetime.datetime.now()
    if args.workload == "serving":
        clocks.stop()
        run_serving_line(args, device, rank, world)
        return
    dtype = torch.float32 if args.precision == "mixed" else torch.float64
    wb = water_box(args.workload, seed=rank)
    system = FixedChargeSystem.from_water_box(wb, dtype=dtype, device=device)
    x = torch.tensor(wb.coords, dtype=dtype, device=device)
    b = torch.tensor(wb.box, dtype=dtype, device=device)
    energy = torch.empty(1, dtype=torch.float64, device=device)
    forces = torch.empty_like(x)
    timer = StageTimer()

    # capture one evaluation in a CUDA graph (timed steps), and one with stage events between
    # its kernels (stage breakdown; the events split the chain of dependent launches)
    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        for _ in range(2):
            system.evaluate_timed_into(x, b, energy, forces, timer)
            system.evaluate_into(x, b, energy, forces)
    torch.cuda.current_stream(device).wait_stream(side)
    torch.cuda.synchronize(device)
    if system.status() != 0:
        raise RuntimeError("cluster neighbour list overflow")
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        system.evaluate_into(x, b, energy, forces)
    tgraph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(tgraph):
        system.evaluate_timed_into(x, b, energy, forces, timer)

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)   # > 126 MB L2
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(args.warmup):
        flush.fill_(i & 0xff)
        graph.replay()
    torch.cuda.synchronize(device)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(device)
    clocks.begin()
    step_ms = []
    for i in range(args.steps):
        flush.fill_(i & 0xff)
        start.record()
        graph.replay()
        end.record()
        end.synchronize()
        step_ms.append(start.elapsed_time(end))
    torch.cuda.synchronize(device)
    clocks.end()
    if world > 1:
        dist.barrier()
    # stage breakdown (and the tile-kernel time of the roofline) from the graph with events
    n_stage = min(args.steps, 200)
    tile_ms, stage_acc = [], {k: 0.0 for k in StageTimer.STAGES}
    for i in range(n_stage):
        flush.fill_(i & 0xff)
        tgraph.replay()
        torch.cuda.synchronize(device)
        st = timer.stages_ms()
        tile_ms.append(st["tile_kernel"])
        for k, v in st.items():
            stage_acc[k] += v
    total_ms = sum(step_ms)
    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * args.steps / (max_ms / 1e3)

    # end to end through the C ABI with host buffers (H2D coords+box, eval, D2H forces+energy)
    hx = torch.tensor(wb.coords, dtype=torch.float64).pin_memory()
    hb = torch.tensor(wb.box, dtype=torch.float64).pin_memory()
    hf = torch.empty((wb.natoms, 3), dtype=torch.float64).pin_memory()
    for i in range(5):
        system.evaluate_host(hx, hb, hf)
    e2e_ms = []
    if world > 1:
        dist.barrier()
    for i in range(args.e2e_steps):
        flush.fill_(i & 0xff)
        start.record()
        system.evaluate_host(hx, hb, hf)
        end.record()
        end.synchronize()
        e2e_ms.append(start.elapsed_time(end))
    te = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * args.e2e_steps / (float(te.item()) / 1e3)
    fm = None
    if not args.no_force_matching and args.workload == "water3000":
        fm = [run_force_matching(device, torch.float64, rank, world), run_force_matching(device, torch.float32, rank, world)]
    h2d = wb.natoms * 3 * 8 + 9 * 8
    d2h = wb.natoms * 3 * 8 + 8

    result = None
    if rank == 0:
        npairs = count_pairs(wb, dtype, device)
        peaks = measured_peaks()
        sm_max = float(peaks.get("sm_max_mhz", 1965.0))
        fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12        # TFLOP/s, FMA = 2 flops
        tile_mean_ms = statistics.mean(tile_ms)
        flops = 60.0 * npairs                                   # algorithmic flops per launch
        achieved = flops / (tile_mean_ms * 1e-3) / 1e12
        stages = {k: round(v / n_stage * 1e3, 3) for k, v in stage_acc.items()}
        traffic = ncu_traffic("pair_tile_kernel", args.workload)
        issue = ncu_traffic("pair_tile_kernel", args.workload, "ncu_issue.txt")
        result = {
            "metric": METRIC if args.workload == "water3000" else f"{args.workload} PME energy+force evals/s",
            "value": round(value, 2),
            "unit": "evals/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 5),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if dtype == torch.float32 else "f64",
            "data": "synthetic (seeded TIP3P lattice box, one replica per rank)",
            "config": {
                "workload": f"{args.workload}: {WORKLOAD_TEXT[args.workload]}",
                "precision": "mixed: FP32 pair/spline arithmetic, int64 fixed-point forces, FP64 energies"
                if dtype == torch.float32 else "fp64",
                "path": "FixedChargeSystem (cluster-pair build + fused real-space tile kernel + PME), "
                        "one CUDA-graph replay per step",
                "l2": "flushed between timed steps (256 MiB device write)",
                "parallelism": f"replicas x{world}",
                "stage_us_mean": stages,
            },
            "e2e": {"value": round(e2e_value, 2), "unit": "evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "tff_system_eval_host (C ABI): pinned host coords/box -> device -> host forces"},
            "gpu_launches": system.kernel_launches() * args.steps,
            "roofline": {
                "kernel": "pair_tile_kernel<float> (fused real-space LJ + erfc Coulomb over half cluster lists, 8x8 sub-tiles, each pair once)",
                "bound": "fp32",
                "achieved": round(achieved, 4),
                "peak": round(fp32_peak, 2),
                "unit": "TFLOP/s",
                "frac": round(achieved / fp32_peak, 5),
                "traffic": traffic["value"],
                "traffic_source": traffic,
                "algorithmic": f"60 flop x {npairs} in-cutoff pairs per launch / mean tile-kernel time "
                               f"{tile_mean_ms * 1e3:.2f} us (CUDA events in the graph)",
                "peak_source": f"FP32 nominal 148 SM x 128 lanes x 2 flop x {sm_max:.0f} MHz (sm_max_mhz of "
                               "MEASURED_PEAKS.json; no measured FP32 peak exists)",
                "issue_active": issue["value"],
                "issue_source": issue,
                "issue_note": "fraction of issue slots the pair kernel uses, from ncu (profiles/ncu_issue.txt): "
                              "sub-tile screening, staging and the shuffle reductions share the issue slots "
                              "with the pair math",
            },
        }
        result["throughput"] = throughput_fields(npairs, value, tile_mean_ms, traffic["value"])
        if fm is not None:
            result["force_matching"] = fm
        fp64_result = None
        if world == 1 and not args.no_fp64 and dtype == torch.float32:
            result["fp64"] = time_graph_evals(wb, torch.float64, device, min(args.steps, 500), args.warmup)
            fp64_result = result["fp64"].pop("_result")
        if world == 1 and not args.no_large_box and args.workload == "water3000":
            result["large_box"] = time_large_box(device)
        if world == 1 and not args.no_serving:
            result["serving"] = run_serving(device, args.serving_requests)
        oracle_ref = None
        if world == 1 and not args.no_cpu_baseline:
            if args.workload == "water100k":
                result["cpu_baseline"] = {"value": None, "unit": "evals/s", "cores": 0, "kind": "port",
                                          "sample": "not run: the reference CPU path's O(N^2) pair search over "
                                                    "300,000 atoms (4.5e10 pairs) is infeasible"}
            else:
                result["cpu_baseline"], oracle_ref = cpu_baseline_sample(wb)
        if oracle_ref is not None:
            # the result the timed graph produced (last replay) and the FP64 one, against the oracle
            result["accuracy"] = {("mixed" if dtype == torch.float32 else "fp64"):
                                  accuracy_vs_oracle(float(energy.item()), forces.double().cpu().numpy(), oracle_ref)}
            if fp64_result is not None:
                result["accuracy"]["fp64"] = accuracy_vs_oracle(fp64_result[0], fp64_result[1], oracle_ref)
        if world == 1 and not args.no_reference_gpu and args.workload in ("water3000", "water216"):
            rg = reference_gpu_leg(args)
            result["reference_gpu"] = rg
            if "value" in rg and rg.get("value"):
                result["speedup_vs_reference_fp64_cuda"] = {
                    "device": round(value / rg["value"], 2), "e2e": round(e2e_value / rg["value"], 2),
                    "formula": "this line's value (and e2e value) / reference_gpu.value (the reference's FP64 CUDA "
                               f"ops on the same box and GPU, {rg['fp64']['mode']}, L2 flushed)"}
            if "large_box" in result:
                # the same composition of the reference's ops on the 300,000-atom box
                lb = result["large_box"]
                rg = reference_gpu_leg(args, "water100k", 20)
                lb["reference_gpu"] = rg
                if "value" in rg and rg.get("value"):
                    lb["speedup_vs_reference_fp64_cuda"] = {
                        "device": round(lb["value"] / rg["value"], 2),
                        "formula": "large_box.value / large_box.reference_gpu.value (the reference's FP64 CUDA ops "
                                   f"on the same 300,000-atom box and GPU, {rg['fp64']['mode']}, L2 flushed)"}
        clocks.stop()
        result["clocks"] = clocks.summary()
        result["clocks_whole_run"] = dict(clocks.summary((run_t0, datetime.datetime.now())), note=(
            "nvidia-smi samples over the whole run of this line (timed steps, stage timing, e2e, force matching, "
            "FP64, large box, serving, reference GPU): the timed steps alone can be shorter than one 50 ms sample"))
    else:
        clocks.stop()
    del graph
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)


def run_serving_line(args, device, rank, world):
    """--workload serving: one server per rank on its own requests (no collective on the data
    path); value = the ranks' saturation throughputs summed."""
    import torch
    import torch.distributed as dist

    res = run_serving(device, args.serving_requests, seed=rank)
    v = torch.tensor([res["saturation"]["systems_per_s"], res["saturation"]["p99_ms"]], dtype=torch.float64,
                     device=device)
    if world > 1:
        tot = v.clone()
        dist.all_reduce(tot[:1], op=dist.ReduceOp.SUM)
        dist.all_reduce(tot[1:], op=dist.ReduceOp.MAX)
        v = tot
    if rank == 0:
        bytes_in = res["atoms_mean"] * (3 * 8 + 3 * 8 + 2 * 8) + 72
        line = {
            "metric": "serving systems/s (continuous batching, saturation)",
            "value": round(float(v[0]), 1), "unit": "systems/s", "n_gpus": world, "steps": args.serving_requests,
            "warmup": args.serving_requests, "ms_per_step": round(1e3 / float(v[0]), 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded TIP3P boxes)",
            "config": {"workload": f"serving: {WORKLOAD_TEXT['serving']}", "parallelism": f"server per rank x{world}",
                       "l2": "inputs of a batch (tens of MB) exceed nothing; each request is new data"},
            "e2e": {"value": round(float(v[0]), 1), "unit": "systems/s",
                    "h2d_bytes_per_step": int(bytes_in), "d2h_bytes_per_step": int(res["atoms_mean"] * 24 + 8),
                    "path": "tff_server_submit of host arrays -> batched evaluation -> host energy/forces"},
            "p99_ms_max_over_ranks": round(float(v[1]), 3),
            "serving": res,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------
# reference arm: the reference's own pure-torch path on the host cores
# ---------------------------------------------------------------------------------------

REF_EXTENSIONS = ("torchff_bond", "torchff_angle", "torchff_nblist", "torchff_nb", "torchff_coulomb", "torchff_vdw",
                  "torchff_multipoles", "torchff_pme", "torchff_torsion", "torchff_dispersion", "torchff_slater",
                  "torchff_ewald", "torchff_amoeba", "torchff_cmm")


def import_reference_cpu():
    """The reference package (THGLab/torchff-lib, installed without its CUDA extensions into
    baseline/_ref) imported for its pure-torch path. Its modules import their compiled
    extension modules by name; the pure-torch path never calls them, so empty modules stand
    in. torchff/pme_ref.py:8 switches the default device to CUDA at import time; it is set
    back to the CPU afterwards, and the default dtype to FP64. Returns None when the install
    is absent."""
    import types

    root = os.path.join(REPO, "baseline", "_ref")
    if not os.path.isdir(os.path.join(root, "torchff")):
        return None
    import torch

    for name in REF_EXTENSIONS:
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, root)
    import torchff  # noqa: F401
    from torchff.multipoles import MultipolarInteraction
    from torchff.nblist import NeighborList
    from torchff.pme import PME
    from torchff.vdw import Vdw

    torch.set_default_device("cpu")
    # FP64 throughout: the pure-torch PME builds its B-spline moduli from default-dtype
    # tensors (torchff/pme_ref.py:268-274), which FP32 would round to ~1e-6 of the
    # reciprocal energy
    torch.set_default_dtype(torch.float64)
    return types.SimpleNamespace(NeighborList=NeighborList, MultipolarInteraction=MultipolarInteraction, PME=PME,
                                 Vdw=Vdw, root=root)


def water_box_unregistered(name: str, seed: int):
    """torchff_b200/water.py loaded by path (the box generator only: importing the package
    would load libtffb200 and register its own torch.ops.torchff schemas)."""
    import importlib.util

    mod = sys.modules.get("_tff_water")
    if mod is None:
        spec = importlib.util.spec_from_file_location(
            "_tff_water", os.path.join(REPO, "torchff-lib_b200", "torchff_b200", "water.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["_tff_water"] = mod
        spec.loader.exec_module(mod)
    return {"water3000": mod.water_box_3000, "water216": mod.water_box_216, "water100k": mod.water_box_100k}[name](seed)


def run_reference_cpu(args, ref) -> dict:
    """The nonbonded part of the reference's TIP3P model (examples/tip3p/model.py:100-133)
    through the reference's own modules with use_customized_ops=False, FP64, on the host
    cores: NeighborList._forward_python (torchff/nblist.py:137-140) with the water
    exclusions, Vdw('LennardJones') with type tables (torchff/vdw.py), rank-0
    MultipolarInteraction with pairs_excl (torchff/multipoles.py:244-341) and
    138.935456 x PME(alpha, K, 0) (torchff/pme_ref.py:422-469); energy + backward() for the
    forces. One step = one full evaluation of the box rank 0 of the other arm evaluates
    (seed 0). The one-off NeighborList construction (its all-pairs buffer) is timed apart."""
    import torch

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    wb = water_box_unregistered(args.workload, 0)
    t0 = time.perf_counter()
    nbl = ref.NeighborList(wb.natoms, exclusions=torch.tensor(wb.nblist_exclusions), use_customized_ops=False)
    lj = ref.Vdw("LennardJones", cutoff=wb.cutoff, use_customized_ops=False, use_type_pairs=True)
    coul = ref.MultipolarInteraction(rank=0, cutoff=wb.cutoff, ewald_alpha=wb.alpha, prefactor=138.935456,
                                     use_customized_ops=False)
    pme = ref.PME(wb.alpha, wb.grid, 0, use_customized_ops=False)
    t_init = time.perf_counter() - t0
    box = torch.tensor(wb.box, dtype=torch.float64)
    q = torch.tensor(wb.charges, dtype=torch.float64)
    sig_t = torch.tensor(wb.sigma_table, dtype=torch.float64)
    eps_t = torch.tensor(wb.epsilon_table, dtype=torch.float64)
    types_ = torch.tensor(wb.atom_types)
    excl = torch.tensor(wb.coulomb_exclusions)

    def evaluate():
        x = torch.tensor(wb.coords, dtype=torch.float64, requires_grad=True)
        pairs = nbl(x.detach(), box, wb.cutoff)
        e = (lj(x, pairs, box, sig_t, eps_t, wb.cutoff, atom_types=types_)
             + coul(x, box, pairs, q, pairs_excl=excl)
             + pme(x, box, q) * 138.935456)
        e.backward()
        return float(e.item()), x.grad

    t0 = time.perf_counter()
    evaluate()
    t_first = time.perf_counter() - t0
    # bounded: the whole arm stays within a few minutes on a host with few cores
    budget_s = 240.0
    warm = max(0, min(args.warmup, int(60.0 / max(t_first, 1e-3))) - 1)
    for _ in range(warm):
        evaluate()
    steps = max(1, min(args.steps, int(budget_s / max(t_first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        energy, _ = evaluate()
    wall = time.perf_counter() - t0
    return {"value": steps / wall, "ms_per_step": wall / steps * 1e3, "steps": steps, "warmup": warm + 1,
            "threads": threads, "init_s": t_init, "energy": energy, "natoms": wb.natoms}


def run_reference_gpu(args):
    """The reference's own compiled CUDA ops (built for sm_100a from its sources into
    oracle/_ref) on this GPU, FP64 and FP32, CUDA-graph replay of forward + backward as the
    reference's perf_op does (torchff/test_utils.py:52-146), L2 flushed before each timed
    step. Runs in a process of its own: the reference's libraries register
    torch.ops.torchff like libtffb200 does. Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import glob

    if args.workload not in ("water3000", "water216", "water100k"):
        print(json.dumps({"impl": "reference-gpu", "unavailable": f"no reference GPU run for {args.workload}"}))
        return
    if not glob.glob(os.path.join(REPO, "oracle", "_ref", "*", "*.so")):
        print(json.dumps({"impl": "reference-gpu", "unavailable": "the reference's CUDA ops are not built "
                          "(oracle/_ref is empty; oracle/build_ref.py builds them)"}))
        return
    import torch

    from oracle import ref_gpu

    torch.cuda.set_device(0)
    clocks = ClockSampler(0)
    clocks.start()
    clocks.begin()
    r = ref_gpu.measure(args.workload, max(args.steps, 1), max(args.warmup, 3), check=True)
    clocks.end()
    clocks.stop()
    line = {
        "impl": "reference-gpu",
        "metric": METRIC if args.workload == "water3000" else f"{args.workload} PME energy+force evals/s",
        "value": round(r["fp64_evals_per_s"], 2), "unit": "evals/s", "n_gpus": 1, "steps": max(args.steps, 1),
        "warmup": max(args.warmup, 3), "ms_per_step": round(r["fp64_ms_per_eval"], 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded TIP3P lattice box, seed 0)",
        "config": {"workload": f"{args.workload}: {WORKLOAD_TEXT[args.workload]}",
                   "path": "reference CUDA ops (oracle/_ref): build_neighbor_list_cell_list + "
                           "compute_lennard_jones_energy (type tables) + compute_multipolar_energy_from_atom_pairs "
                           "(rank 0, pairs_excl) + 138.935456 x pme_long_range, energy + backward",
                   "timing": f"{r['fp64_timing_mode']}, {r['l2']}, median of the per-step CUDA-event times"},
        "fp64": {"evals_per_s": round(r["fp64_evals_per_s"], 2), "ms_per_eval": round(r["fp64_ms_per_eval"], 5),
                 "mode": r["fp64_timing_mode"], "capture_error": r.get("fp64_capture_error"),
                 "ms_spread": {k: round(v, 5) for k, v in r["fp64_ms_spread"].items()},
                 "energy_rel_err_vs_oracle": r.get("fp64_energy_rel_err_vs_oracle"),
                 "force_rel_rms_vs_oracle": r.get("fp64_force_rel_rms_vs_oracle")},
        "fp32": {"evals_per_s": round(r["fp32_evals_per_s"], 2), "ms_per_eval": round(r["fp32_ms_per_eval"], 5),
                 "mode": r["fp32_timing_mode"], "capture_error": r.get("fp32_capture_error"),
                 "ms_spread": {k: round(v, 5) for k, v in r["fp32_ms_spread"].items()},
                 "energy_rel_err_vs_oracle": r.get("fp32_energy_rel_err_vs_oracle"),
                 "force_rel_rms_vs_oracle": r.get("fp32_force_rel_rms_vs_oracle")},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def reference_gpu_leg(args, workload: str | None = None, steps: int | None = None) -> dict:
    """Runs the reference-gpu arm in a child process (after our timed regions) and returns
    its line, or the reason it did not run."""
    steps = steps if steps is not None else min(max(args.steps, 20), 200)
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference-gpu", "--workload", workload or args.workload,
           "--steps", str(steps), "--warmup", str(max(args.warmup, 3))]
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference GPU run took longer than 600 s"}
    for ln in reversed(p.stdout.splitlines()):
        if ln.startswith("{"):
            try:
                return json.loads(ln)
            except ValueError:
                break
    return {"unavailable": f"exit {p.returncode}: {(p.stderr or '').strip().splitlines()[-1:]}"}


def _ref_worker_init():
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"


def _ref_eval(task):
    workload, seed = task
    from oracle import oracle as O

    if workload == "serving":
        import numpy as np

        from torchff_b200.water import serving_water_box

        n = np.exp(np.random.default_rng(seed).uniform(math.log(64), math.log(4000))).astype(int)
        wb = serving_water_box(int(n), seed=seed)
    else:
        wb = water_box(workload, seed)
    t0 = time.perf_counter()
    O.fixed_charge_energy(wb.coords, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                          wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid, 138.935456)
    return time.perf_counter() - t0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    if args.workload == "water100k":
        print(json.dumps({"impl": "reference", "unavailable": "the reference CPU path keeps an O(N^2) all-pairs "
                          "buffer (~720 GB at 300,000 atoms); not run"}))
        return
    ref = import_reference_cpu() if args.workload != "serving" else None
    if ref is not None:
        r = run_reference_cpu(args, ref)
        line = {
            "impl": "reference",
            "metric": METRIC if args.workload == "water3000" else f"{args.workload} PME energy+force evals/s",
            "value": round(r["value"], 4), "unit": "evals/s", "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": r["warmup"], "ms_per_step": round(r["ms_per_step"], 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded TIP3P lattice box, seed 0: the box rank 0 of the other arm evaluates)",
            "config": {"workload": f"{args.workload}: {WORKLOAD_TEXT[args.workload]}",
                       "path": "reference torchff (baseline/_ref) pure-torch path: NeighborList + Vdw(LennardJones, "
                               "type tables) + MultipolarInteraction(rank 0, pairs_excl) + 138.935456 x PME, "
                               "use_customized_ops=False, FP64, energy + backward()",
                       "parallelism": f"one process, torch.set_num_threads({r['threads']})",
                       "one_off_init_s": round(r["init_s"], 3),
                       "energy_kj_mol": r["energy"]},
            "cpu_baseline": {"value": round(r["value"], 4), "unit": "evals/s", "cores": r["threads"],
                             "kind": "reference",
                             "sample": f"{r['steps']} full evaluations of the {r['natoms']}-atom box (each a step), "
                                       f"after {r['warmup']} untimed; bounded to ~4 min; NeighborList construction "
                                       f"({r['init_s']:.1f} s, all-pairs buffer) timed apart"},
            "e2e": {"value": round(r["value"], 4), "unit": "evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    workers = max(1, min(os.cpu_count() or 1, 16, max(args.steps, 1)))
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers, initializer=_ref_worker_init) as pool:
        warm = pool.map(_ref_eval, [(args.workload, 1000 + i) for i in range(max(min(args.warmup, 2 * workers),
                                                                                 workers))])
        # bounded sample: at most ~90 s of wall time for the timed evaluations
        t_eval = statistics.median(warm)
        n_eval = max(workers, min(args.steps, int(90.0 * workers / max(t_eval, 1e-3))))
        t0 = time.perf_counter()
        per = pool.map(_ref_eval, [(args.workload, i) for i in range(n_eval)])
        wall = time.perf_counter() - t0
    value = n_eval / wall
    serving = args.workload == "serving"
    line = {
        "impl": "reference",
        "metric": (METRIC if args.workload == "water3000" else
                   "serving systems/s (continuous batching, saturation)" if serving else
                   f"{args.workload} PME energy+force evals/s"),
        "value": round(value, 4),
        "unit": "systems/s" if serving else "evals/s",
        "n_gpus": args.gpus,
        "steps": n_eval,
        "warmup": len(warm),
        "ms_per_step": round(wall / n_eval * 1e3, 2),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded TIP3P lattice boxes)",
        "config": {"workload": f"{args.workload}: {WORKLOAD_TEXT[args.workload]}",
                   "path": "numpy restatement of the reference pure-torch path (O(N^2) pair search, LJ type "
                           "tables, real-space Ewald with exclusion correction, PME), analytic forces",
                   "parallelism": f"{workers} host processes, one evaluation each at a time"},
        "cpu_baseline": {"value": round(value, 4), "unit": "systems/s" if serving else "evals/s", "cores": workers,
                         "kind": "port",
                         "sample": f"{n_eval} full evaluations (of {args.steps} requested steps, bounded to ~90 s) "
                                   f"spread over {workers} single-thread processes"},
        "e2e": {"value": round(value, 4), "unit": "systems/s" if serving else "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def free_port() -> int:
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch_command(argv: list[str], nproc: int, port: int) -> list[str]:
    """The command that runs this script as `nproc` ranks on this node (one per GPU)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + argv


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # started as a plain process: run the N ranks under torch.distributed.run and pass
        # on their exit status (rank 0 prints the line)
        cmd = relaunch_command(sys.argv[1:], args.gpus, free_port())
        raise SystemExit(subprocess.call(cmd))
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference-gpu":
        run_reference_gpu(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
