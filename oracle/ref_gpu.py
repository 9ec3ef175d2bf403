"""The reference's own CUDA operators on the GPU: timing baseline and an oracle cross-check.

TEST/MEASUREMENT INFRASTRUCTURE. Loads the reference's compiled extension libraries from
``oracle/_ref`` (built by ``oracle/build_ref.py``). These register ``torch.ops.torchff``
exactly like torchff_b200 does, so this script always runs in a process of its own.

It evaluates the nonbonded part of the reference's TIP3P model
(``examples/tip3p/model.py:100-133``): ``build_neighbor_list_cell_list`` with the water
exclusions, ``compute_lennard_jones_energy`` with type tables,
``compute_multipolar_energy_from_atom_pairs`` (rank 0, Ewald, ``pairs_excl``) and
138.935456 x ``pme_long_range``, energy + backward. Timing follows the reference's
``perf_op`` (``torchff/test_utils.py:52-146``): warm-up, then forward + backward captured in
one CUDA graph and replayed. Prints one JSON line per precision.

    python oracle/ref_gpu.py [--workload water3000] [--steps 200] [--check]
"""
from __future__ import annotations

import argparse
import glob
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)


def water_module():
    """torchff_b200/water.py loaded by path: importing the torchff_b200 package would
    register its own torch.ops.torchff schemas, which clash with the reference's."""
    import importlib.util

    path = os.path.join(REPO, "torchff-lib_b200", "torchff_b200", "water.py")
    spec = importlib.util.spec_from_file_location("_tff_water", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["_tff_water"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_reference_ops() -> list[str]:
    import torch

    libs = sorted(glob.glob(os.path.join(HERE, "_ref", "*", "*.so")))
    if not libs:
        raise SystemExit("oracle/_ref has no reference libraries (run oracle/build_ref.py)")
    for lib in libs:
        torch.ops.load_library(lib)
    return libs


def moduli(K: int, dtype):
    """B-spline moduli with the reference's float32 buffers (torchff/pme.py:21-28)."""
    import torch

    m = [0.0, 1.0 / 120, 26.0 / 120, 66.0 / 120, 26.0 / 120, 1.0 / 120]

    def mod(count):
        k = torch.arange(count, dtype=torch.float64)
        out = torch.zeros(count, dtype=torch.float64)
        for j in range(-3, 3):
            out += m[j + 3] * torch.cos(2 * math.pi * j * k / K)
        return out.to(torch.float32).to(dtype).cuda()

    return mod(K), mod(K), mod(K // 2 + 1)


def build_inputs(wb, dtype):
    import torch

    from oracle import oracle as O

    dev = "cuda"
    rp, col = (torch.tensor(a, device=dev) for a in O.exclusions_coo_to_csr(wb.nblist_exclusions, wb.natoms))
    return {
        "coords": torch.tensor(wb.coords, dtype=dtype, device=dev, requires_grad=True),
        "box": torch.tensor(wb.box, dtype=dtype, device=dev),
        "q": torch.tensor(wb.charges, dtype=dtype, device=dev),
        "sig": torch.tensor(wb.sigma_table, dtype=dtype, device=dev),
        "eps": torch.tensor(wb.epsilon_table, dtype=dtype, device=dev),
        "types": torch.tensor(wb.atom_types, dtype=torch.int64, device=dev),
        "excl": torch.tensor(wb.coulomb_exclusions, dtype=torch.int64, device=dev),
        "rp": rp, "col": col,
        "mod": moduli(wb.grid, dtype),
        "cap": int(wb.natoms * 4 / 3 * 3.1416 * wb.cutoff ** 3 * 100 / 2 * 1.2),
    }


def energy(wb, d):
    import torch

    ops = torch.ops.torchff
    x, b = d["coords"], d["box"]
    pairs, _ = ops.build_neighbor_list_cell_list(x.detach(), b, wb.cutoff, d["cap"], d["rp"], d["col"], False)
    e_lj = ops.compute_lennard_jones_energy(x, pairs, b, d["sig"], d["eps"], wb.cutoff, d["types"])
    e_c = ops.compute_multipolar_energy_from_atom_pairs(x, b, pairs, d["excl"], d["q"], None, None, wb.cutoff,
                                                         wb.alpha, 138.935456)
    e_p = ops.pme_long_range(x, b, d["q"], None, None, wb.grid, wb.alpha, *d["mod"]) * 138.935456
    return e_lj + e_c + e_p


def time_graph(wb, d, steps: int, warmup: int = 5, flush_l2: bool = True) -> tuple[list, str, str]:
    """ms of each of `steps` forwards + backwards: CUDA-graph replay as in torchff/test_utils.py:52-146, or,
    when the composition cannot be captured, eager calls. With flush_l2 a 256 MiB device
    write (larger than the 126 MB L2) runs before every timed replay, outside its events.

    Capture is tried in torch's "global", "thread_local" and "relaxed" error modes in turn.
    A captured graph is used only if one replay reproduces the eager energy and forces, i.e.
    the graph does the whole evaluation. The reference's ops accumulate with atomics (and
    the LJ force accumulation races, so eager forces differ from call to call), so
    "reproduces" means: within 1e-12 relative, or within 4x the largest difference seen
    between three eager calls. Returns (per-step ms, mode, the capture errors of the
    modes that failed)."""
    import torch

    x = d["coords"]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(warmup):
            x.grad = None
            energy(wb, d).backward()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    eager = []
    for _ in range(3):
        x.grad = None
        e = energy(wb, d)
        e.backward()
        eager.append((float(e.item()), x.grad.detach().clone()))
    e_ref, g_ref = eager[0]
    e_tol = 1e-12 * abs(e_ref) + 4 * max(abs(ei - ej) for ei, _ in eager for ej, _ in eager)
    g_tol = 1e-12 * float(g_ref.abs().max()) + 4 * max(float((gi - gj).abs().max()) for _, gi in eager
                                                         for _, gj in eager)
    flush = torch.empty(256 * 1024 * 1024 if flush_l2 else 1, dtype=torch.uint8, device="cuda")
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    errors = []
    run, mode = None, "eager"
    for cmode in ("global", "thread_local", "relaxed"):
        try:
            g = torch.cuda.CUDAGraph()
            x.grad = None
            with torch.cuda.graph(g, capture_error_mode=cmode):
                e = energy(wb, d)
                e.backward()
            g.replay()
            torch.cuda.synchronize()
            same = (abs(float(e.item()) - e_ref) <= e_tol
                    and float((x.grad - g_ref).abs().max()) <= g_tol)
            if not same:
                errors.append(f"{cmode}: captured, but a replay does not reproduce the eager result")
                continue
            for _ in range(warmup):
                g.replay()
            torch.cuda.synchronize()
            run, mode = g.replay, f"cuda_graph ({cmode} capture)"
            break
        except Exception as exc:  # capture invalidated, e.g. by a host synchronisation inside an op
            msg = str(exc).strip().splitlines()[0][:200] if str(exc).strip() else ""
            errors.append(f"{cmode}: {type(exc).__name__}: {msg}")
            torch.cuda.synchronize()
    if run is None:
        def run():
            x.grad = None
            energy(wb, d).backward()
    times = []
    for i in range(steps):
        flush.fill_(i & 0xff)
        a.record()
        run()
        z.record()
        z.synchronize()
        times.append(a.elapsed_time(z))
    return times, mode, "; ".join(errors)


def measure(workload: str = "water3000", steps: int = 200, warmup: int = 5, check: bool = True,
            flush_l2: bool = True) -> dict:
    """FP64 and FP32 evaluations of the box (seed 0) through the reference's ops: energy,
    timing and, with check, the energy and force error against the FP64 oracle."""
    import numpy as np
    import torch

    W = water_module()
    libs = load_reference_ops()
    wb = {"water216": W.water_box_216, "water3000": W.water_box_3000, "water100k": W.water_box_100k}[workload](0)
    out = {"workload": workload, "natoms": wb.natoms, "libraries": [os.path.relpath(p, REPO) for p in libs],
           "l2": "flushed before every timed step (256 MiB device write)" if flush_l2 else "not flushed"}
    forces = {}
    for name, dtype in (("fp64", torch.float64), ("fp32", torch.float32)):
        d = build_inputs(wb, dtype)
        e = energy(wb, d)
        e.backward()
        out[f"{name}_energy"] = float(e.item())
        forces[name] = (-d["coords"].grad).double().cpu().numpy()
        times, mode, error = time_graph(wb, d, steps, warmup, flush_l2)
        # eager calls are bounded by the host (the ops synchronise), whose share of the box
        # varies from run to run: the median step is the figure, the spread is reported beside it
        ms = float(np.median(times))
        out[f"{name}_ms_per_eval"], out[f"{name}_timing_mode"] = ms, mode
        out[f"{name}_ms_spread"] = {"mean": float(np.mean(times)), "p10": float(np.percentile(times, 10)),
                                    "p90": float(np.percentile(times, 90)), "min": float(np.min(times))}
        if error:
            out[f"{name}_capture_error"] = error
        out[f"{name}_evals_per_s"] = 1e3 / ms
    if check and workload == "water100k":
        # the oracle at 300,000 atoms: cell-binned real-space energy, PME energy, and the forces
        # on 256 sampled atoms (distances to every atom + PME gathered there)
        from oracle import oracle as O

        k = 138.935456
        e_real = O.real_space_cells(wb.coords, wb.box, wb.charges, wb.atom_types, wb.sigma_table, wb.epsilon_table,
                                    wb.coulomb_exclusions, wb.cutoff, wb.alpha, k)
        subset = np.random.default_rng(11).choice(wb.natoms, 256, replace=False)
        e_pme, g_pme = O.pme_subset(wb.coords, wb.box, wb.charges, wb.alpha, wb.grid, subset)
        g = O.real_space_grad_subset(wb.coords, wb.box, wb.charges, wb.atom_types, wb.sigma_table, wb.epsilon_table,
                                     wb.coulomb_exclusions, wb.cutoff, wb.alpha, k, subset) + k * g_pme
        total = e_real + k * e_pme
        for name, f in forces.items():
            out[f"{name}_energy_rel_err_vs_oracle"] = abs(out[f"{name}_energy"] - total) / abs(total)
            out[f"{name}_force_rel_rms_vs_oracle"] = float(np.sqrt(np.mean((f[subset] + g) ** 2)) /
                                                         np.sqrt(np.mean(g ** 2)))
        out["oracle_energy"] = total
        out["force_check"] = "256 sampled atoms"
    elif check:
        from oracle import oracle as O

        ref = O.fixed_charge_energy(wb.coords, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                    wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                    138.935456)
        f0 = -ref["grad_coords"]
        for name, f in forces.items():
            out[f"{name}_energy_rel_err_vs_oracle"] = abs(out[f"{name}_energy"] - ref["total"]) / abs(ref["total"])
            out[f"{name}_force_rel_rms_vs_oracle"] = float(np.sqrt(np.mean((f - f0) ** 2)) / np.sqrt(np.mean(f0 ** 2)))
        out["oracle_energy"] = ref["total"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="water3000", choices=["water216", "water3000", "water100k"])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--check", action="store_true", help="compare the energy/forces with the FP64 oracle")
    ap.add_argument("--no-flush", action="store_true", help="no L2 flush between timed steps")
    args = ap.parse_args()
    print(json.dumps(measure(args.workload, args.steps, check=args.check, flush_l2=not args.no_flush)), flush=True)


if __name__ == "__main__":
    main()
