"""Multi-rank host logic on CPU (gloo, world size 2): frames of a force-matching step are
split across ranks and the parameter gradients summed with one all-reduce; the result must
equal one process doing every frame. Timings reduce with a max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import REPO

NFRAMES = 4


def _problem():
    import sys

    sys.path.insert(0, os.path.join(REPO, "torchff-lib_b200"))
    import importlib.util

    spec = importlib.util.spec_from_file_location("tff_water", os.path.join(REPO, "torchff-lib_b200", "torchff_b200",
                                                                            "water.py"))
    W = importlib.util.module_from_spec(spec)
    sys.modules["tff_water"] = W
    spec.loader.exec_module(W)
    wb = W.make_water_box(32, 1.2, 4, cutoff=0.55, grid=12, seed=4)
    q, s, e = W.force_matching_parameters(wb, seed=5)
    frames = W.perturbed_frames(wb, NFRAMES, 0.005, seed=6)
    targets = np.random.default_rng(7).normal(0.0, 100.0, size=frames.shape)
    return wb, q, s, e, frames, targets


def _frame_grads(frame_ids):
    from oracle import oracle as O
    from oracle import torch_energy as TE

    wb, q, s, e, frames, targets = _problem()
    params = [torch.tensor(a, requires_grad=True) for a in (q, s, e)]
    rp, col = O.exclusions_coo_to_csr(wb.nblist_exclusions, wb.natoms)
    for f in frame_ids:
        pairs = torch.tensor(O.nblist_pairs(frames[f], wb.box, wb.cutoff, rp, col))
        x = torch.tensor(frames[f], requires_grad=True)
        E = TE.fixed_charge_energy(x, torch.tensor(wb.box), *params, pairs, torch.tensor(wb.coulomb_exclusions),
                                   wb.cutoff, wb.alpha, wb.grid)
        (gx,) = torch.autograd.grad(E, x, create_graph=True)
        (torch.mean((-gx - torch.tensor(targets[f])) ** 2) / NFRAMES).backward()
    return [p.grad if p.grad is not None else torch.zeros_like(p) for p in params]


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "torchff-lib_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import importlib.util

    spec = importlib.util.spec_from_file_location("tff_dist", os.path.join(REPO, "torchff-lib_b200", "torchff_b200",
                                                                           "distributed.py"))
    D = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(D)
    mine = D.frame_shard(NFRAMES, rank, world)
    grads = _frame_grads(mine)
    D.allreduce_sum_(grads)
    t = D.max_over_ranks(1.0 + rank, "cpu")
    if rank == 0:
        torch.save({"grads": [g.clone() for g in grads], "max": t, "mine": mine}, out)
    dist.barrier()
    dist.destroy_process_group()


def test_frame_sharded_gradient_allreduce_matches_single_process(tmp_path):
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "r0.pt")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    res = torch.load(out)
    assert res["mine"] == [0, 2] and res["max"] == 2.0
    ref = _frame_grads(range(NFRAMES))
    for a, b in zip(res["grads"], ref):
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-12 * float(b.abs().max()))


def test_bench_starts_its_own_ranks(tmp_path):
    """`python bench.py --gpus 2` started as a plain process re-runs itself as 2 ranks under
    torch.distributed.run (127.0.0.1); rank 0 prints the one JSON line and the other rank
    exits 0. Driven through the reference arm's quick path (the 300,000-atom workload it does
    not run), which needs no GPU."""
    import json
    import subprocess
    import sys

    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "2", "--impl", "reference",
                        "--workload", "water100k", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, env=env, cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(ln) for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and "unavailable" in lines[0]


def test_bench_relaunch_command():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(REPO, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    cmd = bench.relaunch_command(["--gpus", "4", "--steps", "3"], 4, 29501)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-3:] == ["--gpus", "4", "--steps", "3"][-3:] and cmd[cmd.index("--master-port") + 1] == "29501"
