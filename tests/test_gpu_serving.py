"""Batched evaluation (tff_batch) and the continuous-batching server (tff_server).

Each system of a batch must give the single-system result. The cluster lists and the
fixed-point real-space sums are the same; the reciprocal part of a batch uses a direct DFT
where the single-system path uses cuFFT, so the two agree to FP32 transform rounding:
energy within 1e-8 of the summed magnitudes of the energy terms (the total is a
near-cancelling sum), forces 1e-6 of the largest component. Within the batched path the
summation order of every reduction and transform depends on the system alone, so a
system's result alone and in a mix agree to 1e-9 (energy, relative) and 1e-6 (forces).
FP64 batches match the FP64 oracle to 1e-10 (energy) and 1e-8 (forces). The request sizes
include boxes shorter than twice the cutoff (64 and 150 waters), evaluated with the
minimum-image convention like the single-system path and the oracle.
"""
import numpy as np
import pytest
import torch

from gpu_util import rel, rel_max, rel_rms, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RC = 0.9
NS = [64, 150, 333, 900, 2500, 4000]


def _boxes(ns, seed0=0):
    from torchff_b200.serving import SystemSpec
    from torchff_b200.water import serving_water_box

    wbs = [serving_water_box(n, seed=seed0 + k) for k, n in enumerate(ns)]
    return wbs, [SystemSpec.from_water_box(w) for w in wbs]


def _single(wb, dtype):
    from torchff_b200.system import FixedChargeSystem

    s = FixedChargeSystem.from_water_box(wb, dtype=dtype)
    return s.evaluate(t(wb.coords, dtype), t(wb.box, dtype), terms=True)


def _evaluator(dtype, wbs):
    from torchff_b200.serving import BatchEvaluator

    return BatchEvaluator(RC, wbs[0].alpha, dtype, max_systems=32, max_atoms=100_000, max_grid_points=2_000_000)


@pytest.fixture(scope="module")
def mixed_boxes():
    return _boxes(NS)


def test_batch_matches_single_system_mixed(mixed_boxes):
    wbs, specs = mixed_boxes
    ev = _evaluator(torch.float32, wbs)
    e, f = ev.evaluate(specs)
    torch.cuda.synchronize()
    assert ev.status() == 0
    for k, wb in enumerate(wbs):
        ref = _single(wb, torch.float32)
        scale = float(ref["terms"].abs().sum())
        assert abs(e[k].item() - ref["energy"].item()) < 1e-8 * scale, wb.n_waters
        assert rel_max(f[k], ref["forces"]) < 1e-6, wb.n_waters


def test_batch_fp64_matches_oracle():
    wbs, specs = _boxes([64, 150, 333], seed0=10)
    ev = _evaluator(torch.float64, wbs)
    e, f = ev.evaluate(specs)
    torch.cuda.synchronize()
    for k, wb in enumerate(wbs):
        ref = O.fixed_charge_energy(wb.coords, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                    wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                    138.935456)
        assert rel(e[k].item(), ref["total"]) < 1e-10, wb.n_waters
        assert rel_max(f[k], -ref["grad_coords"]) < 1e-8, wb.n_waters


def test_result_alone_equals_result_in_a_mix(mixed_boxes):
    wbs, specs = mixed_boxes
    ev = _evaluator(torch.float32, wbs)
    target = specs[3]
    e1, f1 = ev.evaluate([target])
    e1, f1 = e1.clone(), f1[0].clone()
    # a mix with the same K twice more (a batched FFT group of 3) and other sizes around it
    others, _ = _boxes([900, 900, 64, 4000, 150], seed0=50)
    from torchff_b200.serving import SystemSpec

    mix = [SystemSpec.from_water_box(w) for w in others[:2]] + [target] + [SystemSpec.from_water_box(w) for w in others[2:]]
    assert all(s.pme_grid == target.pme_grid for s in mix[:3])
    e2, f2 = ev.evaluate(mix)
    torch.cuda.synchronize()
    assert rel(e2[2].item(), e1.item()) < 1e-9
    assert rel_max(f2[2], f1) < 1e-6


def test_server_results_match_batch_and_timestamps():
    from torchff_b200.serving import Server

    rng = np.random.default_rng(5)
    ns = np.exp(rng.uniform(np.log(64), np.log(2000), 40)).astype(int)
    wbs, specs = _boxes(ns, seed0=100)
    srv = Server(RC, wbs[0].alpha, torch.float32, lanes=2, max_systems_per_batch=16, hbm_budget_bytes=2 << 30)
    reqs = [srv.submit(s) for s in specs]
    srv.drain(timeout=120)
    st = srv.stats()
    assert st["systems_done"] == len(specs) and st["batches"] >= 3 and st["max_batch_systems"] <= 16
    ev = _evaluator(torch.float32, wbs)
    for k in range(0, len(specs), 7):
        e, f = ev.evaluate([specs[k]])
        torch.cuda.synchronize()
        en, fn = reqs[k].wait()
        assert rel(en, e.item()) < 1e-9
        assert rel_max(fn, f[0]) < 1e-6
    for r in reqs:
        a, b, c = r.times()
        assert a <= b <= c
        r.release()
    srv.close()


def test_server_request_alone_equals_request_in_a_mix(mixed_boxes):
    from torchff_b200.serving import Server

    wbs, specs = mixed_boxes
    srv = Server(RC, wbs[0].alpha, torch.float32, lanes=3, max_systems_per_batch=8, hbm_budget_bytes=2 << 30)
    alone = srv.submit(specs[4])
    ea, fa = alone.wait(timeout=60)
    fa = fa.copy()
    others, ospecs = _boxes([120, 700, 2000, 64, 3000, 400, 1000, 250], seed0=200)
    reqs = [srv.submit(s) for s in ospecs[:4]] + [srv.submit(specs[4])] + [srv.submit(s) for s in ospecs[4:]]
    eb, fb = reqs[4].wait(timeout=60)
    srv.drain(timeout=60)
    assert rel(eb, ea) < 1e-9
    assert rel_max(fb, fa) < 1e-6
    srv.close()


def test_faulty_requests_are_refused_and_the_rest_served():
    """Failures injected on the host. Requests beyond the per-request limits (16,386 atoms,
    a 97^3 PME grid; a lane always has room for one request within them), one with an
    exclusion index outside its own system and one with more than 8 excluded partners for an
    atom are refused at submission (invalid argument); a wait on a held
    server gives up after its timeout and the request still completes once the hold is
    lifted. The requests around the refused ones are served with the results a batch of
    their own gives."""
    from dataclasses import replace

    from torchff_b200.serving import Server, SystemSpec
    from torchff_b200.water import serving_water_box

    wbs, specs = _boxes([150, 300, 500], seed0=300)
    srv = Server(RC, wbs[0].alpha, torch.float32, lanes=2, max_systems_per_batch=8, hbm_budget_bytes=64 << 20)
    huge = SystemSpec.from_water_box(serving_water_box(5462, seed=1))
    assert huge.natoms > 16384
    with pytest.raises(RuntimeError, match="invalid"):
        srv.submit(huge)
    with pytest.raises(RuntimeError, match="invalid"):
        srv.submit(replace(specs[0], pme_grid=97))
    n0 = specs[0].natoms
    with pytest.raises(RuntimeError, match="invalid"):
        srv.submit(replace(specs[0], excl_pairs=np.array([[0, n0]], dtype=np.int64)))
    with pytest.raises(RuntimeError, match="invalid"):
        srv.submit(replace(specs[0], excl_pairs=np.array([[0, j] for j in range(1, 10)], dtype=np.int64)))
    srv.hold(True)
    held = srv.submit(specs[1])
    with pytest.raises(RuntimeError, match="timeout"):
        held.wait(timeout=0.2)
    srv.hold(False)
    reqs = [held] + [srv.submit(s) for s in specs]
    srv.drain(timeout=60)
    assert srv.stats()["systems_done"] == 4
    ev = _evaluator(torch.float32, wbs)
    for r, s in zip(reqs, [specs[1]] + specs):
        e, f = ev.evaluate([s])
        torch.cuda.synchronize()
        en, fn = r.wait(timeout=10)
        assert rel(en, e.item()) < 1e-9
        assert rel_max(fn, f[0]) < 1e-6
        r.release()
    srv.close()


def test_batch_triclinic_system_matches_oracle():
    """A sheared box (rows a, b + (0.15, 0, 0), c + (0.1, 0.12, 0)) next to an orthorhombic one
    in one FP64 batch: each against the oracle (energy 1e-10 relative, forces 1e-8 of the
    largest)."""
    from dataclasses import replace

    wbs, specs = _boxes([300, 900], seed0=40)
    box = wbs[0].box.copy()
    box[1, 0] += 0.15
    box[2, 0] += 0.1
    box[2, 1] += 0.12
    specs[0] = replace(specs[0], box=box)
    ev = _evaluator(torch.float64, wbs)
    e, f = ev.evaluate(specs)
    torch.cuda.synchronize()
    assert ev.status() == 0
    for k, (wb, b) in enumerate(zip(wbs, (box, wbs[1].box))):
        ref = O.fixed_charge_energy(wb.coords, b, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                    wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                    138.935456)
        assert rel(e[k].item(), ref["total"]) < 1e-10, k
        assert rel_max(f[k], -ref["grad_coords"]) < 1e-8, k


def test_graph_replay_serves_other_compositions():
    """Evaluations through one set of device buffers: the second call with the same buffers
    and DFT size class captures the device part in a CUDA graph, and later calls of that
    class replay it with other systems in the buffers. Every result is bit-identical to a
    direct evaluation of the same systems by another batch object, and a class whose graph
    is not yet captured runs directly."""
    from torchff_b200.serving import BatchEvaluator, exclusion_table

    # grid sides: a and c at most 30 (DFT class 52), b 54 (5,000 waters; the larger class)
    sizes = {"a": [64, 900, 333], "b": [5000, 150], "c": [333, 64, 900, 150]}
    boxes = {k: _boxes(v, seed0=40 + 10 * i) for i, (k, v) in enumerate(sizes.items())}
    cap_atoms, cap_sys = 30_000, 8
    wbs0 = boxes["a"][0]
    ev = BatchEvaluator(RC, wbs0[0].alpha, torch.float32, max_systems=cap_sys, max_atoms=cap_atoms,
                        max_grid_points=2_000_000)
    ref_ev = BatchEvaluator(RC, wbs0[0].alpha, torch.float32, max_systems=cap_sys, max_atoms=cap_atoms,
                            max_grid_points=2_000_000)
    dev, f32 = torch.device("cuda"), torch.float32
    buf = {"coords": torch.empty(3 * cap_atoms, dtype=f32, device=dev),
           "boxes": torch.empty(9 * cap_sys, dtype=f32, device=dev),
           "charges": torch.empty(cap_atoms, dtype=f32, device=dev),
           "sigma": torch.empty(cap_atoms, dtype=f32, device=dev),
           "epsilon": torch.empty(cap_atoms, dtype=f32, device=dev),
           "excl": torch.empty(8 * cap_atoms, dtype=torch.int32, device=dev),
           "energies": torch.empty(cap_sys, dtype=torch.float64, device=dev),
           "forces": torch.empty(3 * cap_atoms, dtype=f32, device=dev)}

    def packed_in_buffers(specs):
        natoms = np.array([s.natoms for s in specs], dtype=np.int64)
        n = int(natoms.sum())
        cat = lambda a: torch.from_numpy(np.concatenate(a)).to(dev, f32)  # noqa: E731
        buf["coords"][:3 * n] = cat([s.coords.reshape(-1) for s in specs])
        buf["boxes"][:9 * len(specs)] = cat([s.box.reshape(-1) for s in specs])
        buf["charges"][:n] = cat([s.charges for s in specs])
        buf["sigma"][:n] = cat([s.sigma for s in specs])
        buf["epsilon"][:n] = cat([s.epsilon for s in specs])
        ex = np.concatenate([exclusion_table(s.natoms, s.excl_pairs) for s in specs]).reshape(-1)
        buf["excl"][:ex.size] = torch.from_numpy(ex).to(dev)
        return {"natoms": natoms, "pme_grid": np.array([s.pme_grid for s in specs], dtype=np.int32),
                "coords": buf["coords"], "boxes": buf["boxes"], "charges": buf["charges"], "sigma": buf["sigma"],
                "epsilon": buf["epsilon"], "excl": buf["excl"], "energies": buf["energies"],
                "forces": buf["forces"]}, n

    kept = []  # reference packs stay allocated, so each reference call has new addresses

    def check(name):
        specs = boxes[name][1]
        p, n = packed_in_buffers(specs)
        ev.evaluate_packed(p)
        e = p["energies"][:len(specs)].clone()
        f = p["forces"][:3 * n].clone()
        kept.append(ref_ev.pack(specs))
        ref_ev.evaluate_packed(kept[-1])  # always the direct path
        torch.cuda.synchronize()
        assert ev.status() == 0 and ref_ev.status() == 0
        assert torch.equal(e, kept[-1]["energies"]), name
        assert torch.equal(f, kept[-1]["forces"].reshape(-1)), name

    check("a")                        # direct
    check("a")                        # same buffers and class: captured, then replayed
    assert ev.graph_launches() == 1
    check("c")                        # the class-52 graph replayed with other systems
    assert ev.graph_launches() == 2
    check("b")                        # the larger class: direct
    assert ev.graph_launches() == 2
    check("b")                        # captured
    check("a")                        # the class-52 graph again
    assert ev.graph_launches() == 4
    assert ref_ev.graph_launches() == 0


def test_batch_coordinates_outside_the_primary_cell(mixed_boxes):
    """Batched evaluation of systems whose waters were moved by up to 3 box vectors: energies
    and forces as for the original coordinates (mixed precision; the coordinates' FP32
    rounding at a few box lengths bounds the agreement: forces 2e-5 RMS and 1e-4 of the
    largest, energy 1e-6 of the summed term magnitudes)."""
    import dataclasses

    from torchff_b200.serving import SystemSpec

    wbs, specs = mixed_boxes
    moved = []
    for k, wb in enumerate(wbs[:4]):
        rng = np.random.default_rng(100 + k)
        n = np.rint(rng.uniform(-3, 3, (wb.n_waters, 3)))
        moved.append(dataclasses.replace(wb, coords=wb.coords + np.repeat(n @ wb.box, 3, axis=0)))
    ev = _evaluator(torch.float32, wbs)
    e0, f0 = ev.evaluate(specs[:4])
    e1, f1 = ev.evaluate([SystemSpec.from_water_box(w) for w in moved])
    torch.cuda.synchronize()
    assert ev.status() == 0
    for k, wb in enumerate(wbs[:4]):
        scale = float(_single(wb, torch.float32)["terms"].abs().sum())
        assert abs(e1[k].item() - e0[k].item()) < 1e-6 * scale, wb.n_waters
        assert rel_rms(f1[k], f0[k]) < 2e-5, wb.n_waters
        assert rel_max(f1[k], f0[k]) < 1e-4, wb.n_waters
