"""Fused system (cluster-pair build + real-space tile kernel + PME) vs the oracle.

FP64: energy 1e-10 relative, forces 1e-8 of their max magnitude. Mixed precision (FP32
arithmetic, fixed-point forces, FP64 energy): energy error below 1e-6 of the summed
component magnitudes |E_LJ| + |E_real| + |k E_pme| (the total is a near-cancelling sum:
-422 kJ/mol from terms of +-5e4 kJ/mol for 216 waters), force RMS error below 1e-5
relative to the FP64 oracle; results bit-identical run to run.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_util import rel, rel_max, rel_rms, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mixed_energy_err(e, ref):
    scale = abs(ref["lj"]) + abs(ref["coul_real"]) + abs(138.935456 * ref["pme_raw"])
    return abs(float(e) - ref["total"]) / scale


def _oracle(wb, coords=None):
    x = wb.coords if coords is None else coords
    return O.fixed_charge_energy(x, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                 wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                 138.935456)


@pytest.fixture(scope="module")
def ref216():
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    return wb, _oracle(wb)


@pytest.fixture(scope="module")
def ref3000():
    from torchff_b200.water import water_box_3000

    wb = water_box_3000()
    return wb, _oracle(wb)


def test_oracle_composition_matches_golden(ref216):
    wb, ref = ref216
    g = np.load(os.path.join(GOLDEN, "water216.npz"))
    total = float(g["e_lj"] + g["e_coul"] + 138.935456 * g["e_pme"])
    assert rel(ref["total"], total) < 1e-12


def test_fp64_water216(ref216):
    from torchff_b200.system import FixedChargeSystem

    wb, ref = ref216
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float64)
    out = sysm.evaluate(t(wb.coords), t(wb.box), grad_charges=True, terms=True)
    assert rel(out["energy"].item(), ref["total"]) < 1e-10
    assert rel_max(out["forces"], -ref["grad_coords"]) < 1e-8
    assert rel_max(out["grad_charges"], ref["grad_charges"]) < 1e-8
    terms = out["terms"].cpu().numpy()
    assert rel(terms[2] + terms[3], 138.935456 * ref["pme_raw"]) < 1e-10
    assert sysm.status() == 0


def test_mixed_water216(ref216):
    from torchff_b200.system import FixedChargeSystem

    wb, ref = ref216
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    out = sysm.evaluate(t(wb.coords, torch.float32), t(wb.box, torch.float32))
    assert _mixed_energy_err(out["energy"].item(), ref) < 1e-6
    assert rel_rms(out["forces"], -ref["grad_coords"]) < 1e-5


def test_mixed_water3000_accuracy_and_determinism(ref3000):
    from torchff_b200.system import FixedChargeSystem

    wb, ref = ref3000
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    x, b = t(wb.coords, torch.float32), t(wb.box, torch.float32)
    outs = [sysm.evaluate(x, b) for _ in range(3)]
    for o in outs[1:]:
        assert torch.equal(o["energy"], outs[0]["energy"]) and torch.equal(o["forces"], outs[0]["forces"])
    assert _mixed_energy_err(outs[0]["energy"].item(), ref) < 1e-6
    assert rel_rms(outs[0]["forces"], -ref["grad_coords"]) < 1e-5
    assert sysm.status() == 0


def test_mixed_shuffled_atoms():
    """A 216-water box with its atoms in a random order (molecules no longer contiguous, the
    exclusions renumbered): repeated mixed-precision evaluations are bit-identical and match
    the oracle, forces mapped back to the original order, within the mixed tolerances."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    perm = np.random.default_rng(3).permutation(wb.natoms)
    inv = np.argsort(perm)
    coords = wb.coords[perm]
    excl = inv[wb.coulomb_exclusions]
    ref = _oracle(wb)
    sysm = FixedChargeSystem(wb.charges[perm], wb.sigma[perm], wb.epsilon[perm], excl, wb.cutoff, wb.alpha, wb.grid,
                             dtype=torch.float32)
    x, b = t(coords, torch.float32), t(wb.box, torch.float32)
    outs = [sysm.evaluate(x, b) for _ in range(3)]
    for o in outs[1:]:
        assert torch.equal(o["energy"], outs[0]["energy"]) and torch.equal(o["forces"], outs[0]["forces"])
    assert _mixed_energy_err(outs[0]["energy"].item(), ref) < 1e-6
    assert rel_rms(outs[0]["forces"][torch.as_tensor(inv, device="cuda")], -ref["grad_coords"]) < 1e-5
    assert sysm.status() == 0


def test_fp64_water3000(ref3000):
    from torchff_b200.system import FixedChargeSystem

    wb, ref = ref3000
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float64)
    out = sysm.evaluate(t(wb.coords), t(wb.box))
    assert rel(out["energy"].item(), ref["total"]) < 1e-10
    assert rel_max(out["forces"], -ref["grad_coords"]) < 1e-8


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_triclinic_box(dtype):
    """A sheared 216-water box (rows a = (L,0,0), b = (0.15,L,0), c = (0.1,0.12,L) nm, every
    perpendicular width above 2 rc): the fused system against the oracle, which takes the
    minimum image through fractional coordinates as torchff/pbc.py:59-62 does."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    L = wb.box[0, 0]
    box = np.array([[L, 0.0, 0.0], [0.15, L, 0.0], [0.1, 0.12, L]])
    ref = O.fixed_charge_energy(wb.coords, box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                138.935456)
    sysm = FixedChargeSystem(wb.charges, wb.sigma, wb.epsilon, wb.coulomb_exclusions, wb.cutoff, wb.alpha,
                             wb.grid, dtype=dtype)
    out = sysm.evaluate(t(wb.coords, dtype), t(box, dtype))
    assert sysm.status() == 0
    if dtype == torch.float64:
        assert rel(out["energy"].item(), ref["total"]) < 1e-10
        assert rel_max(out["forces"], -ref["grad_coords"]) < 1e-8
    else:
        assert _mixed_energy_err(out["energy"].item(), ref) < 1e-6
        assert rel_rms(out["forces"], -ref["grad_coords"]) < 1e-5


@pytest.mark.parametrize("n_waters", [1, 2, 11])
def test_tiny_systems(n_waters):
    """One, two and eleven waters in a 2.0 nm box (rc 0.9 nm, K = 20): one partial cluster,
    and for one water no pair beyond its own excluded ones (exclusion correction and PME
    only). FP64 against the oracle (energy 1e-10, forces 1e-8 of the largest). In mixed
    precision the net force on a lone water is what remains of two terms of about
    k |q_O q_H| / r_OH^2 = 5,300 kJ/mol/nm (the reciprocal sum and the exclusion correction)
    that cancel to a few kJ/mol/nm, so its error is bounded against that term: every force
    component within 1e-6 of it; the energy within the usual mixed tolerance."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import make_water_box

    wb = make_water_box(n_waters, 2.0, 3, 0.9, 20, seed=5)
    ref = _oracle(wb)
    for dtype in (torch.float64, torch.float32):
        sysm = FixedChargeSystem.from_water_box(wb, dtype=dtype)
        out = sysm.evaluate(t(wb.coords, dtype), t(wb.box, dtype))
        assert sysm.status() == 0
        if dtype == torch.float64:
            assert rel(out["energy"].item(), ref["total"]) < 1e-10
            assert rel_max(out["forces"], -ref["grad_coords"]) < 1e-8
        else:
            assert _mixed_energy_err(out["energy"].item(), ref) < 1e-6
            term = 138.935456 * 0.834 * 0.417 / 0.09572 ** 2
            err = np.abs(out["forces"].double().cpu().numpy() + ref["grad_coords"]).max()
            assert err < 1e-6 * term, err


def test_empty_system():
    """A system of no atoms evaluates to zero energy and an empty force array."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    for dtype in (torch.float64, torch.float32):
        sysm = FixedChargeSystem(np.zeros(0), np.zeros(0), np.zeros(0), None, wb.cutoff, wb.alpha, wb.grid,
                                 dtype=dtype)
        out = sysm.evaluate(torch.zeros((0, 3), dtype=dtype, device="cuda"), t(wb.box, dtype))
        assert out["energy"].item() == 0.0 and out["forces"].shape == (0, 3)
        assert sysm.status() == 0


def test_cluster_list_overflow_is_reported(ref216):
    """A neighbour-cluster capacity far below what the box needs (4 clusters, where the
    216-water box's clusters see ~20) drops pairs: the host entry point returns
    TFF_ERR_CAPACITY (RuntimeError), evaluate() raises when check_status is on, and the status
    word says so; the same system with the default capacity evaluates without an error."""
    from torchff_b200.system import FixedChargeSystem

    wb, _ = ref216
    for pinned in (False, True):
        small = FixedChargeSystem.from_water_box(wb, dtype=torch.float32, max_cluster_neighbors=4, check_status=True)
        x = torch.tensor(wb.coords, dtype=torch.float64)
        b = torch.tensor(wb.box, dtype=torch.float64)
        f = torch.zeros_like(x)
        if pinned:
            x, b, f = x.pin_memory(), b.pin_memory(), f.pin_memory()
        with pytest.raises(RuntimeError, match="capacity overflow"):   # TFF_ERR_CAPACITY
            small.evaluate_host(x, b, f)
        assert small.status() & 1
    with pytest.raises(RuntimeError, match="overflow"):
        small.evaluate(t(wb.coords, torch.float32), t(wb.box, torch.float32))
    ok = FixedChargeSystem.from_water_box(wb, dtype=torch.float32, check_status=True)
    f = np.zeros_like(wb.coords)
    ok.evaluate_host(np.ascontiguousarray(wb.coords), np.ascontiguousarray(wb.box), f)
    ok.evaluate(t(wb.coords, torch.float32), t(wb.box, torch.float32))
    assert ok.status() == 0


def test_host_entry_point_matches_device(ref216):
    from torchff_b200.system import FixedChargeSystem

    wb, ref = ref216
    for dtype in (torch.float32, torch.float64):
        sysm = FixedChargeSystem.from_water_box(wb, dtype=dtype)
        dev = sysm.evaluate(t(wb.coords, dtype), t(wb.box, dtype))
        f = np.zeros_like(wb.coords)
        e = sysm.evaluate_host(np.ascontiguousarray(wb.coords), np.ascontiguousarray(wb.box), f)
        if dtype == torch.float32:
            # mixed precision is bit-reproducible: identical results
            assert e == dev["energy"].item()
            assert np.array_equal(f.astype(np.float32), dev["forces"].cpu().numpy())
        else:
            # FP64 mode sums forces with FP64 atomics: equal to rounding, not bitwise
            assert rel(e, dev["energy"].item()) < 1e-13
            assert rel_max(f, dev["forces"]) < 1e-12


def test_host_entry_point_page_locked_buffers(ref216):
    """Page-locked coords/forces take the one-graph path (a 648-atom box: kernels read the
    coordinates and write the forces in host memory, no copies): results equal the device
    path on consecutive calls with new coordinates, on a second pair of buffers, and when the
    box is not page-locked."""
    from torchff_b200.system import FixedChargeSystem

    wb, _ = ref216
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    rng = np.random.default_rng(4)
    bufs = [(torch.empty((wb.natoms, 3), dtype=torch.float64).pin_memory(),
             torch.empty((wb.natoms, 3), dtype=torch.float64).pin_memory()) for _ in range(2)]
    box = np.ascontiguousarray(wb.box)
    for step in range(4):
        hx, hf = bufs[step // 2]
        x = wb.coords + rng.normal(0.0, 0.003, wb.coords.shape)
        hx.copy_(torch.from_numpy(x))
        e = sysm.evaluate_host(hx, box, hf)
        dev = sysm.evaluate(t(x, torch.float32), t(wb.box, torch.float32))
        assert e == dev["energy"].item()
        assert np.array_equal(hf.numpy().astype(np.float32), dev["forces"].cpu().numpy())


def test_host_entry_point_page_locked_buffers_large():
    """Above 1 MiB of coordinates (15,000 waters) the one-graph path copies inside the graph;
    results equal the device path."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import serving_water_box

    wb = serving_water_box(15000, seed=3)
    assert 3 * wb.natoms * 8 > 1 << 20
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    hx = torch.from_numpy(np.ascontiguousarray(wb.coords, dtype=np.float64)).pin_memory()
    hf = torch.empty((wb.natoms, 3), dtype=torch.float64).pin_memory()
    for step in range(2):
        if step:
            hx.add_(0.001)
        e = sysm.evaluate_host(hx, np.ascontiguousarray(wb.box), hf)
        dev = sysm.evaluate(hx.to("cuda", torch.float32), t(wb.box, torch.float32))
        assert e == dev["energy"].item()
        assert np.array_equal(hf.numpy().astype(np.float32), dev["forces"].cpu().numpy())


def test_cuda_graph_replay_matches_eager(ref3000):
    from torchff_b200.system import FixedChargeSystem

    wb, _ = ref3000
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    x, b = t(wb.coords, torch.float32), t(wb.box, torch.float32)
    e = torch.empty(1, dtype=torch.float64, device="cuda")
    f = torch.empty_like(x)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        sysm.evaluate_into(x, b, e, f)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        sysm.evaluate_into(x, b, e, f)
    x.add_(0.001)
    graph.replay()
    torch.cuda.synchronize()
    eager = sysm.evaluate(x, b)
    assert torch.equal(e, eager["energy"].reshape(1)) and torch.equal(f, eager["forces"])


def test_module_autograd_and_charge_gradient(ref216):
    from torchff_b200.system import FixedChargeNonbonded, FixedChargeSystem

    wb, ref = ref216
    sysm = FixedChargeSystem.from_water_box(wb, dtype=torch.float64)
    model = FixedChargeNonbonded(sysm)
    x = t(wb.coords, grad=True)
    q = t(wb.charges, grad=True)
    e = model(x, t(wb.box), q)
    e.backward()
    assert rel_max(x.grad, ref["grad_coords"]) < 1e-8
    assert rel_max(q.grad, ref["grad_charges"]) < 1e-8


def test_fused_matches_operator_composition(ref216):
    """The reference composition through torch.ops.torchff gives the same energy."""
    from torchff_b200 import PME, MultipolarInteraction, NeighborList, Vdw

    wb, ref = ref216
    x, b, q = t(wb.coords, grad=True), t(wb.box), t(wb.charges)
    nbl = NeighborList(wb.natoms, exclusions=torch.tensor(wb.nblist_exclusions), algorithm="cell_list").cuda()
    pairs, _ = nbl(x.detach(), b, wb.cutoff, 200000, padding=True)
    e_lj = Vdw("LennardJones", use_customized_ops=True, use_type_pairs=True)(
        x, pairs, b, t(wb.sigma_table), t(wb.epsilon_table), wb.cutoff, atom_types=t(wb.atom_types, torch.int64))
    e_c = MultipolarInteraction(0, wb.cutoff, wb.alpha, 138.935456)(x, b, pairs, q,
                                                                     pairs_excl=t(wb.coulomb_exclusions, torch.int64))
    e_p = PME(wb.alpha, wb.grid, 0, use_customized_ops=True).cuda()(x, b, q) * 138.935456
    e = e_lj + e_c + e_p
    e.backward()
    assert rel(e.item(), ref["total"]) < 1e-10
    assert rel_max(x.grad, ref["grad_coords"]) < 1e-8


def test_large_box_matches_independent_composition():
    """12,000 waters (36,000 atoms): the cell grid is rounded to 16^3 (power-of-two branch).
    Fused FP64 vs the O(N^2) pair list + pair ops + PME op composition, and mixed vs FP64."""
    from torchff_b200 import PME, MultipolarInteraction, NeighborList, Vdw
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import make_water_box

    wb = make_water_box(12000, 4.482 * (4.0 ** (1.0 / 3.0)), 23, cutoff=1.0, grid=72, seed=3)
    s64 = FixedChargeSystem.from_water_box(wb, dtype=torch.float64)
    out = s64.evaluate(t(wb.coords), t(wb.box))
    assert s64.status() == 0
    x, b, q = t(wb.coords, grad=True), t(wb.box), t(wb.charges)
    nbl = NeighborList(wb.natoms, exclusions=torch.tensor(wb.nblist_exclusions), algorithm="nsquared").cuda()
    pairs, npairs = nbl(x.detach(), b, wb.cutoff, 8_000_000, padding=True)
    assert int(npairs.item()) <= 8_000_000
    e = (Vdw("LennardJones", use_customized_ops=True, use_type_pairs=True)(
            x, pairs, b, t(wb.sigma_table), t(wb.epsilon_table), wb.cutoff, atom_types=t(wb.atom_types, torch.int64))
         + MultipolarInteraction(0, wb.cutoff, wb.alpha, 138.935456)(
            x, b, pairs, q, pairs_excl=t(wb.coulomb_exclusions, torch.int64))
         + PME(wb.alpha, wb.grid, 0, use_customized_ops=True).cuda()(x, b, q) * 138.935456)
    e.backward()
    assert rel(out["energy"].item(), e.item()) < 1e-10
    assert rel_max(out["forces"], -x.grad) < 1e-8
    s32 = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    o32 = s32.evaluate(t(wb.coords, torch.float32), t(wb.box, torch.float32))
    assert s32.status() == 0
    assert rel_rms(o32["forces"], out["forces"]) < 1e-5


def test_water100k_against_oracle():
    """The 100,000-water box (300,000 atoms, L = 14.42 nm, rc = 1.0 nm, PME 144^3): FP64
    total energy against the oracle (cell-binned real space + PME) to 1e-12 of the summed
    magnitudes of the real-space and reciprocal terms (each about 2.1e7 kJ/mol; their sum,
    3.1e4, cancels 690-fold, so this is about 7e-10 of the total: FP64 sums over 63 M pairs
    in different orders, here and in the oracle, agree to a few 1e-13 of the terms), FP64
    forces on 256 sampled atoms against the oracle (distances to every atom + PME gathered
    there) to 1e-8 of their largest component; both status words 0 (no cluster list cut at
    this size).

    Mixed precision: its arithmetic against FP64 evaluated at the same (FP32) coordinates,
    force RMS error < 1e-5 and energy within 1e-6 of the summed term magnitudes; and the
    whole error against FP64 at the original coordinates < 2e-5. The second bound is wider
    because rounding the inputs to FP32 moves atoms by up to 4.8e-7 nm in the outer half of
    a 14.42 nm box (FP32 spacing 9.5e-7 nm between 8 and 16), which alone changes the
    FP64 forces by about 1e-5 RMS (at 3000 waters, L = 4.48 nm, the same rounding gives
    4.0e-6 of the mixed path's 4.5e-6)."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_100k

    wb = water_box_100k(0)
    s64 = FixedChargeSystem.from_water_box(wb, dtype=torch.float64)
    o64 = s64.evaluate(t(wb.coords), t(wb.box), terms=True)
    assert s64.status() == 0
    x32, b32 = t(wb.coords, torch.float32), t(wb.box, torch.float32)
    o64r = s64.evaluate(x32.double(), b32.double(), terms=True)
    s32 = FixedChargeSystem.from_water_box(wb, dtype=torch.float32)
    o32 = s32.evaluate(x32, b32)
    assert s32.status() == 0
    f64 = o64["forces"].cpu().numpy()
    assert rel_rms(o32["forces"], o64r["forces"].cpu().numpy()) < 1e-5
    assert rel_rms(o32["forces"], f64) < 2e-5
    scale = float(o64r["terms"].abs().sum())
    assert abs(o32["energy"].item() - o64r["energy"].item()) < 1e-6 * scale

    k = 138.935456
    e_real = O.real_space_cells(wb.coords, wb.box, wb.charges, wb.atom_types, wb.sigma_table, wb.epsilon_table,
                                wb.coulomb_exclusions, wb.cutoff, wb.alpha, k)
    subset = np.random.default_rng(11).choice(wb.natoms, 256, replace=False)
    e_pme, g_pme = O.pme_subset(wb.coords, wb.box, wb.charges, wb.alpha, wb.grid, subset)
    assert abs(o64["energy"].item() - (e_real + k * e_pme)) < 1e-12 * (abs(e_real) + abs(k * e_pme))
    g = O.real_space_grad_subset(wb.coords, wb.box, wb.charges, wb.atom_types, wb.sigma_table, wb.epsilon_table,
                                 wb.coulomb_exclusions, wb.cutoff, wb.alpha, k, subset) + k * g_pme
    assert np.max(np.abs(-f64[subset] - g)) < 1e-8 * np.max(np.abs(g))


def _shift_waters(wb, span, seed):
    """The same box with every water moved by a seeded integer combination of the box
    vectors (each count in [-span, span]): molecules stay whole, coordinates leave the
    primary cell by up to `span` box lengths."""
    import dataclasses

    rng = np.random.default_rng(seed)
    n = np.rint(rng.uniform(-span, span, (wb.n_waters, 3))).astype(np.float64)
    shift = np.repeat(n @ wb.box, 3, axis=0)
    return dataclasses.replace(wb, coords=wb.coords + shift)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_coordinates_outside_the_primary_cell(dtype):
    """Waters moved by up to 3 box vectors (216 waters; PME stencil origins far outside
    [0, K) before wrapping): the same energy and forces as the original box. FP64 against
    the oracle of the original coordinates (energy 1e-10, forces 1e-8 of the largest); mixed
    precision energy within the usual tolerance and forces within 2e-5 RMS (the coordinates'
    FP32 rounding at up to 7.5 nm moves atoms by up to 2.4e-7 nm)."""
    from torchff_b200.system import FixedChargeSystem
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    ws = _shift_waters(wb, 3, 5)
    assert np.abs(ws.coords).max() > 2.5 * wb.box[0, 0]
    ref = O.fixed_charge_energy(wb.coords, wb.box, wb.charges, wb.sigma_table, wb.epsilon_table, wb.atom_types,
                                wb.nblist_exclusions, wb.coulomb_exclusions, wb.cutoff, wb.alpha, wb.grid,
                                138.935456)
    s = FixedChargeSystem.from_water_box(ws, dtype=dtype)
    out = s.evaluate(t(ws.coords, dtype), t(ws.box, dtype))
    assert s.status() == 0
    if dtype == torch.float64:
        assert rel(out["energy"].item(), ref["total"]) < 1e-10
        assert rel_max(out["forces"], -ref["grad_coords"]) < 1e-8
    else:
        assert _mixed_energy_err(out["energy"].item(), ref) < 1e-6
        assert rel_rms(out["forces"], -ref["grad_coords"]) < 2e-5
