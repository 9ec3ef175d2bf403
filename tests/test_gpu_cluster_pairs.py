"""Cluster-pair format (build_cluster_pairs / decode_cluster_pairs and the nonbonded terms over
it): decoded pair SETS equal to the oracle neighbour list (bit-exact, each pair once), and
energies / gradients equal to the oracle's fused Coulomb + LJ over that list."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_util import canon, rel, rel_max, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DTYPES = [torch.float64, torch.float32]
K_COUL = 138.935456


def _oracle_pairs(x, box, cutoff, excl, dtype):
    x = np.asarray(x, np.float64)
    if dtype == torch.float32:  # boundary pairs are decided in FP64 on the FP32 inputs
        x = x.astype(np.float32).astype(np.float64)
        box = np.asarray(box).astype(np.float32).astype(np.float64)
    n = x.shape[0]
    rp, col = O.exclusions_coo_to_csr(excl, n) if excl is not None and len(excl) else (None, None)
    return O.nblist_pairs(x, box, cutoff, rp, col, False)


def _decode(x, box, cutoff, excl):
    from torchff_b200.nblist import build_cluster_pairs, decode_cluster_pairs

    ex = None if excl is None or not len(excl) else torch.tensor(np.asarray(excl).T, device="cuda")
    fmt = build_cluster_pairs(x, box, cutoff, ex)
    pairs, npairs = decode_cluster_pairs(x, box, *fmt, cutoff)
    return fmt, pairs, npairs


def _check_unique(pairs):
    p = pairs.detach().cpu().numpy().astype(np.int64)
    keys = np.maximum(p[:, 0], p[:, 1]) * (1 << 32) + np.minimum(p[:, 0], p[:, 1])
    assert len(np.unique(keys)) == len(keys), "a pair is listed twice"


@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_cases_pair_sets(dtype):
    import torchff_b200  # noqa: F401

    g = np.load(os.path.join(GOLDEN, "nblist_small.npz"))
    for c in range(int(g["ncases"])):
        if not bool(g[f"c{c}_periodic"]):
            continue
        x = g[f"c{c}_coords"]
        ex = g[f"c{c}_excl"]
        rc = float(g[f"c{c}_cutoff"])
        fmt, pairs, npairs = _decode(t(x, dtype), t(g[f"c{c}_box"], dtype), rc, ex)
        _check_unique(pairs)
        got = canon(pairs, npairs)
        if dtype == torch.float64:
            want = g[f"c{c}_pairs"]
            want = want[want[:, 0] != want[:, 1]]  # the format never lists self pairs
        else:
            want = O.canonical_pairs(_oracle_pairs(x, g[f"c{c}_box"], rc, ex, dtype))
        assert np.array_equal(got, want), f"case {c}: {got.shape} vs {want.shape}"


@pytest.mark.parametrize("dtype", DTYPES)
def test_water216_pairs_and_format_invariants(dtype):
    import torchff_b200  # noqa: F401
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    x, box = t(wb.coords, dtype), t(wb.box, dtype)
    fmt, pairs, npairs = _decode(x, box, wb.cutoff, wb.nblist_exclusions)
    sa, tiles, masks, ecl, eat = fmt
    n = wb.coords.shape[0]
    ncl = (n + 31) // 32
    # sorted atoms: a permutation of the atoms, then -1 padding
    s = sa.cpu().numpy()
    assert s.shape == (ncl * 32,) and sorted(s[:n].tolist()) == list(range(n)) and (s[n:] == -1).all()
    # tiles: x <= y, every diagonal tile present, masks of padding atoms all set
    tl = tiles.cpu().numpy()
    assert (tl[0] <= tl[1]).all() and set(range(ncl)) <= {int(a) for a, b in tl.T if a == b}
    assert masks.dtype == torch.uint32 and masks.shape == (tl.shape[1], 32)
    # entries: cluster ids valid, atoms -1 padded only at the end of a row
    e = eat.cpu().numpy()
    assert ((ecl.cpu().numpy() >= 0) & (ecl.cpu().numpy() < ncl)).all()
    for row in e:
        k = int((row >= 0).sum())
        assert (row[:k] >= 0).all() and (row[k:] == -1).all()
    _check_unique(pairs)
    want = O.canonical_pairs(_oracle_pairs(wb.coords, wb.box, wb.cutoff, wb.nblist_exclusions, dtype))
    assert np.array_equal(canon(pairs, npairs), want)


def test_triclinic_pair_set():
    import torchff_b200  # noqa: F401

    rng = np.random.default_rng(11)
    box = np.array([[2.0, 0.0, 0.0], [0.5, 1.9, 0.0], [-0.3, 0.4, 2.1]])
    x = rng.uniform(0, 1, size=(700, 3)) @ box
    excl = rng.integers(0, 700, size=(200, 2))
    excl = excl[excl[:, 0] != excl[:, 1]]
    fmt, pairs, npairs = _decode(t(x), t(box), 0.7, excl)
    _check_unique(pairs)
    assert np.array_equal(canon(pairs, npairs), O.canonical_pairs(_oracle_pairs(x, box, 0.7, excl, torch.float64)))


def test_water3000_fp32_pair_set():
    import torchff_b200  # noqa: F401
    from torchff_b200.water import water_box_3000

    wb = water_box_3000()
    fmt, pairs, npairs = _decode(t(wb.coords, torch.float32), t(wb.box, torch.float32), wb.cutoff,
                                 wb.nblist_exclusions)
    _check_unique(pairs)
    want = O.canonical_pairs(_oracle_pairs(wb.coords, wb.box, wb.cutoff, wb.nblist_exclusions, torch.float32))
    assert np.array_equal(canon(pairs, npairs), want)


def test_capacities_and_padding():
    import torchff_b200  # noqa: F401
    from torchff_b200.nblist import build_cluster_pairs, decode_cluster_pairs
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    x, box = t(wb.coords), t(wb.box)
    ex = torch.tensor(wb.nblist_exclusions.T, device="cuda")
    fmt = build_cluster_pairs(x, box, wb.cutoff, ex)
    m = fmt[3].shape[0]
    padded = build_cluster_pairs(x, box, wb.cutoff, ex, max_num_interacting_clusters=m + 5)
    assert padded[3].shape == (m + 5,) and bool((padded[3][m:] == -1).all()) and bool((padded[4][m:] == -1).all())
    with pytest.raises(RuntimeError, match="interacting entries"):
        build_cluster_pairs(x, box, wb.cutoff, ex, max_num_interacting_clusters=max(1, m // 2))
    pairs, npairs = decode_cluster_pairs(x, box, *fmt, wb.cutoff)
    found = int(npairs.item())
    pp, npp = decode_cluster_pairs(x, box, *fmt, wb.cutoff, max_npairs=found + 7, padding=True)
    assert pp.shape == (found + 7, 2) and bool((pp[found:] == -1).all()) and int(npp.item()) == found
    with pytest.raises(RuntimeError, match="Too many neighbor pairs"):
        decode_cluster_pairs(x, box, *fmt, wb.cutoff, max_npairs=found - 1)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("do_shift", [True, False])
def test_energy_and_gradients_vs_oracle(dtype, do_shift):
    import torchff_b200  # noqa: F401
    from torchff_b200.nblist import build_cluster_pairs
    from torchff_b200.nonbonded import compute_nonbonded_energy_from_cluster_pairs
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    rng = np.random.default_rng(5)
    q = wb.charges * (1.0 + 0.05 * rng.uniform(-1, 1, wb.charges.shape))
    sig = wb.sigma * (1.0 + 0.05 * rng.uniform(-1, 1, wb.sigma.shape))
    eps = wb.epsilon * (1.0 + 0.05 * rng.uniform(-1, 1, wb.epsilon.shape))
    x = t(wb.coords, dtype, grad=True)
    box = t(wb.box, dtype)
    ts, te, tq = t(sig, dtype, True), t(eps, dtype, True), t(q, dtype, True)
    k = torch.tensor(K_COUL, dtype=dtype, device="cuda", requires_grad=True)
    ex = torch.tensor(wb.coulomb_exclusions.T, device="cuda")
    fmt = build_cluster_pairs(x.detach(), box, wb.cutoff, ex)
    e = compute_nonbonded_energy_from_cluster_pairs(x, box, ts, te, tq, k, wb.cutoff, *fmt, do_shift)
    e.backward()
    xo = wb.coords if dtype == torch.float64 else wb.coords.astype(np.float32).astype(np.float64)
    pairs = _oracle_pairs(wb.coords, wb.box, wb.cutoff, wb.coulomb_exclusions, dtype)
    cast = (lambda a: a) if dtype == torch.float64 else (lambda a: np.asarray(a).astype(np.float32).astype(np.float64))
    E, gx, gq, gs, ge = O.nonbonded(xo, pairs, cast(wb.box), cast(sig), cast(eps), cast(q), K_COUL, wb.cutoff, do_shift)
    Ec, _, _ = O.coulomb(xo, pairs, cast(wb.box), cast(q), K_COUL, wb.cutoff, do_shift)
    tol_e, tol_g = (1e-11, 1e-9) if dtype == torch.float64 else (2e-5, 2e-5)
    assert e.shape == (1,)
    assert rel(e.item(), E) < tol_e
    assert rel_max(x.grad, gx) < tol_g
    assert rel_max(tq.grad, gq) < tol_g
    assert rel_max(ts.grad, gs) < tol_g
    assert rel_max(te.grad, ge) < tol_g
    assert rel(k.grad.item(), Ec / K_COUL) < tol_e * 10


def test_energy_matches_atom_pair_op_and_forces_op():
    import torchff_b200  # noqa: F401
    from torchff_b200.nblist import build_cluster_pairs, build_neighbor_list_cell_list, convert_pairs_coo_to_csr
    from torchff_b200.nonbonded import (compute_nonbonded_energy_from_atom_pairs,
                                        compute_nonbonded_energy_from_cluster_pairs,
                                        compute_nonbonded_forces_from_cluster_pairs)
    from torchff_b200.water import water_box_3000

    wb = water_box_3000()
    x = t(wb.coords, grad=True)
    box, s, e, q = t(wb.box), t(wb.sigma), t(wb.epsilon), t(wb.charges)
    exc = torch.tensor(wb.coulomb_exclusions, device="cuda")
    fmt = build_cluster_pairs(x.detach(), box, wb.cutoff, exc.T)
    e1 = compute_nonbonded_energy_from_cluster_pairs(x, box, s, e, q, K_COUL, wb.cutoff, *fmt)
    (g1,) = torch.autograd.grad(e1, x)
    rp, col = convert_pairs_coo_to_csr(exc, x.shape[0])
    pairs, _ = build_neighbor_list_cell_list(x.detach(), box, wb.cutoff, max_npairs=3_000_000, excl_row_ptr=rp,
                                             excl_col_indices=col)
    x2 = x.detach().clone().requires_grad_(True)
    e2 = compute_nonbonded_energy_from_atom_pairs(x2, pairs, box, s, e, q, K_COUL, wb.cutoff, True)
    (g2,) = torch.autograd.grad(e2, x2)
    assert rel(e1.item(), e2.item()) < 1e-12
    assert rel_max(g1, g2) < 1e-10
    f = torch.ones_like(x.detach())
    compute_nonbonded_forces_from_cluster_pairs(x.detach(), box, s, e, q, K_COUL, wb.cutoff, *fmt, f)
    assert rel_max(f - 1.0, -g1) < 1e-12


def test_fp32_results_are_run_to_run_identical():
    import torchff_b200  # noqa: F401
    from torchff_b200.nblist import build_cluster_pairs
    from torchff_b200.nonbonded import compute_nonbonded_energy_from_cluster_pairs
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    x, box = t(wb.coords, torch.float32), t(wb.box, torch.float32)
    s, e, q = (t(a, torch.float32) for a in (wb.sigma, wb.epsilon, wb.charges))
    fmt = build_cluster_pairs(x, box, wb.cutoff, torch.tensor(wb.coulomb_exclusions.T, device="cuda"))
    fmt2 = build_cluster_pairs(x, box, wb.cutoff, torch.tensor(wb.coulomb_exclusions.T, device="cuda"))
    for a, b in zip(fmt, fmt2):
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
    outs = []
    for _ in range(2):
        xx = x.clone().requires_grad_(True)
        en = compute_nonbonded_energy_from_cluster_pairs(xx, box, s, e, q, K_COUL, wb.cutoff, *fmt)
        (g,) = torch.autograd.grad(en, xx)
        outs.append((en.detach(), g))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
