"""Neighbour-list parity: pair SETS equal to the oracle's (bit-exact), both algorithms, FP32 and FP64."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_util import canon, t
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALGOS = ["nsquared", "cell_list"]
DTYPES = [torch.float64, torch.float32]


def _op(algorithm):
    return getattr(torch.ops.torchff, f"build_neighbor_list_{algorithm}")


def _oracle_pairs(coords, box, cutoff, excl, n, include_self, dtype):
    x = np.asarray(coords, np.float64)
    if dtype == torch.float32:  # the FP32 path decides boundary pairs in FP64 on the FP32 inputs
        x = x.astype(np.float32).astype(np.float64)
        box = None if box is None else np.asarray(box).astype(np.float32).astype(np.float64)
    rp, col = O.exclusions_coo_to_csr(excl, n) if excl is not None and len(excl) else (None, None)
    return O.nblist_pairs(x, box, cutoff, rp, col, include_self)


@pytest.mark.parametrize("algorithm", ALGOS)
@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_small_cases(algorithm, dtype):
    import torchff_b200  # noqa: F401
    from torchff_b200.nblist import convert_pairs_coo_to_csr

    g = np.load(os.path.join(GOLDEN, "nblist_small.npz"))
    for c in range(int(g["ncases"])):
        periodic = bool(g[f"c{c}_periodic"])
        if algorithm == "cell_list" and not periodic:
            continue
        x = g[f"c{c}_coords"]
        n = x.shape[0]
        ex = g[f"c{c}_excl"]
        rp = col = None
        if ex.shape[0]:
            rp, col = (a.cuda() for a in convert_pairs_coo_to_csr(torch.tensor(ex), n))
        box = t(g[f"c{c}_box"], dtype) if periodic else None
        inc = bool(g[f"c{c}_include_self"])
        pairs, npairs = _op(algorithm)(t(x, dtype), box, float(g[f"c{c}_cutoff"]), -1, rp, col, inc)
        got = canon(pairs, npairs)
        if dtype == torch.float64:
            want = g[f"c{c}_pairs"]
        else:
            want = O.canonical_pairs(_oracle_pairs(x, g[f"c{c}_box"] if periodic else None,
                                                   float(g[f"c{c}_cutoff"]), ex, n, inc, dtype))
        assert np.array_equal(got, want), f"case {c}: {got.shape} vs {want.shape}"
        # padding: rows past npairs are -1
        assert bool((pairs[int(npairs.item()):] == -1).all())


@pytest.mark.parametrize("algorithm", ALGOS)
@pytest.mark.parametrize("dtype", DTYPES)
def test_water_boxes(algorithm, dtype):
    from torchff_b200.nblist import NeighborList
    from torchff_b200.water import water_box_216, water_box_3000

    for wb in (water_box_216(), water_box_3000()):
        nbl = NeighborList(wb.natoms, exclusions=torch.tensor(wb.nblist_exclusions), algorithm=algorithm).cuda()
        cap = int(wb.natoms * 4 / 3 * 3.1416 * wb.cutoff ** 3 * 100 / 2 * 1.2)
        pairs, npairs = nbl(t(wb.coords, dtype), t(wb.box, dtype), wb.cutoff, cap, padding=True)
        want = _oracle_pairs(wb.coords, wb.box, wb.cutoff, wb.nblist_exclusions, wb.natoms, False, dtype)
        assert int(npairs.item()) == want.shape[0]
        assert np.array_equal(canon(pairs, npairs), O.canonical_pairs(want))


@pytest.mark.parametrize("algorithm", ALGOS)
def test_overflow_reports_count(algorithm):
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    cap = 1000
    pairs, npairs = _op(algorithm)(t(wb.coords), t(wb.box), wb.cutoff, cap, None, None, False)
    want = O.nblist_pairs(wb.coords, wb.box, wb.cutoff)
    assert int(npairs.item()) == want.shape[0] > cap
    got = canon(pairs)
    assert got.shape[0] == cap
    s = set(map(tuple, O.canonical_pairs(want).tolist()))
    assert all(tuple(p) in s for p in got.tolist())


@pytest.mark.parametrize("algorithm", ALGOS)
def test_module_grows_a_short_capacity(algorithm):
    """NeighborList with max_npairs far below the pair count: by default it builds again with
    the exact count and returns the full list (the reference truncates); with
    grow_on_overflow=False it warns and returns the first max_npairs pairs."""
    from torchff_b200.nblist import NeighborList
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    excl = torch.tensor(wb.nblist_exclusions)
    want = O.canonical_pairs(_oracle_pairs(wb.coords, wb.box, wb.cutoff, wb.nblist_exclusions, wb.natoms, False,
                                           torch.float64))
    got = NeighborList(wb.natoms, exclusions=excl, algorithm=algorithm).cuda()(t(wb.coords), t(wb.box), wb.cutoff, 1000)
    assert np.array_equal(canon(got), want)
    short = NeighborList(wb.natoms, exclusions=excl, algorithm=algorithm, grow_on_overflow=False).cuda()
    with pytest.warns(UserWarning, match="truncated"):
        cut = short(t(wb.coords), t(wb.box), wb.cutoff, 1000)
    assert cut.shape[0] == 1000


def test_cell_list_count_equals_nsquared_at_one_million_atoms():
    """The reference's large-system check (tests/test_nblist.py:230-250): 1,000,000 uniformly
    random atoms at 100 atoms/nm^3 (L = 21.54 nm), FP64, rc = 0.8 nm; the cell list finds as
    many pairs as the all-pairs search. Both report the full count when the pair buffer
    overflows, so a small buffer serves."""
    n = 1_000_000
    box_len = (n / 100.0) ** (1.0 / 3.0)
    rng = np.random.default_rng(5)
    x = torch.tensor(rng.uniform(0.0, box_len, (n, 3)), device="cuda")
    box = torch.tensor(np.diag([box_len] * 3), device="cuda")
    counts = [int(_op(a)(x, box, 0.8, 1024, None, None, False)[1].item()) for a in ALGOS]
    assert counts[0] == counts[1] > 100 * n


@pytest.mark.parametrize("algorithm", ALGOS)
def test_out_variant_and_trim(algorithm):
    from torchff_b200 import nblist as nb
    from torchff_b200.water import water_box_216

    wb = water_box_216()
    fn = nb.build_neighbor_list_nsquared if algorithm == "nsquared" else nb.build_neighbor_list_cell_list
    out = torch.empty((200000, 2), dtype=torch.int64, device="cuda")
    pairs, npairs = fn(t(wb.coords), t(wb.box), wb.cutoff, out=out)
    want = O.canonical_pairs(O.nblist_pairs(wb.coords, wb.box, wb.cutoff))
    assert np.array_equal(canon(pairs), want)
    with pytest.raises(RuntimeError):
        fn(t(wb.coords), t(wb.box), wb.cutoff, max_npairs=10)


def test_single_atom_and_tiny_systems():
    for algorithm in ALGOS:
        x = t(np.array([[0.1, 0.2, 0.3]]))
        pairs, npairs = _op(algorithm)(x, t(np.eye(3)), 0.5, -1, None, None, False)
        assert int(npairs.item()) == 0
        pairs, npairs = _op(algorithm)(x, t(np.eye(3)), 0.5, -1, None, None, True)
        assert int(npairs.item()) == 1 and canon(pairs, npairs).tolist() == [[0, 0]]


def test_cell_list_triclinic_box():
    rng = np.random.default_rng(11)
    box = np.array([[3.0, 0.0, 0.0], [0.9, 2.8, 0.0], [-0.6, 0.7, 2.6]])
    frac = rng.random((700, 3))
    x = frac @ box
    for dtype in DTYPES:
        pairs, npairs = _op("cell_list")(t(x, dtype), t(box, dtype), 0.7, -1, None, None, False)
        want = _oracle_pairs(x, box, 0.7, None, 700, False, dtype)
        assert np.array_equal(canon(pairs, npairs), O.canonical_pairs(want))
