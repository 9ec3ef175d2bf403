"""CPU checks of the C-ABI library and the host-side logic (no kernel is launched)."""
import math
import os
import re

import numpy as np
import pytest
import torch

from conftest import REPO
from oracle import oracle as O


def _declared_symbols():
    src = open(os.path.join(REPO, "include", "tffb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tff_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from torchff_b200 import _lib

    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(_lib.lib, name), name
    assert set(declared) == set(_lib.EXPORTED)


def _header_prototypes():
    """name -> (return class, [argument classes]) for every prototype in the header; classes
    are int / int64 / double / size_t / ptr (pointers, handles and the stream type)."""
    src = open(os.path.join(REPO, "include", "tffb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    src = re.sub(r"^\s*#[^\n]*", "", src, flags=re.M)
    handles = set(re.findall(r"typedef\s+struct\s+\w+\s*\*\s*(\w+)\s*;", src))

    def cls(decl):
        decl = decl.strip()
        if "*" in decl:
            return "ptr"
        words = decl.replace("const ", "").split()
        base = words[0]
        if base in handles:
            return "ptr"
        return {"int": "int", "int64_t": "int64", "double": "double", "size_t": "size_t"}[base]

    out = {}
    for ret, name, params in re.findall(r"(\b[A-Za-z_][\w\s\*]*?)\b(tff_\w+)\s*\(([^;{]*?)\)\s*;", src):
        args = [p for p in (q.strip() for q in params.split(",")) if p and p != "void"]
        out[name] = (cls(ret + " x"), [cls(a) for a in args])
    return out


def test_ctypes_signatures_match_the_header():
    """Every entry point's ctypes binding has the header's arity and argument types, so a
    changed prototype cannot silently shift the arguments of a Python caller."""
    import ctypes as C

    from torchff_b200 import _lib

    def cls(t):
        if t is None:
            return "void"
        if t in (C.c_void_p, C.c_char_p) or (isinstance(t, type) and issubclass(t, C._Pointer)):
            return "ptr"
        return {C.c_int: "int", C.c_int64: "int64", C.c_double: "double", C.c_size_t: "size_t"}[t]

    protos = _header_prototypes()
    assert set(protos) == set(_lib._SIGS)
    for name, (ret, args) in protos.items():
        res, argtypes = _lib._SIGS[name]
        assert cls(res) == ret, name
        assert [cls(a) for a in argtypes] == args, name


def test_example_ctypes_stub_matches_the_header():
    """The ctypes stub a maintainer adds (torchff_b200/capi_example.py) declares the header's
    return and argument types in the header's order, on the built library."""
    import ctypes as C

    from torchff_b200 import capi_example

    kinds = {C.c_int: "int", C.c_int64: "int64", C.c_double: "double", C.c_size_t: "size_t", C.c_void_p: "ptr",
             C.c_char_p: "ptr"}
    protos = _header_prototypes()
    lib = capi_example.load()
    declared = ["tff_pairs_workspace_bytes", "tff_last_error", "tff_nonbonded_atom_pairs"]
    for name in declared:
        fn = getattr(lib, name)
        ret, args = protos[name]
        assert kinds[fn.restype] == ret, name
        assert [kinds[a] for a in fn.argtypes] == args, name


def test_bench_throughput_fields():
    """The pair-throughput / DRAM-bandwidth object of the bench line: pairs x evals/s, and the
    tile kernel's ncu DRAM bytes over its event time (left out when no ncu figure exists)."""
    import importlib.util
    import json

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(REPO, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    f = bench.throughput_fields(1891879, 9646.67, 0.0669, 1035904.0)
    assert f["pairs_per_s"] == round(1891879 * 9646.67)
    assert abs(f["tile_kernel_dram_gbs"] - 1035904.0 / 66.9e-6 / 1e9) < 0.01
    assert "tile_kernel_dram_gbs" not in bench.throughput_fields(10, 1.0, 1.0, None)
    json.dumps(f)


def test_pure_queries_need_no_gpu():
    from torchff_b200 import _lib

    assert _lib.lib.tff_version() >= 10000
    a = _lib.lib.tff_pairs_workspace_bytes(0, 9000, 0)
    b = _lib.lib.tff_pairs_workspace_bytes(1, 9000, 2)
    assert a > 9000 * 6 * 8 and b >= a
    assert _lib.lib.tff_nblist_cell_list_workspace_bytes(0, 9000, 0) > 0


def test_operator_schemas_match_reference():
    import torchff_b200  # noqa: F401

    expected = {
        "build_neighbor_list_nsquared": "(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)",
        "compute_nonbonded_energy_from_atom_pairs": "(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, bool do_shift) -> Tensor",
        "pme_long_range": "(Tensor coords, Tensor box, Tensor q, Tensor? p, Tensor? t, Scalar K, Scalar alpha, Tensor xmoduli, Tensor ymoduli, Tensor zmoduli) -> Tensor",
        "compute_multipolar_energy_from_atom_pairs": "(Tensor coords, Tensor box, Tensor pairs, Tensor? pairs_excl, Tensor q, Tensor? p, Tensor? t, Scalar cutoff, Scalar ewald_alpha, Scalar prefactor) -> Tensor",
    }
    for name, sig in expected.items():
        op = getattr(torch.ops.torchff, name).default
        assert str(op._schema) == f"torchff::{name}{sig}"


def test_csr_conversion_matches_oracle():
    from torchff_b200.nblist import convert_pairs_coo_to_csr

    rng = np.random.default_rng(3)
    pairs = rng.integers(0, 50, size=(80, 2))
    rp, col = convert_pairs_coo_to_csr(torch.tensor(pairs), 50)
    rp0, col0 = O.exclusions_coo_to_csr(pairs, 50)
    assert np.array_equal(rp.numpy(), rp0) and np.array_equal(col.numpy(), col0)


def test_bspline_moduli_match_oracle():
    from torchff_b200 import bsplines

    for K in (10, 20, 21, 48):
        m = bsplines.compute_bspline_moduli_1d(K, dtype=torch.float64).numpy()
        assert np.allclose(m, O.bspline_moduli(K), rtol=0, atol=1e-15)
        mz = bsplines.compute_bspline_moduli_z(K, dtype=torch.float64).numpy()
        assert np.allclose(mz, O.bspline_moduli(K)[: K // 2 + 1], rtol=0, atol=1e-15)


def test_water_box_geometry():
    from torchff_b200.water import water_box_216, water_box_3000

    for wb in (water_box_216(), water_box_3000(seed=1)):
        x = wb.coords.reshape(-1, 3, 3)
        oh1 = np.linalg.norm(x[:, 1] - x[:, 0], axis=1)
        oh2 = np.linalg.norm(x[:, 2] - x[:, 0], axis=1)
        assert np.allclose(oh1, 0.09572) and np.allclose(oh2, 0.09572)
        cosang = np.einsum("ij,ij->i", x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]) / (oh1 * oh2)
        assert np.allclose(np.degrees(np.arccos(cosang)), 104.52)
        assert abs(wb.charges.sum()) < 1e-9
        assert wb.nblist_exclusions.shape == (9 * wb.n_waters, 2)
        assert wb.coulomb_exclusions.shape == (3 * wb.n_waters, 2)
    assert math.isclose(water_box_216().alpha, 2.920290, rel_tol=1e-6)
    assert math.isclose(water_box_3000().alpha, 2.628261, rel_tol=1e-6)


def test_pbc_helper_matches_oracle():
    from torchff_b200.pbc import applyPBC

    rng = np.random.default_rng(5)
    box = np.array([[3.0, 0.0, 0.0], [0.4, 2.5, 0.0], [0.2, -0.3, 2.8]])
    dr = rng.normal(0, 3.0, (100, 3))
    a = applyPBC(torch.tensor(dr), torch.tensor(box)).numpy()
    assert np.allclose(a, O.min_image(dr, box), atol=1e-13)


def test_ops_reject_cpu_tensors():
    import torchff_b200  # noqa: F401

    x = torch.zeros(4, 3, dtype=torch.float64)
    with pytest.raises(Exception):
        torch.ops.torchff.build_neighbor_list_nsquared(x, None, 0.5, -1, None, None, False)


def test_batch_exclusion_table_layout():
    from torchff_b200.serving import exclusion_table

    pairs = np.array([[0, 1], [0, 2], [1, 2], [2, 1], [3, 3], [5, 4]])
    tab = exclusion_table(6, pairs)
    expect = {0: [1, 2], 1: [0, 2], 2: [0, 1], 3: [], 4: [5], 5: [4]}
    for a, partners in expect.items():
        row = tab[a]
        assert list(row[: len(partners)]) == partners and np.all(row[len(partners):] == -1)
    with pytest.raises(ValueError):
        exclusion_table(10, np.array([[0, k] for k in range(1, 10)]))


def test_batch_and_server_argument_checks_need_no_gpu():
    import ctypes as C

    from torchff_b200 import _lib

    d = _lib.BatchDesc(0, 64, 200_000, 2_000_000, 0.9, 2.92, 138.935456, 0, 0.0)
    small = _lib.lib.tff_batch_device_bytes(C.byref(d))
    d.max_atoms = 400_000
    assert _lib.lib.tff_batch_device_bytes(C.byref(d)) > small > 0
    h = C.c_void_p()
    bad = _lib.ServerDesc(0, 0, 16, 1 << 30, 16.0, 0.9, 2.92, 138.935456, 0.0)  # lanes = 0
    assert _lib.lib.tff_server_create(C.byref(bad), C.byref(h)) == 1
    bad = _lib.BatchDesc(0, 64, 200_000, 2_000_000, 0.9, 2.92, 138.935456, 0, 100.0)  # atoms_per_cell
    assert _lib.lib.tff_batch_create(C.byref(bad), C.byref(h)) == 1
