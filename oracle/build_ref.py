"""Builds the reference's own CUDA operators (FP64 GPU oracle and GPU timing baseline).

Compiles, for sm_100a, the reference's extension sources for the fixed-charge path
straight from a THGLab/torchff-lib checkout (nothing is copied into this repository):

    torchff_nblist     csrc/nblist/{nblist_interface.cpp, nblist_nsquared_cuda.cu, nblist_clist_cuda.cu}
    torchff_nb         csrc/nonbonded/{nonbonded_interface.cpp, nonbonded_atom_pairs_cuda.cu}
    torchff_coulomb    csrc/coulomb/*
    torchff_vdw        csrc/vdw/*
    torchff_multipoles csrc/multipoles/{multipoles_interface.cpp, multipoles.cu, multipoles_field.cu, rotation.cu}
    torchff_pme        csrc/pme/{pme_interface.cpp, pme.cu}

(the module/source lists of the reference's setup.py:36-70), with torch's JIT extension
builder into ``oracle/_ref/<module>/<module>.so``. Those libraries register
``torch.ops.torchff.*`` exactly like libtffb200's shim does, so they are only ever loaded
in a separate process (oracle/ref_gpu.py).

    python oracle/build_ref.py /path/to/torchff-lib
"""
from __future__ import annotations

import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

MODULES = {
    "torchff_nblist": ["nblist/nblist_interface.cpp", "nblist/nblist_nsquared_cuda.cu", "nblist/nblist_clist_cuda.cu"],
    "torchff_nb": ["nonbonded/nonbonded_interface.cpp", "nonbonded/nonbonded_atom_pairs_cuda.cu"],
    "torchff_coulomb": ["coulomb/*"],
    "torchff_vdw": ["vdw/*"],
    "torchff_multipoles": ["multipoles/multipoles_interface.cpp", "multipoles/multipoles.cu",
                           "multipoles/multipoles_field.cu", "multipoles/rotation.cu"],
    "torchff_pme": ["pme/pme_interface.cpp", "pme/pme.cu"],
}


def sources(root: str, pats: list[str]) -> list[str]:
    out = []
    for p in pats:
        for f in sorted(glob.glob(os.path.join(root, "csrc", p))):
            if f.endswith((".cpp", ".cu")):
                out.append(f)
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCHFF_REFERENCE", "")
    if not root or not os.path.isdir(os.path.join(root, "csrc")):
        raise SystemExit("usage: build_ref.py /path/to/torchff-lib")
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils.cpp_extension import load

    for name, pats in MODULES.items():
        bdir = os.path.join(OUT, name)
        os.makedirs(bdir, exist_ok=True)
        load(name=name, sources=sources(root, pats), build_directory=bdir,
             extra_include_paths=[os.path.join(root, "csrc")],
             extra_cflags=["-O3"],
             extra_cuda_cflags=["-O3", "-gencode", "arch=compute_100a,code=sm_100a"],
             is_python_module=False, verbose=False)
        print("built", os.path.join(bdir, name + ".so"), flush=True)


if __name__ == "__main__":
    main()
