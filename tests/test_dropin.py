"""The C++ drop-in layer (include/verb4d_dropin.hpp) keeps the reference's
exact C++ signatures: every routine it replaces is exported under the very
mangled name that the reference's own object file defines, so a driver
compiled against the reference's headers links against it unchanged.
(CPU only: symbols and loading, no device calls.)"""
import os
import subprocess

import pytest

import oracle as O

ROUTINES = {  # reference object file -> routines the drop-in replaces
    "MatrixSolver.o": ["tridag("],
    "Diffusion_1D.o": ["Diffusion_1D("],
    "Diffusion_2D.o": ["Diffusion_2D("],
    "Convection_2D.o": ["Convection_2D("],
    "Convection_1D_ULTIMATE_QUICKEST6.o": ["Convection_1D_ULTIMATE_QUICKEST6("],
}


def defined(path, dynamic=False):
    args = ["nm", "--defined-only"] + (["-D"] if dynamic else []) + [path]
    out = subprocess.run(args, check=True, capture_output=True, text=True).stdout
    syms = set()
    for line in out.splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[1] in ("T", "W"):
            syms.add(parts[2])
    return syms


def demangle(names):
    out = subprocess.run(["c++filt"], input="\n".join(names), check=True, capture_output=True,
                         text=True).stdout.splitlines()
    return dict(zip(names, out))


@pytest.mark.skipif(not os.path.exists(O.DROPIN_SO), reason="drop-in not built (needs the reference tree)")
def test_dropin_exports_the_reference_signatures():
    drop = defined(O.DROPIN_SO, dynamic=True)
    for variant in ("plain", "lu"):
        for obj, prefixes in ROUTINES.items():
            path = os.path.join(os.path.dirname(O.REF_SO), variant, obj)
            ref = defined(path)
            names = demangle(sorted(ref))
            wanted = [m for m, d in names.items() if any(d.startswith(p) for p in prefixes)]
            assert wanted, (variant, obj)
            for m in wanted:
                assert m in drop, (variant, obj, names[m])
