"""Build the reference's CUDA plugins from their sources into oracle/_ref (test infrastructure only).

Each of init.cu, update_sig.cu, compi.cu is compiled unmodified from the reference
tree, with the flags of its compile.m (-use_fast_math -maxrregcount=50 -O3) but for
sm_100a, into its own shared object (they define the same helper symbols):
    oracle/_ref/libref_init.so, libref_update_sig.so, libref_compi.so
The built objects are kept with the repository's other build outputs, so that machines
without the reference sources can still load them; this recipe only runs where the
reference sources exist.  Nothing here is part of the product library.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference tree: DUGMA_REFERENCE, else where this build environment mounts it (the one place
# the path is named); absent on machines that only run the prebuilt objects
REF = os.environ.get("DUGMA_REFERENCE", "/root/reference")


def reference_tree() -> str | None:
    """The reference tree if it is present on this machine, else None."""
    return REF if os.path.isdir(REF) else None
PLUGINS = ("init", "update_sig", "compi")


def build(ref: str = REF) -> list[str]:
    os.makedirs(OUT, exist_ok=True)
    outs = []
    for name in PLUGINS:
        src = os.path.join(ref, f"{name}.cu")
        lib = os.path.join(OUT, f"libref_{name}.so")
        outs.append(lib)
        if os.path.exists(lib) and os.path.getmtime(lib) >= os.path.getmtime(src):
            continue
        cmd = ["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-use_fast_math",
               "-maxrregcount=50", "-O3", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static", "-o", lib, src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"building {name}.cu failed:\n{r.stderr}")
    return outs


if __name__ == "__main__":
    print("\n".join(build(sys.argv[1] if len(sys.argv) > 1 else REF)))
