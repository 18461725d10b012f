"""Build the translated reference time step into oracle/_ref/ (test infrastructure).

Reads the reference's own Fortran (3dmhdsub.f, 3dmhdparam.f) from the
read-only reference checkout, translates STEP, FLUXES, BCON, COMMUNICATE,
COMM_MPI and HORIZONTAL_MEAN with oracle/fortran_subset.py, and compiles the
result with oracle/ref_harness.c into oracle/_ref/ref3dmhd.  Nothing it
writes is committed (oracle/_ref/ is git-ignored); the binary travels with
the working tree so the benchmark host can time the reference without the
reference checkout.

    python oracle/make_ref.py [--src DIR] [--if-present]

The checkout's location comes from --src, else the environment variable
MHD3D_REFERENCE_SRC, else the container's read-only mount.  With
--if-present a missing checkout is not an error (the GPU box has none).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from fortran_subset import Translator  # noqa: E402

DEFAULT_SRC = os.environ.get("MHD3D_REFERENCE_SRC", "/root/reference")

UNITS = ["STEP", "FLUXES", "BCON", "COMMUNICATE", "COMM_MPI", "HORIZONTAL_MEAN"]


def build(src: str = DEFAULT_SRC, out_dir: str | None = None, cc: str = "gcc") -> str:
    out_dir = out_dir or os.path.join(HERE, "_ref")
    sub = os.path.join(src, "3dmhdsub.f")
    par = os.path.join(src, "3dmhdparam.f")
    if not (os.path.exists(sub) and os.path.exists(par)):
        raise FileNotFoundError(f"reference sources not found under {src}")
    os.makedirs(out_dir, exist_ok=True)
    tr = Translator(par, overrides=set())
    code = tr.translate(sub, UNITS)
    gen = os.path.join(out_dir, "ref_generated.c")
    with open(gen, "w") as f:
        f.write(code)
    exe = os.path.join(out_dir, "ref3dmhd")
    cmd = [cc, "-O2", "-std=gnu11", "-ffp-contract=off", "-fno-fast-math", "-w",
           "-I", HERE, "-o", exe, gen, os.path.join(HERE, "ref_harness.c"), "-lm", "-lpthread"]
    subprocess.run(cmd, check=True)
    return exe


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--out", default=None)
    ap.add_argument("--if-present", action="store_true",
                    help="exit quietly when the reference checkout is absent")
    a = ap.parse_args()
    if a.if_present and not os.path.isdir(a.src):
        sys.exit(0)
    print(build(a.src, a.out))
