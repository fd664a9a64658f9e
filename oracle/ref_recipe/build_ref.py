"""Recipe: compile self-contained pieces of the reference for the host.

Test infrastructure only.  It reads the reference checkout (``FSD_REFERENCE_DIR``,
else a sibling directory ``reference`` next to this repository), extracts the named
per-thread device functions and two host set-up blocks verbatim into
``oracle/_ref/`` (git-ignored), and compiles them together with
``ref_harness.cpp`` and the reference's standalone ``rcm.cpp`` into
``oracle/_ref/libfsdref.so``.  Nothing extracted here is ever committed, and the
product library never links it.

The reference as a whole cannot be built here (HOOMD-blue, CUSP and LAPACKE are
absent and it uses APIs removed in CUDA 12); the pieces chosen below need only
the CUDA builtins and HOOMD box operations supplied by ``hoomd_shim.h``.

Usage:  python oracle/ref_recipe/build_ref.py
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
REF = Path(os.environ.get("FSD_REFERENCE_DIR", str(HERE.parents[2] / "reference"))) / "source"

# (file, function name) for every device function compiled for the host.
KERNELS = [
    ("Helper_Mobility.cu", "Mobility_SetGridk_kernel"),
    ("Helper_Mobility.cu", "Mobility_TS2C_kernel"),
    ("Helper_Mobility.cu", "Mobility_D2WE_kernel"),
    ("Mobility.cu", "Mobility_WaveSpace_Green_kernel"),
    ("Mobility.cu", "Mobility_RealSpace_kernel"),
    ("Lubrication.cu", "Lubrication_RFU_kernel"),
    ("Lubrication.cu", "Lubrication_RFE_kernel"),
    ("Lubrication.cu", "Lubrication_RSU_kernel"),
    ("Lubrication.cu", "Lubrication_RSE_kernel"),
    ("Precondition.cu", "Precondition_GetPrunedNneigh_kernel"),
    ("Precondition.cu", "Precondition_GetPrunedNlist_kernel"),
    ("Precondition.cu", "Precondition_NEPP_kernel"),
    ("Precondition.cu", "Precondition_RFU_kernel"),
    ("Helper_Precondition.cu", "Precondition_AddIdentity_kernel"),
    ("Helper_Stokes.cu", "Stokes_SetForce_manually_kernel"),
    ("Helper_Integrator.cu", "Integrator_AddStrainRate_kernel"),
    ("Integrator.cu", "Integrator_ExplicitEuler_kernel"),
    ("Integrator.cu", "Integrator_ExplicitEuler_Shear_kernel"),
    ("Brownian_FarField.cu", "Brownian_FarField_RNG_Grid1of2_kernel"),
    ("Brownian_FarField.cu", "Brownian_FarField_RNG_Grid2of2_kernel"),
]

# Host blocks of Stokes::setParams, delimited by their first and last lines.
STOKES_BLOCKS = {
    "setparams_grid.inc": ("m_ewald_cut = sqrtf( - logf( m_error ) ) / m_xi;", "m_eta = (2.0*w/m_gaussm)"),
    "setparams_ewald.inc": ("m_ewald_dr = 0.001;", "} // kk loop over distances"),
}


def extract_function(text: str, name: str) -> str:
    m = re.search(r"^[^\n]*__global__\s+void\s+" + re.escape(name) + r"\s*\(", text, re.M)
    if not m:
        raise SystemExit(f"function {name} not found")
    start = m.start()
    i = text.index("{", m.end())
    depth = 0
    j = i
    while True:
        c = text[j]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                break
        j += 1
    body = text[start : j + 1]
    return body.replace('extern "C"', "")


def extract_block(text: str, first: str, last: str) -> str:
    lines = text.splitlines()
    i0 = next(i for i, l in enumerate(lines) if first in l)
    i1 = next(i for i, l in enumerate(lines) if i > i0 and last in l)
    return "\n".join(lines[i0 : i1 + 1]) + "\n"


def main() -> int:
    if not REF.is_dir():
        print(f"reference checkout not found at {REF}; nothing built", file=sys.stderr)
        return 1
    OUT.mkdir(parents=True, exist_ok=True)
    cache: dict[str, str] = {}
    parts = []
    for fname, fn in KERNELS:
        if fname not in cache:
            cache[fname] = (REF / fname).read_text(errors="replace")
        parts.append(f"// ---- {fname}: {fn}\n" + extract_function(cache[fname], fn) + "\n")
    (OUT / "extracted_kernels.inc").write_text("".join(parts))
    stokes = (REF / "Stokes.cc").read_text(errors="replace")
    for out, (a, b) in STOKES_BLOCKS.items():
        (OUT / out).write_text(extract_block(stokes, a, b))
    cmd = [
        "g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-w",
        f"-I{OUT}", f"-I{HERE}", f"-I{REF}",
        str(HERE / "ref_harness.cpp"), str(REF / "rcm.cpp"),
        "-lquadmath", "-o", str(OUT / "libfsdref.so"),
    ]
    print(" ".join(cmd))
    subprocess.check_call(cmd)
    print(f"built {OUT / 'libfsdref.so'}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
