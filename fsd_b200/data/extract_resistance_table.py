"""Extract the tabulated near-field resistance functions into a binary blob.

The reference hard-codes 1000 log-spaced gaps and 22 Jeffrey-Onishi
resistance scalars per gap as literal assignments in
``Stokes_ResistanceTable.cc`` (lines 56-1055 for the distances, 1058 onwards
for the values; minimum gap 1e-4 and log10 step 0.004305 at lines 37-40).
This script parses those literals and writes ``resistance_table.bin``:

    float32 dist[1000]      tabulated centre-to-centre distances
    float32 vals[1000][22]  XA11 XA12 YA11 YA12 YB11 YB12 XC11 XC12 YC11 YC12
                            XG11 XG12 YG11 YG12 YH11 YH12
                            XM11 XM12 YM11 YM12 ZM11 ZM12

Each literal is parsed and rounded to float32, which is what assigning it to a
``Scalar`` array does in the reference.  The blob is committed; this script
only needs re-running if the reference table changes.

Usage:  python fsd_b200/data/extract_resistance_table.py [reference_dir]
"""
from __future__ import annotations

import hashlib
import re
import sys
from pathlib import Path

import numpy as np

N_DIST = 1000
N_FUNC = 22


def main() -> int:
    # default: a sibling checkout named `reference` next to this repository
    default = Path(__file__).resolve().parents[3] / "reference"
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else default) / "source" / "Stokes_ResistanceTable.cc"
    text = ref.read_text(errors="replace")
    dist = np.full(N_DIST, np.nan, np.float32)
    vals = np.full(N_DIST * N_FUNC, np.nan, np.float32)
    for m in re.finditer(r"h_ResTable_(dist|vals)\.data\[(\d+)\]\s*=\s*([-+0-9.eE]+)\s*;", text):
        arr = dist if m.group(1) == "dist" else vals
        arr[int(m.group(2))] = np.float32(float(m.group(3)))
    if np.isnan(dist).any() or np.isnan(vals).any():
        raise SystemExit("table incomplete")
    out = Path(__file__).with_name("resistance_table.bin")
    blob = dist.tobytes() + vals.tobytes()
    out.write_bytes(blob)
    print(f"wrote {out} ({len(blob)} bytes, sha256 {hashlib.sha256(blob).hexdigest()})")
    return 0


if __name__ == "__main__":
    sys.exit(main())
