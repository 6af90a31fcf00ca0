"""Dump the unit-sphere Lebedev tables used by ProteinDF's grid generator.

The tables are produced by running the reference's own TlLebedevGrid
(src/libpdftl/TlLebedevGrid.cpp) through the oracle harness
(`oracle/_ref/pdfxc_ref lebedev`); the resulting lebedev.npz (orders and, per
order, x y z weight rows) is committed beside this script so that the grid
helper in proteindf_b200.grids needs no reference files at run time.
Build the harness first: `make -C oracle/ref`.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle.refio import REF_BIN, read_records  # noqa: E402


def main():
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "leb.bin")
        subprocess.run([REF_BIN, "lebedev", "-", out], check=True)
        r = read_records(out)
    orders = r["orders"].astype(np.int64)
    arrays = {"orders": orders}
    for n in orders:
        arrays[f"leb_{n}"] = r[f"leb_{n}"].reshape(n, 4)
    np.savez_compressed(os.path.join(HERE, "lebedev.npz"), **arrays)


if __name__ == "__main__":
    main()
