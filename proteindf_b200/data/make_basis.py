"""Extract basis-set data from ProteinDF's basis library into a JSON table.

Run once in a checkout that has the reference data (default
/root/reference/data/basis2); the JSON it writes is committed beside this
script so that the package needs no reference files at run time.

The basis2 text format (one entry per `O-<name>.<element>` line) is: a line of
shell counts (s, p, d, ...), then for each contracted shell a primitive count
followed by that many `exponent coefficient` lines. The reference's reader is
src/libpdf/Fl_Db_Basis.cpp; coefficients are stored un-normalised and are
normalised by TlOrbitalInfoObject::setCGTO (src/libpdf/TlOrbitalInfoObject.cpp:38-99).
"""
import json
import os
import sys

SHELLS = "spdfg"


def parse_basis2(path, name, elements):
    lines = open(path).read().splitlines()
    out = {}
    for el in elements:
        key = f"O-{name}.{el}"
        try:
            i = lines.index(key)
        except ValueError:
            raise SystemExit(f"{key} not found in {path}")
        counts = [int(x) for x in lines[i + 1].split()]
        i += 2
        shells = []
        for l, cnt in enumerate(counts):
            for _ in range(cnt):
                nprim = int(lines[i].split()[0])
                prims = []
                for k in range(nprim):
                    e, c = (float(x) for x in lines[i + 1 + k].split()[:2])
                    prims.append([e, c])
                shells.append({"shell": SHELLS[l], "prims": prims})
                i += 1 + nprim
        out[el] = shells
    return out


def main():
    ref = os.environ.get("PDFXC_REFERENCE", "/root/reference")
    src = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ref, "data", "basis2")
    here = os.path.dirname(os.path.abspath(__file__))
    data = {"cc-pVDZ": parse_basis2(src, "cc-pVDZ", ["H", "C", "N", "O"])}
    with open(os.path.join(here, "basis_sets.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
