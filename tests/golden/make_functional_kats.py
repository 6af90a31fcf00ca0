"""Extract the functional known-answer tests of the reference into JSON.

The reference pins its functionals with point-wise known-answer tests in
src/unit_test/DfFunctional_{Slater,VWN,Becke88,LYP,B3LYP}Test.cpp (gtest).
This script reads those files as text (no code from them is compiled here),
and for every active TEST block records the inputs (dRhoA, dRhoB, dGammaAA,
dGammaAB, dGammaBB), the expected values it checks with EXPECT_NEAR, the
tolerance, and whether the closed-shell overload was called. The output,
functional_kats.json, is the fixture tests/test_oracle_pins.py checks the
oracle's functionals against.

usage: python tests/golden/make_functional_kats.py [/root/reference/src/unit_test]
"""
import json
import os
import re
import sys

FILES = {
    "Slater": "DfFunctional_SlaterTest.cpp",
    "VWN5": "DfFunctional_VWNTest.cpp",
    "Becke88": "DfFunctional_Becke88Test.cpp",
    "LYP": "DfFunctional_LYPTest.cpp",
    "B3LYP": "DfFunctional_B3LYPTest.cpp",
}
INPUTS = ["dRhoA", "dRhoB", "dGammaAA", "dGammaAB", "dGammaBB"]
OUTPUTS = {"zk": "f", "vRhoA": "vA", "vRhoB": "vB", "vGammaAA": "vgAA", "vGammaAB": "vgAB", "vGammaBB": "vgBB"}


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return "\n".join(line.split("//", 1)[0] for line in text.splitlines())


def blocks(text):
    for m in re.finditer(r"TEST\s*\(\s*(\w+)\s*,\s*(\w+)\s*\)\s*\{", text):
        depth, i = 1, m.end()
        while depth and i < len(text):
            depth += {"{": 1, "}": -1}.get(text[i], 0)
            i += 1
        yield m.group(2), text[m.end():i - 1]


def main():
    ref = os.environ.get("PDFXC_REFERENCE", "/root/reference")
    src = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ref, "src", "unit_test")
    cases = []
    for comp, fname in FILES.items():
        text = strip_comments(open(os.path.join(src, fname)).read())
        eps_m = re.search(r"const double EPS\s*=\s*([-+0-9.eE]+)", text)
        eps = float(eps_m.group(1))
        for name, body in blocks(text):
            vals = {k: float(v) for k, v in re.findall(r"const double (\w+)\s*=\s*([-+0-9.eE]+)\s*;", body)}
            checked = re.findall(r"EXPECT_NEAR\(\s*(\w+)\s*,", body)
            rks = "dRhoB" not in vals
            ra = vals["dRhoA"]
            inp = [ra, vals.get("dRhoB", ra)]
            gaa = vals.get("dGammaAA", 0.0)
            inp += [gaa, vals.get("dGammaAB", gaa), vals.get("dGammaBB", gaa)]
            expect = {OUTPUTS[c]: vals[c] for c in checked if c in OUTPUTS}
            if not expect:
                continue
            cases.append({"component": comp, "test": name, "closed_shell": rks, "inputs": inp,
                          "expected": expect, "tol": eps,
                          "source": f"src/unit_test/{fname}"})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "functional_kats.json")
    with open(out, "w") as f:
        json.dump(cases, f, indent=1)
    print(len(cases), "cases")


if __name__ == "__main__":
    main()
