"""AO table construction: the host-side mirror of ProteinDF's TlOrbitalInfo.

ProteinDF orders AOs atom by atom, and within an atom shell by shell in the
order the basis entry lists them; each shell expands to its components
s; px,py,pz; dxy,dxz,dyz,d(x2-y2),dz2 (basis types 0..8,
src/libpdf/TlOrbitalInfoObject.cpp:181-256). Primitive coefficients are
normalised per primitive for the angular factor x^l y^m z^n with
(l,m,n) = (0,0,0), (1,0,0) and, for every d component, (1,1,0)
(src/libpdf/Fl_Gto.cpp:686-708), then the contraction is normalised
(src/libpdf/Fl_Gto.cpp:560-650), and primitives are sorted by ascending
exponent (src/libpdf/TlOrbitalInfoObject.cpp:38-99).

The device side works per shell: a shell is (atom, L, first AO, nprim,
exponents, normalised coefficients), and the kernels expand the components.
"""
import json
import math
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
SHELL_L = {"s": 0, "p": 1, "d": 2}
# "X" is the reference's dummy atom: atomic number 0, no basis functions, no grid
# (src/libpdf/Fl_Geometry.cpp:326-333, src/libpdf/DfGenerateGrid.cpp:950)
ELEMENT_Z = {"X": 0, "H": 1, "He": 2, "C": 6, "N": 7, "O": 8}


def load_basis(name="cc-pVDZ"):
    """A basis set of the reference's library (data/basis2, dumped to basis_sets.json).
    "cc-pVDZ-noHp" is cc-pVDZ with the hydrogen p shell left out (3s2p1d on C/N/O, 2s on H):
    the shell structure of 6-31G*, which the reference's library does not have."""
    derived = name == "cc-pVDZ-noHp"
    with open(os.path.join(_DATA, "basis_sets.json")) as f:
        b = json.load(f)["cc-pVDZ" if derived else name]
    if derived:
        b = dict(b)
        b["H"] = [sh for sh in b["H"] if sh["shell"] != "p"]
    return b


def _dfact(n):
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def _prim_norm(alpha, lmn):
    L = sum(lmn)
    dd = _dfact(2 * lmn[0] - 1) * _dfact(2 * lmn[1] - 1) * _dfact(2 * lmn[2] - 1)
    return (2.0 ** L) * dd ** -0.5 * (2.0 / math.pi) ** 0.75 * alpha ** ((L + 1.5) / 2.0)


def normalised_contraction(shell, prims):
    """Return (exponents, coefficients) as the reference stores them."""
    lmn = {"s": (0, 0, 0), "p": (1, 0, 0), "d": (1, 1, 0)}[shell]
    L = sum(lmn)
    exps = np.array([p[0] for p in prims], dtype=np.float64)
    cs = np.array([p[1] for p in prims], dtype=np.float64)
    nrm = np.array([_prim_norm(a, lmn) for a in exps])
    dd = _dfact(2 * lmn[0] - 1) * _dfact(2 * lmn[1] - 1) * _dfact(2 * lmn[2] - 1)
    s = 0.0
    for a in range(len(exps)):
        for b in range(len(exps)):
            s += cs[a] * cs[b] * nrm[a] * nrm[b] * (exps[a] + exps[b]) ** -(L + 1.5)
    s *= dd * 2.0 ** -L * math.pi ** 1.5
    cn = math.sqrt(1.0 / s)
    coefs = cs * nrm * cn
    order = np.argsort(exps, kind="stable")
    return exps[order], coefs[order]


class ShellTable:
    """Flattened shell table for a molecule (structure of arrays).

    Attributes (numpy): shell_atom, shell_l, shell_ao0, shell_nprim, shell_p0,
    prim_exp, prim_coef, atom_xyz (bohr), atom_z; nao, nshell, natom.
    """

    def __init__(self, symbols, xyz_bohr, basis):
        self.symbols = list(symbols)
        self.atom_xyz = np.ascontiguousarray(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
        self.atom_z = np.array([ELEMENT_Z[s] for s in self.symbols], dtype=np.int32)
        sa, sl, s0, sn, sp, pe, pc = [], [], [], [], [], [], []
        ao = 0
        for ia, el in enumerate(self.symbols):
            for sh in basis.get(el, []) if el == "X" else basis[el]:
                e, c = normalised_contraction(sh["shell"], sh["prims"])
                L = SHELL_L[sh["shell"]]
                sa.append(ia)
                sl.append(L)
                s0.append(ao)
                sn.append(len(e))
                sp.append(len(pe))
                pe.extend(e)
                pc.extend(c)
                ao += 2 * L + 1
        self.shell_atom = np.array(sa, dtype=np.int32)
        self.shell_l = np.array(sl, dtype=np.int32)
        self.shell_ao0 = np.array(s0, dtype=np.int32)
        self.shell_nprim = np.array(sn, dtype=np.int32)
        self.shell_p0 = np.array(sp, dtype=np.int32)
        self.prim_exp = np.array(pe, dtype=np.float64)
        self.prim_coef = np.array(pc, dtype=np.float64)
        self.nao = ao
        self.nshell = len(sa)
        self.natom = len(self.symbols)

    def ao_atom(self):
        out = np.empty(self.nao, dtype=np.int32)
        for s in range(self.nshell):
            n = 2 * self.shell_l[s] + 1
            out[self.shell_ao0[s]:self.shell_ao0[s] + n] = self.shell_atom[s]
        return out

    def ao_type(self):
        """Reference basis type per AO: 0 s, 1..3 p, 4..8 d."""
        out = np.empty(self.nao, dtype=np.int32)
        for s in range(self.nshell):
            L = self.shell_l[s]
            n = 2 * L + 1
            out[self.shell_ao0[s]:self.shell_ao0[s] + n] = L * L + np.arange(n)
        return out
