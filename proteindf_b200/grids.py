"""Atom-centred quadrature grids (host-side producer of the path's input).

Mirrors the single-centre part of ProteinDF's DfGenerateGrid
(src/libpdf/DfGenerateGrid.cpp): per atom and radial shell i = 1..Nr an
abscissa r_i and weight w_i from Gauss-Chebyshev (second kind, with the
Becke / Treutler-Ahlrichs / KK mapping, :1612-1655) or Euler-Maclaurin
(:1597-1610); shells with r_i > 30 are dropped (:1005-1007); the angular
order is pruned as Murray-Handy-Laming with K = 5 and the Bragg-Slater radius,
rounded down to a supported Lebedev order (:1658-1688); points are the unit
Lebedev points scaled by r_i about the atom, weights w_leb * w_i (:1715-1734).
The grid orientation matrix O of the reference (:1739-1809) only rotates the
angular grid; this helper uses the identity orientation, as the reference
oracle harness does, so that both sides see the same points.

The multi-centre (Becke) partition weights are computed on the GPU by
pdfxc_becke_weights; screen_by_weight then drops points whose final weight is
<= 1e-16 as DfGenerateGrid::screeningGridsByWeight0 does (:1979-2004).

The Lebedev tables are the reference's own (dumped once by
proteindf_b200/data/make_lebedev.py).
"""
import math
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

# Bragg-Slater radii as the reference tabulates them (src/libpdftl/TlPrdctbl.cpp),
# used for the radial mapping and the pruning; the Becke size adjustment uses
# 0.35 for hydrogen and the Bragg-Slater radius otherwise
# (src/libpdf/DfGenerateGrid.cpp:1958-1968).
# A dummy atom (atomic number 0) has radius 0 in both tables and no grid of its own.
BRAGG_SLATER = {0: 0.0, 1: 0.25, 6: 0.70, 7: 0.65, 8: 0.60}
BECKE_RADIUS = {0: 0.0, 1: 0.35, 6: 0.70, 7: 0.65, 8: 0.60}
# Radial scales of the SG-1 grid (and of USER grids' gradient grid), as the reference
# sets them for those grid types (src/libpdf/DfGenerateGrid.cpp:409-418).
SG1_RADIUS = {1: 1.0000, 6: 1.2308, 7: 1.0256, 8: 0.8791}

_LEB = None


def lebedev_table():
    global _LEB
    if _LEB is None:
        d = np.load(os.path.join(_DATA, "lebedev.npz"))
        _LEB = {int(n): d[f"leb_{n}"] for n in d["orders"]}
    return _LEB


def radial_gc(R, Nr, i, mapping="TA"):
    Nr1 = Nr + 1.0
    t = i * math.pi / Nr1
    s, c = math.sin(t), math.cos(t)
    ss = s * s
    x = (Nr1 - 2.0 * i) / Nr1 + (2.0 / math.pi) * (1.0 + (2.0 / 3.0) * ss) * c * s
    inv_x1 = 1.0 / (x - 1.0)
    inv_ln2 = 1.0 / math.log(2.0)
    if mapping == "BECKE":
        r = R * (1.0 + x) / (1.0 - x)
        jac = R * ((x + 1.0) * inv_x1 * inv_x1 - inv_x1)
    elif mapping == "TA":
        r = inv_ln2 * math.log(2.0 * (-inv_x1)) * R
        jac = R * inv_ln2 / (1.0 - x)
    elif mapping == "KK":
        r = inv_ln2 * math.log(2.0 * (-inv_x1))
        jac = inv_ln2 / (1.0 - x)
    else:
        raise ValueError(mapping)
    w = (16.0 / (3.0 * Nr1)) * ss * ss * jac * r * r * 4.0 * math.pi
    return r, w


def radial_em(R, Nr, i):
    inv = 1.0 / float(Nr + 1 - i)
    r = R * float(i * i) * inv * inv
    w = 2.0 * R ** 3 * float(Nr + 1) * float(i ** 5) * inv ** 7 * 4.0 * math.pi
    return r, w


def pruned_order(r, max_ang, Z, pruning=True):
    n = max_ang
    if pruning:
        n = min(int((5.0 * r / BRAGG_SLATER[Z]) * max_ang), max_ang)
    orders = sorted(lebedev_table())
    cands = [o for o in orders if o <= n]
    return cands[-1] if cands else orders[0]


def atom_grid(center, Z, nrad=75, nang=302, radial="GC", mapping="TA", pruning=True):
    R = BRAGG_SLATER[Z]
    leb = lebedev_table()
    pts, ws = [], []
    for i in range(1, nrad + 1):
        r, wr = radial_gc(R, nrad, i, mapping) if radial == "GC" else radial_em(R, nrad, i)
        if r > 30.0:
            continue
        n = pruned_order(r, nang, Z, pruning)
        t = leb[n]
        pts.append(t[:, :3] * r + center)
        ws.append(t[:, 3] * wr)
    return np.concatenate(pts), np.concatenate(ws)


def molecular_grid(atom_xyz, atom_z, **kw):
    """Single-centre grid for every atom: (points (n,3), w_single (n,), atom (n,))."""
    P, W, A = [], [], []
    for a, (c, z) in enumerate(zip(np.asarray(atom_xyz), atom_z)):
        if int(z) == 0:  # dummy atom: no grid (DfGenerateGrid::generateGrid_atom, :950)
            continue
        p, w = atom_grid(np.asarray(c, dtype=np.float64), int(z), **kw)
        P.append(p)
        W.append(w)
        A.append(np.full(len(w), a, dtype=np.int32))
    return np.concatenate(P), np.concatenate(W), np.concatenate(A)


def screen_by_weight(points, weights, atom, cutoff=1e-16):
    keep = np.abs(weights) > cutoff
    return points[keep], weights[keep], atom[keep]


# Grid presets named as the reference names them (src/libpdf/DfGenerateGrid.cpp:56-135).
PRESETS = {
    "USER-75x302": dict(nrad=75, nang=302, radial="GC", mapping="TA", pruning=True),
    "ULTRA_FINE": dict(nrad=99, nang=590, radial="EM", mapping="TA", pruning=True),
    "FINE": dict(nrad=75, nang=302, radial="EM", mapping="TA", pruning=True),
}
