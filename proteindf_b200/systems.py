"""Seeded synthetic molecules and density matrices for tests and benchmarks.

No public dataset exists for this path; every input is generated here from a
seed. Coordinates are produced in Angstrom and returned in bohr using the
reference's conversion factor (src/libpdf/Fl_Geometry.h:95, 0.52917721067 A/bohr).

* water_cluster: n O atoms uniform in a cube (rejection sampling for a minimum
  O-O distance), H at 0.96 A with H-O-H 104.5 deg in a random orientation
  (QR of a seeded 3x3 normal draw).
* peptide_chain: a seeded random walk of heavy atoms (bond lengths
  U(1.33, 1.53) A, C:N:O = 30:8:10) with hydrogens (U(1.0, 1.1) A) hung on them
  until the C:N:O:H = 30:8:10:52 mix is reached; a clash test keeps
  non-bonded heavy-heavy pairs >= 2.0 A and every pair >= 1.0 A.
* density_matrix: P = 2 C C^T with C the Q factor of a seeded N(0,1)
  N x nocc matrix; the XC path receives the alpha density P_A = 0.5 P.
"""
import numpy as np

ANG_PER_BOHR = 0.52917721067


def water_cluster(n=8, seed=0, box=9.0, min_oo=2.6):
    rng = np.random.default_rng(seed)
    O = []
    while len(O) < n:
        p = rng.uniform(0.0, box, size=3)
        if all(np.linalg.norm(p - q) >= min_oo for q in O):
            O.append(p)
    th = np.deg2rad(104.5)
    syms, xyz = [], []
    for o in O:
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        h1 = 0.96 * np.array([np.sin(th / 2), 0.0, np.cos(th / 2)])
        h2 = 0.96 * np.array([-np.sin(th / 2), 0.0, np.cos(th / 2)])
        syms += ["O", "H", "H"]
        xyz += [o, o + q @ h1, o + q @ h2]
    return syms, np.array(xyz) / ANG_PER_BOHR


def _unit(rng):
    v = rng.standard_normal(3)
    return v / np.linalg.norm(v)


def peptide_chain(natoms=100, seed=1, max_tries=2000):
    """Heavy-atom random walk plus hydrogens; returns (symbols, xyz_bohr)."""
    rng = np.random.default_rng(seed)
    mix = {"C": 30, "N": 8, "O": 10, "H": 52}
    counts = {e: int(round(natoms * m / 100.0)) for e, m in mix.items()}
    counts["H"] = natoms - counts["C"] - counts["N"] - counts["O"]
    heavy = ["C"] * counts["C"] + ["N"] * counts["N"] + ["O"] * counts["O"]
    rng.shuffle(heavy)
    pos = [np.zeros(3)]
    direction = _unit(rng)
    for i in range(1, len(heavy)):
        for _ in range(max_tries):
            d = direction + 0.9 * _unit(rng)
            d /= np.linalg.norm(d)
            # keep the backbone angle away from folding back on itself
            if i > 1 and np.dot(d, direction) < -0.3:
                continue
            p = pos[-1] + rng.uniform(1.33, 1.53) * d
            if all(np.linalg.norm(p - q) >= 2.0 for q in pos[:-1]):
                pos.append(p)
                direction = d
                break
        else:
            raise RuntimeError("peptide_chain: could not place heavy atom")
    hpos = []
    allpos = list(pos)
    for k in range(counts["H"]):
        for _ in range(max_tries):
            host = pos[rng.integers(len(pos))]
            p = host + rng.uniform(1.0, 1.1) * _unit(rng)
            if all(np.linalg.norm(p - q) >= 1.0 for q in allpos) and \
                    min(np.linalg.norm(p - q) for q in pos) >= 0.99:
                hpos.append(p)
                allpos.append(p)
                break
        else:
            raise RuntimeError("peptide_chain: could not place hydrogen")
    syms = heavy + ["H"] * len(hpos)
    return syms, np.array(pos + hpos) / ANG_PER_BOHR


def density_matrix(nao, nocc, seed=0):
    """Total density P = 2 C C^T (symmetric positive semi-definite)."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((nao, nocc)))
    return 2.0 * q @ q.T


def density_matrix_device(nao, nocc, seed=0, device="cuda"):
    """The same matrix as density_matrix (the same seeded N(0,1) draw), with the QR and the
    product formed on a CUDA device as a torch FP64 tensor: for the ~18,600-AO inputs whose
    host QR takes minutes. Equal to density_matrix up to rounding (P is invariant to the
    signs of Q's columns)."""
    import torch
    rng = np.random.default_rng(seed)
    a = torch.from_numpy(rng.standard_normal((nao, nocc))).to(device)
    q, _ = torch.linalg.qr(a)
    del a
    return 2.0 * (q @ q.T)


def nuclear_charges(symbols):
    z = {"X": 0, "H": 1, "C": 6, "N": 7, "O": 8}
    return [float(z[s]) for s in symbols]
