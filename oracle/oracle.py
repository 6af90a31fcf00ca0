"""ctypes front end to the CPU restatement oracle (oracle/pdfxc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. Never used by the product path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpdfxc_oracle.so")

FUNCTIONALS = {"SVWN": 0, "HFS": 1, "HFB": 2, "BLYP": 3, "B88LYP": 3, "B3LYP": 4, "PBE": 5}
GGA = {"HFB", "BLYP", "B88LYP", "B3LYP", "PBE"}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import subprocess
            subprocess.run(["make", "-C", HERE, "-s"], check=True)
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(a, dt):
    return np.ascontiguousarray(a, dtype=dt).ctypes.data_as(ctypes.c_void_p)


def functional(name, ra, rb, gaa, gab, gbb):
    """Vectorised over numpy inputs; returns (n, 6): f, vA, vB, vgAA, vgAB, vgBB."""
    L = lib()
    arr = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in (ra, rb, gaa, gab, gbb)))
    flat = [a.ravel() for a in arr]
    out = np.zeros((len(flat[0]), 6))
    o = np.zeros(6)
    for i in range(len(flat[0])):
        L.pdfxc_oracle_functional(ctypes.c_int(FUNCTIONALS[name]), *(ctypes.c_double(float(f[i])) for f in flat),
                                  o.ctypes.data_as(ctypes.c_void_p))
        out[i] = o
    return out


def _shell_args(sh):
    keep = [np.ascontiguousarray(sh.shell_atom, np.int32), np.ascontiguousarray(sh.shell_l, np.int32),
            np.ascontiguousarray(sh.shell_ao0, np.int32), np.ascontiguousarray(sh.shell_nprim, np.int32),
            np.ascontiguousarray(sh.shell_p0, np.int32), np.ascontiguousarray(sh.prim_exp, np.float64),
            np.ascontiguousarray(sh.prim_coef, np.float64), np.ascontiguousarray(sh.atom_xyz, np.float64)]
    return keep, [k.ctypes.data_as(ctypes.c_void_p) for k in keep]


def aos(sh, xyz):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = len(xyz)
    phi = np.zeros((n, sh.nao))
    dphi = np.zeros((n, sh.nao, 3))
    keep, args = _shell_args(sh)
    lib().pdfxc_oracle_aos(ctypes.c_int(sh.nshell), ctypes.c_int(sh.nao), *args, ctypes.c_long(n),
                           xyz.ctypes.data_as(ctypes.c_void_p), phi.ctypes.data_as(ctypes.c_void_p),
                           dphi.ctypes.data_as(ctypes.c_void_p))
    return phi, dphi


def xc(name, sh, xyzw, PA, rho_cut=1e-16, threads=0):
    """Returns dict(exc, nelec_alpha, vxc, rho)."""
    xyzw = np.ascontiguousarray(xyzw, dtype=np.float64).reshape(-1, 4)
    PA = np.ascontiguousarray(PA, dtype=np.float64)
    n = len(xyzw)
    gga = name in GGA
    vxc = np.zeros((sh.nao, sh.nao))
    rho = np.zeros((n, 4 if gga else 1))
    exc = ctypes.c_double()
    nel = ctypes.c_double()
    keep, args = _shell_args(sh)
    lib().pdfxc_oracle_xc(ctypes.c_int(FUNCTIONALS[name]), ctypes.c_int(sh.nshell), ctypes.c_int(sh.nao), *args,
                          ctypes.c_long(n), xyzw.ctypes.data_as(ctypes.c_void_p), PA.ctypes.data_as(ctypes.c_void_p),
                          ctypes.c_double(rho_cut), ctypes.byref(exc), ctypes.byref(nel),
                          vxc.ctypes.data_as(ctypes.c_void_p), rho.ctypes.data_as(ctypes.c_void_p),
                          ctypes.c_int(threads))
    return {"exc": exc.value, "nelec_alpha": nel.value, "vxc": vxc, "rho": rho}


def becke(atom_xyz, brad, xyz, owner, size_adjust=True, ghost=None):
    """Becke partition factor of each point for its owner atom; ghost (natom bools, optional):
    dummy atoms, left out as partners."""
    g = None if ghost is None else np.ascontiguousarray(ghost, dtype=np.int32)
    atom_xyz = np.ascontiguousarray(atom_xyz, dtype=np.float64)
    brad = np.ascontiguousarray(brad, dtype=np.float64)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    fac = np.zeros(len(xyz))
    lib().pdfxc_oracle_becke(ctypes.c_int(len(atom_xyz)), atom_xyz.ctypes.data_as(ctypes.c_void_p),
                             brad.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(int(size_adjust)),
                             ctypes.c_long(len(xyz)), xyz.ctypes.data_as(ctypes.c_void_p),
                             owner.ctypes.data_as(ctypes.c_void_p),
                             None if g is None else g.ctypes.data_as(ctypes.c_void_p),
                             fac.ctypes.data_as(ctypes.c_void_p))
    return fac


COMPONENTS = {"Slater": 0, "VWN5": 1, "VWN3": 2, "Becke88": 3, "Becke88_ExceptLDA": 4, "LYP": 5}


def component(name, ra, rb, gaa, gab, gbb):
    """One functional term (the reference's per-class objects); returns 6 values."""
    o = np.zeros(6)
    lib().pdfxc_oracle_component(ctypes.c_int(COMPONENTS[name]), ctypes.c_double(ra), ctypes.c_double(rb),
                                 ctypes.c_double(gaa), ctypes.c_double(gab), ctypes.c_double(gbb),
                                 o.ctypes.data_as(ctypes.c_void_p))
    return o


def aos_d2(sh, xyz):
    """AO values, first and second derivatives: (npts, 10, nao) in the order
    phi, x, y, z, xx, xy, xz, yy, yz, zz."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((len(xyz), 10, sh.nao))
    keep, args = _shell_args(sh)
    lib().pdfxc_oracle_aos_d2(ctypes.c_int(sh.nshell), ctypes.c_int(sh.nao), *args, ctypes.c_long(len(xyz)),
                              xyz.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    return out


def xc_grad(name, sh, xyzw, owner, PA, rho_cut=1e-16, threads=0):
    """AO-centre term of the XC nuclear gradient (closed shell, doubled as the
    reference's energyGradient does). Returns dict(grad (natom, 3), exc, f (npts,))."""
    xyzw = np.ascontiguousarray(xyzw, dtype=np.float64).reshape(-1, 4)
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    PA = np.ascontiguousarray(PA, dtype=np.float64)
    natom = len(sh.atom_xyz)
    grad = np.zeros((natom, 3))
    f = np.zeros(len(xyzw))
    exc = ctypes.c_double()
    keep, args = _shell_args(sh)
    lib().pdfxc_oracle_xc_grad(ctypes.c_int(FUNCTIONALS[name]), ctypes.c_int(sh.nshell), ctypes.c_int(sh.nao), *args,
                               ctypes.c_int(natom), ctypes.c_long(len(xyzw)), xyzw.ctypes.data_as(ctypes.c_void_p),
                               owner.ctypes.data_as(ctypes.c_void_p), PA.ctypes.data_as(ctypes.c_void_p),
                               ctypes.c_double(rho_cut), grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(exc),
                               f.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(threads))
    return {"grad": grad, "exc": exc.value, "f": f}


def becke_grad(atom_xyz, brad, xyz, owner, coef, size_adjust=True):
    """Grid-weight term of the XC gradient: sum_g coef_g d omega_{A_g}(r_g) / dR, with
    every point moving with its owner atom. coef = w_single * f."""
    atom_xyz = np.ascontiguousarray(atom_xyz, dtype=np.float64)
    brad = np.ascontiguousarray(brad, dtype=np.float64)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    coef = np.ascontiguousarray(coef, dtype=np.float64)
    grad = np.zeros((len(atom_xyz), 3))
    lib().pdfxc_oracle_becke_grad(ctypes.c_int(len(atom_xyz)), atom_xyz.ctypes.data_as(ctypes.c_void_p),
                                  brad.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(int(size_adjust)),
                                  ctypes.c_long(len(xyz)), xyz.ctypes.data_as(ctypes.c_void_p),
                                  owner.ctypes.data_as(ctypes.c_void_p), coef.ctypes.data_as(ctypes.c_void_p),
                                  grad.ctypes.data_as(ctypes.c_void_p))
    return grad


def xc_uks(name, sh, xyzw, PA, PB, rho_cut=1e-16, threads=0):
    """Open-shell quadrature. Returns dict(exc, nelec_alpha, nelec_beta, vxc_a, vxc_b, rho)."""
    xyzw = np.ascontiguousarray(xyzw, dtype=np.float64).reshape(-1, 4)
    PA = np.ascontiguousarray(PA, dtype=np.float64)
    PB = np.ascontiguousarray(PB, dtype=np.float64)
    n = len(xyzw)
    gga = name in GGA
    va, vb = np.zeros((sh.nao, sh.nao)), np.zeros((sh.nao, sh.nao))
    rho = np.zeros((n, 8 if gga else 2))
    exc, na, nb = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    keep, args = _shell_args(sh)
    lib().pdfxc_oracle_xc_uks(ctypes.c_int(FUNCTIONALS[name]), ctypes.c_int(sh.nshell), ctypes.c_int(sh.nao), *args,
                              ctypes.c_long(n), xyzw.ctypes.data_as(ctypes.c_void_p),
                              PA.ctypes.data_as(ctypes.c_void_p), PB.ctypes.data_as(ctypes.c_void_p),
                              ctypes.c_double(rho_cut), ctypes.byref(exc), ctypes.byref(na), ctypes.byref(nb),
                              va.ctypes.data_as(ctypes.c_void_p), vb.ctypes.data_as(ctypes.c_void_p),
                              rho.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(threads))
    return {"exc": exc.value, "nelec_alpha": na.value, "nelec_beta": nb.value, "vxc_a": va, "vxc_b": vb, "rho": rho}


def ss(atom_xyz, xyz, owner):
    """Stratmann-Scuseria partition factor of each point for its owner atom."""
    atom_xyz = np.ascontiguousarray(atom_xyz, dtype=np.float64)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    fac = np.zeros(len(xyz))
    lib().pdfxc_oracle_ss(ctypes.c_int(len(atom_xyz)), atom_xyz.ctypes.data_as(ctypes.c_void_p),
                          ctypes.c_long(len(xyz)), xyz.ctypes.data_as(ctypes.c_void_p),
                          owner.ctypes.data_as(ctypes.c_void_p), fac.ctypes.data_as(ctypes.c_void_p))
    return fac
