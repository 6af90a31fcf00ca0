"""ctypes front end of libpdfxc (the C ABI in include/pdfxc.h).

The library is loaded from proteindf_b200/lib/libpdfxc.so; there is no
fallback: if it is missing or a call fails, a RuntimeError says why.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpdfxc.so")

FUNCTIONALS = {"SVWN": 0, "HFS": 1, "HFB": 2, "BLYP": 3, "B88LYP": 3, "B3LYP": 4, "PBE": 5}
GGA = {"HFB", "BLYP", "B88LYP", "B3LYP", "PBE"}
PRECISION = {"fp64": 0, "mixed": 1}

# Every entry point include/pdfxc.h declares.
EXPORTS = [
    "pdfxc_default_options", "pdfxc_create", "pdfxc_set_system", "pdfxc_set_grid", "pdfxc_becke_weights",
    "pdfxc_build_vxc", "pdfxc_build_vxc_device", "pdfxc_get_rho", "pdfxc_set_rho", "pdfxc_grid_stats",
    "pdfxc_last_profile", "pdfxc_set_profiling", "pdfxc_last_error", "pdfxc_destroy", "pdfxc_build_vxc_noalloc",
    "pdfxc_xc_gradient", "pdfxc_build_vxc_uks", "pdfxc_get_rho_uks", "pdfxc_set_rho_uks", "pdfxc_ss_weights",
    "pdfxc_block_costs", "pdfxc_partition_blocks", "pdfxc_set_block_range", "pdfxc_set_batch",
    "pdfxc_build_vxc_batched", "pdfxc_density", "pdfxc_generate_grid", "pdfxc_get_grid",
    "pdfxc_build_vxc_delta_device", "pdfxc_pack_upper", "pdfxc_unpack_upper", "pdfxc_plan_grid",
    "pdfxc_xc_backward", "pdfxc_selftest_wait", "pdfxc_autotune", "pdfxc_get_tuning",
]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("block_points", ctypes.c_int), ("ao_cutoff", ctypes.c_double),
                ("rho_cutoff", ctypes.c_double), ("workspace_bytes", ctypes.c_size_t), ("split_terms", ctypes.c_int),
                ("group_blocks", ctypes.c_int), ("vxc_stages", ctypes.c_int)]


class Tuning(ctypes.Structure):
    """pdfxc_tuning: one candidate shape of the autotuner and its build time."""
    _fields_ = [("group_blocks", ctypes.c_int), ("vxc_stages", ctypes.c_int), ("block_points", ctypes.c_int),
                ("ms", ctypes.c_float)]


class GridParams(ctypes.Structure):
    """pdfxc_grid_params: device grid generation."""
    _fields_ = [("nrad", ctypes.c_int), ("nang", ctypes.c_int), ("radial", ctypes.c_int), ("mapping", ctypes.c_int),
                ("pruning", ctypes.c_int), ("partition", ctypes.c_int), ("size_adjust", ctypes.c_int),
                ("weight_cutoff", ctypes.c_double), ("atom_radius", ctypes.c_void_p), ("becke_radius", ctypes.c_void_p),
                ("n_orders", ctypes.c_int), ("orders", ctypes.c_void_p), ("unit_grids", ctypes.c_void_p),
                ("orientation", ctypes.c_void_p)]


RADIAL = {"GC": 0, "EM": 1}
MAPPING = {"BECKE": 0, "TA": 1, "KK": 2}
PRUNING = {False: 0, True: 1, "MHL": 1, "SG1": 2}
PARTITION = {"Becke": 0, "SSWeight": 1}


class Mol(ctypes.Structure):
    """pdfxc_mol: one molecule of a batch."""
    _fields_ = [("natom", ctypes.c_int), ("atom_xyz", ctypes.c_void_p), ("atom_z", ctypes.c_void_p),
                ("nshell", ctypes.c_int), ("shell_atom", ctypes.c_void_p), ("shell_l", ctypes.c_void_p),
                ("shell_nprim", ctypes.c_void_p), ("prim_exp", ctypes.c_void_p), ("prim_coef", ctypes.c_void_p),
                ("npts", ctypes.c_int64), ("xyzw", ctypes.c_void_p), ("atom", ctypes.c_void_p)]


class GridPlan(ctypes.Structure):
    """pdfxc_grid_plan: the host plan of a blocked, screened grid."""
    _fields_ = [("nblocks", ctypes.c_int64), ("ngroups", ctypes.c_int64), ("npts_padded", ctypes.c_int64),
                ("max_nb", ctypes.c_int), ("contraction_flops", ctypes.c_double), ("mean_nb", ctypes.c_double),
                ("workspace_bytes", ctypes.c_size_t), ("nchunks", ctypes.c_int)]


class Profile(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_float), ("ao_ms", ctypes.c_float), ("gemm_x_ms", ctypes.c_float),
                ("rho_ms", ctypes.c_float), ("gemm_v_ms", ctypes.c_float), ("finish_ms", ctypes.c_float),
                ("launches", ctypes.c_int64)]


_lib = None
_vp = ctypes.c_void_p


def load_library(path=LIB_PATH):
    """Load libpdfxc.so and declare the C ABI's signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libpdfxc.so not built ({path}); run `python -c 'import __graft_entry__ as g; g.build()'`")
    L = ctypes.CDLL(path)
    i32, i64, f64 = ctypes.c_int, ctypes.c_int64, ctypes.c_double
    L.pdfxc_default_options.argtypes = [ctypes.POINTER(Options)]
    L.pdfxc_create.argtypes = [ctypes.POINTER(_vp), i32, ctypes.POINTER(Options)]
    L.pdfxc_set_system.argtypes = [_vp, i32, _vp, _vp, i32, _vp, _vp, _vp, _vp, _vp]
    L.pdfxc_set_grid.argtypes = [_vp, i64, _vp, _vp]
    L.pdfxc_becke_weights.argtypes = [_vp, i64, _vp, _vp, _vp, _vp, i32, _vp]
    L.pdfxc_build_vxc.argtypes = [_vp, i32, _vp, i32, _vp, _vp, _vp]
    L.pdfxc_build_vxc_device.argtypes = [_vp, i32, _vp, i32, _vp, _vp, _vp]
    L.pdfxc_build_vxc_delta_device.argtypes = [_vp, i32, _vp, i32, i32, _vp, _vp, _vp, _vp]
    L.pdfxc_get_rho.argtypes = [_vp, i32, _vp]
    L.pdfxc_density.argtypes = [_vp, _vp, i64, _vp, _vp]
    L.pdfxc_generate_grid.argtypes = [_vp, ctypes.POINTER(GridParams), _vp]
    L.pdfxc_get_grid.argtypes = [_vp, _vp, _vp]
    L.pdfxc_set_rho.argtypes = [_vp, i32, _vp]
    L.pdfxc_grid_stats.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.pdfxc_last_profile.argtypes = [_vp, _vp]
    L.pdfxc_set_profiling.argtypes = [_vp, i32]
    L.pdfxc_last_error.argtypes = [_vp]
    L.pdfxc_last_error.restype = ctypes.c_char_p
    L.pdfxc_destroy.argtypes = [_vp]
    L.pdfxc_destroy.restype = None
    L.pdfxc_build_vxc_noalloc.argtypes = [i32, i32, i32, _vp, i32, _vp, _vp, _vp, _vp, _vp, i32, i64, _vp, _vp, _vp,
                                          _vp, _vp]
    L.pdfxc_xc_gradient.argtypes = [_vp, i32, _vp, _vp, _vp, i32, _vp, _vp, _vp]
    L.pdfxc_selftest_wait.argtypes = [_vp, f64]
    L.pdfxc_autotune.argtypes = [_vp, i32, _vp, ctypes.POINTER(Tuning), i32, ctypes.POINTER(i32)]
    L.pdfxc_get_tuning.argtypes = [_vp, ctypes.POINTER(Tuning)]
    L.pdfxc_xc_backward.argtypes = [_vp, i32, _vp, f64, _vp, _vp, i32, _vp, _vp, _vp, _vp]
    L.pdfxc_build_vxc_uks.argtypes = [_vp, i32, _vp, _vp, i32, _vp, _vp, _vp, _vp, _vp]
    L.pdfxc_get_rho_uks.argtypes = [_vp, i32, _vp]
    L.pdfxc_ss_weights.argtypes = [_vp, i64, _vp, _vp, _vp, _vp]
    L.pdfxc_block_costs.argtypes = [_vp, _vp]
    L.pdfxc_partition_blocks.argtypes = [i64, _vp, i32, _vp]
    L.pdfxc_set_block_range.argtypes = [_vp, i64, i64]
    L.pdfxc_set_batch.argtypes = [_vp, i32, _vp]
    L.pdfxc_build_vxc_batched.argtypes = [_vp, i32, _vp, i32, _vp, _vp, _vp]
    L.pdfxc_set_rho_uks.argtypes = [_vp, i32, _vp]
    L.pdfxc_plan_grid.argtypes = [ctypes.POINTER(Options), i32, _vp, i32, _vp, _vp, _vp, _vp, _vp, i64, _vp,
                                  ctypes.POINTER(GridPlan)]
    L.pdfxc_pack_upper.argtypes = [_vp, i32, _vp, _vp]
    L.pdfxc_unpack_upper.argtypes = [_vp, i32, _vp, _vp]
    for name in EXPORTS:
        if name not in ("pdfxc_last_error", "pdfxc_destroy", "pdfxc_default_options"):
            getattr(L, name).restype = i32
    L.pdfxc_default_options.restype = None
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(_vp)


def partition_blocks(cost, nparts):
    """Contiguous block ranges of near-equal cost: bounds (nparts + 1,) int64. Host only."""
    L = load_library()
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    bounds = np.zeros(nparts + 1, dtype=np.int64)
    st = L.pdfxc_partition_blocks(len(cost), _ptr(cost), int(nparts), _ptr(bounds))
    if st != 0:
        raise RuntimeError(f"pdfxc_partition_blocks: status {st}")
    return bounds


def make_options(precision="fp64", block_points=128, ao_cutoff=1e-14, rho_cutoff=1e-16, workspace_bytes=0,
                 split_terms=10, group_blocks=0, vxc_stages=0):
    L = load_library()
    opt = Options()
    L.pdfxc_default_options(ctypes.byref(opt))
    opt.precision = PRECISION[precision]
    opt.block_points = block_points
    opt.ao_cutoff = ao_cutoff
    opt.rho_cutoff = rho_cutoff
    opt.workspace_bytes = workspace_bytes
    opt.split_terms = split_terms
    opt.group_blocks = group_blocks
    opt.vxc_stages = vxc_stages
    return opt


def plan_grid(sh, xyzw, **options):
    """The blocking and screening pdfxc_set_grid would do, planned on the host (no device):
    returns a dict of pdfxc_grid_plan's fields, or raises RuntimeError with the status
    (6 = unsupported: an INT8 group beyond its exact accumulation bound)."""
    L = load_library()
    opt = make_options(**options)
    k = [np.ascontiguousarray(a) for a in (
        sh.atom_xyz.astype(np.float64), sh.shell_atom.astype(np.int32), sh.shell_l.astype(np.int32),
        sh.shell_nprim.astype(np.int32), sh.prim_exp.astype(np.float64), sh.prim_coef.astype(np.float64))]
    xyzw = np.ascontiguousarray(xyzw, dtype=np.float64).reshape(-1, 4)
    out = GridPlan()
    st = L.pdfxc_plan_grid(ctypes.byref(opt), sh.natom, _ptr(k[0]), sh.nshell, _ptr(k[1]), _ptr(k[2]), _ptr(k[3]),
                           _ptr(k[4]), _ptr(k[5]), len(xyzw), _ptr(xyzw), ctypes.byref(out))
    if st != 0:
        raise RuntimeError(f"pdfxc_plan_grid: status {st}")
    return {name: getattr(out, name) for name, _ in GridPlan._fields_}


class XcEngine:
    """One libpdfxc context on one GPU.

    >>> eng = XcEngine(precision="fp64")
    >>> eng.set_system(shell_table)
    >>> eng.set_grid(xyzw, atom)
    >>> exc, nel, V = eng.build_vxc("B3LYP", PA)
    """

    def __init__(self, device=0, precision="fp64", block_points=128, ao_cutoff=1e-14, rho_cutoff=1e-16,
                 workspace_bytes=0, split_terms=10, group_blocks=0, vxc_stages=0):
        self.L = load_library()
        opt = make_options(precision, block_points, ao_cutoff, rho_cutoff, workspace_bytes, split_terms, group_blocks,
                           vxc_stages)
        h = _vp()
        st = self.L.pdfxc_create(ctypes.byref(h), device, ctypes.byref(opt))
        if st != 0:
            raise RuntimeError(f"pdfxc_create failed with status {st}")
        self.h = h
        self.device = device
        self.nao = 0
        self.npts = 0

    def _check(self, st, what):
        if st != 0:
            msg = self.L.pdfxc_last_error(self.h)
            raise RuntimeError(f"{what}: status {st}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            self.L.pdfxc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_system(self, sh):
        """sh: proteindf_b200.basis.ShellTable."""
        self._keep = [np.ascontiguousarray(a) for a in (
            sh.atom_xyz.astype(np.float64), sh.atom_z.astype(np.int32), sh.shell_atom.astype(np.int32),
            sh.shell_l.astype(np.int32), sh.shell_nprim.astype(np.int32), sh.prim_exp.astype(np.float64),
            sh.prim_coef.astype(np.float64))]
        k = self._keep
        self._check(self.L.pdfxc_set_system(self.h, sh.natom, _ptr(k[0]), _ptr(k[1]), sh.nshell, _ptr(k[2]),
                                            _ptr(k[3]), _ptr(k[4]), _ptr(k[5]), _ptr(k[6])), "pdfxc_set_system")
        self.nao = sh.nao
        self.natom = sh.natom

    def set_grid(self, xyzw, atom=None):
        """xyzw: (npts, 4) points and weights; atom: owning atom per point (needed by xc_gradient)."""
        xyzw = np.ascontiguousarray(xyzw, dtype=np.float64).reshape(-1, 4)
        atom = None if atom is None else np.ascontiguousarray(atom, dtype=np.int32)
        self._check(self.L.pdfxc_set_grid(self.h, len(xyzw), _ptr(xyzw), None if atom is None else _ptr(atom)),
                    "pdfxc_set_grid")
        self.npts = len(xyzw)

    def generate_grid(self, atom_radius, nrad=75, nang=302, radial="GC", mapping="TA", pruning=True,
                      partition="Becke", becke_radius=None, size_adjust=True, weight_cutoff=1e-16,
                      orientation=None, unit_grids=None):
        """Build the grid on the device (DfGenerateGrid::generateGrid_atom) and make it the
        context's grid. atom_radius: per atom radial scale (Bragg-Slater; the SG-1 radii with
        pruning="SG1"); unit_grids: {order: (n, 4) x y z w} (default: the package's Lebedev
        tables). Returns the number of points."""
        from . import grids
        tabs = grids.lebedev_table() if unit_grids is None else unit_grids
        orders = np.array(sorted(tabs), dtype=np.int32)
        unit = np.ascontiguousarray(np.concatenate([np.asarray(tabs[int(n)], dtype=np.float64) for n in orders]))
        ar = np.ascontiguousarray(atom_radius, dtype=np.float64)
        br = None if becke_radius is None else np.ascontiguousarray(becke_radius, dtype=np.float64)
        O = None if orientation is None else np.ascontiguousarray(orientation, dtype=np.float64).reshape(3, 3)
        prm = GridParams(nrad, nang, RADIAL[radial], MAPPING[mapping], PRUNING[pruning], PARTITION[partition],
                         int(size_adjust), weight_cutoff, _ptr(ar), None if br is None else _ptr(br), len(orders),
                         _ptr(orders), _ptr(unit), None if O is None else _ptr(O))
        n = ctypes.c_int64(0)
        self._check(self.L.pdfxc_generate_grid(self.h, ctypes.byref(prm), ctypes.byref(n)), "pdfxc_generate_grid")
        self.npts = n.value
        return n.value

    def get_grid(self):
        """The context's grid in input order: (xyzw (n, 4), atom (n,))."""
        xyzw = np.zeros((self.npts, 4))
        atom = np.full(self.npts, -1, dtype=np.int32)
        self._check(self.L.pdfxc_get_grid(self.h, _ptr(xyzw), _ptr(atom)), "pdfxc_get_grid")
        return xyzw, atom

    def becke_weights(self, xyz, atom, w_single, becke_radius, size_adjust=True):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        atom = np.ascontiguousarray(atom, dtype=np.int32)
        ws = np.ascontiguousarray(w_single, dtype=np.float64)
        br = np.ascontiguousarray(becke_radius, dtype=np.float64)
        out = np.zeros(len(xyz))
        self._check(self.L.pdfxc_becke_weights(self.h, len(xyz), _ptr(xyz), _ptr(atom), _ptr(ws), _ptr(br),
                                               int(size_adjust), _ptr(out)), "pdfxc_becke_weights")
        return out

    def ss_weights(self, xyz, atom, w_single):
        """Stratmann-Scuseria partition weights: w_single * P_owner / sum_m P_m."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        atom = np.ascontiguousarray(atom, dtype=np.int32)
        ws = np.ascontiguousarray(w_single, dtype=np.float64)
        out = np.zeros(len(xyz))
        self._check(self.L.pdfxc_ss_weights(self.h, len(xyz), _ptr(xyz), _ptr(atom), _ptr(ws), _ptr(out)),
                    "pdfxc_ss_weights")
        return out

    def build_vxc(self, functional, PA, incremental=False, F=None):
        """Host build. Returns (exc, nelec_alpha, F) with F += Vxc (a new zero matrix if F is None)."""
        PA = np.ascontiguousarray(PA, dtype=np.float64)
        if F is None:
            F = np.zeros((self.nao, self.nao))
        assert F.flags.c_contiguous and F.dtype == np.float64
        exc = ctypes.c_double()
        nel = ctypes.c_double()
        self._check(self.L.pdfxc_build_vxc(self.h, FUNCTIONALS[functional], _ptr(PA), int(incremental), _ptr(F),
                                           ctypes.byref(exc), ctypes.byref(nel)), "pdfxc_build_vxc")
        return exc.value, nel.value, F

    def build_vxc_device(self, functional, d_PA_ptr, d_V_ptr, incremental=False):
        """Device build on raw device pointers (e.g. torch tensor .data_ptr()). Returns (exc, nelec_alpha)."""
        exc = ctypes.c_double()
        nel = ctypes.c_double()
        self._check(self.L.pdfxc_build_vxc_device(self.h, FUNCTIONALS[functional], _vp(d_PA_ptr), int(incremental),
                                                  _vp(d_V_ptr), ctypes.byref(exc), ctypes.byref(nel)),
                    "pdfxc_build_vxc_device")
        return exc.value, nel.value

    def build_vxc_delta_device(self, functional, iteration, d_PA_ptr, d_dV_ptr, d_V_ptr=None, incremental=False):
        """Fxc(iteration) - Fxc(iteration - 1) into d_dV (Fxc(1) at iteration 1), kept on the device
        (DfFockMatrix::setXC_DIRECT, src/libpdf/DfFockMatrix.h:711-721); d_V optionally receives
        Fxc(iteration). Returns (exc, nelec_alpha)."""
        exc = ctypes.c_double()
        nel = ctypes.c_double()
        self._check(self.L.pdfxc_build_vxc_delta_device(self.h, FUNCTIONALS[functional], _vp(d_PA_ptr),
                                                        int(incremental), int(iteration), _vp(d_V_ptr or 0),
                                                        _vp(d_dV_ptr), ctypes.byref(exc), ctypes.byref(nel)),
                    "pdfxc_build_vxc_delta_device")
        return exc.value, nel.value

    def xc_gradient(self, functional, PA, w_single=None, becke_radius=None, size_adjust=True):
        """XC nuclear gradient at fixed PA on the current grid (set with owner atoms).
        Returns (grad_orbital (natom, 3), grad_weight (natom, 3) or None, exc). The
        weight term needs the points' single-centre weights (set_grid order) and
        the Becke radii; without them only the AO-centre term is formed."""
        PA = np.ascontiguousarray(PA, dtype=np.float64)
        natom = self.natom
        go = np.zeros((natom, 3))
        gw = None
        args = [None, None, 0, None]
        if w_single is not None:
            ws = np.ascontiguousarray(w_single, dtype=np.float64)
            br = np.ascontiguousarray(becke_radius, dtype=np.float64)
            gw = np.zeros((natom, 3))
            self._wkeep = (ws, br)
            args = [_ptr(ws), _ptr(br), int(size_adjust), _ptr(gw)]
        exc = ctypes.c_double()
        self._check(self.L.pdfxc_xc_gradient(self.h, FUNCTIONALS[functional], _ptr(PA), args[0], args[1], args[2],
                                             _ptr(go), args[3], ctypes.byref(exc)), "pdfxc_xc_gradient")
        return go, gw, exc.value

    def xc_backward(self, functional, PA, dexc=1.0, w_single=None, becke_radius=None, size_adjust=True):
        """The adjoint of Exc(P, R) (pdfxc_xc_backward): returns (dexc_dP (n, n) -- dL/dP for the
        total density P = 2 PA, equal to Vxc when dexc = 1 --, grad_orbital (natom, 3), grad_weight
        (natom, 3) or None, exc), every derivative scaled by dexc."""
        PA = np.ascontiguousarray(PA, dtype=np.float64)
        dP = np.zeros((self.nao, self.nao))
        go = np.zeros((self.natom, 3))
        gw = None
        args = [None, None, 0, None]
        if w_single is not None:
            ws = np.ascontiguousarray(w_single, dtype=np.float64)
            br = np.ascontiguousarray(becke_radius, dtype=np.float64)
            gw = np.zeros((self.natom, 3))
            self._wkeep = (ws, br)
            args = [_ptr(ws), _ptr(br), int(size_adjust), _ptr(gw)]
        exc = ctypes.c_double()
        self._check(self.L.pdfxc_xc_backward(self.h, FUNCTIONALS[functional], _ptr(PA), float(dexc), args[0], args[1],
                                             args[2], _ptr(dP), _ptr(go), args[3], ctypes.byref(exc)),
                    "pdfxc_xc_backward")
        return dP, go, gw, exc.value

    def build_vxc_uks(self, functional, PA, PB, incremental=False, FA=None, FB=None):
        """Open-shell host build. Returns (exc, nelec_alpha, nelec_beta, FA, FB), FA += Vxc_A, FB += Vxc_B."""
        PA = np.ascontiguousarray(PA, dtype=np.float64)
        PB = np.ascontiguousarray(PB, dtype=np.float64)
        FA = np.zeros((self.nao, self.nao)) if FA is None else FA
        FB = np.zeros((self.nao, self.nao)) if FB is None else FB
        assert FA.flags.c_contiguous and FA.dtype == np.float64 and FB.flags.c_contiguous and FB.dtype == np.float64
        exc, na, nb = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.L.pdfxc_build_vxc_uks(self.h, FUNCTIONALS[functional], _ptr(PA), _ptr(PB), int(incremental),
                                               _ptr(FA), _ptr(FB), ctypes.byref(exc), ctypes.byref(na),
                                               ctypes.byref(nb)), "pdfxc_build_vxc_uks")
        return exc.value, na.value, nb.value, FA, FB

    def get_rho_uks(self, gga):
        out = np.zeros((self.npts, 8 if gga else 2))
        self._check(self.L.pdfxc_get_rho_uks(self.h, int(gga), _ptr(out)), "pdfxc_get_rho_uks")
        return out

    def set_rho_uks(self, rho, gga):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        self._check(self.L.pdfxc_set_rho_uks(self.h, int(gga), _ptr(rho)), "pdfxc_set_rho_uks")

    def get_rho(self, gga):
        out = np.zeros((self.npts, 4 if gga else 1))
        self._check(self.L.pdfxc_get_rho(self.h, int(gga), _ptr(out)), "pdfxc_get_rho")
        return out

    def set_rho(self, rho, gga):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        self._check(self.L.pdfxc_set_rho(self.h, int(gga), _ptr(rho)), "pdfxc_set_rho")

    def density(self, P, xyz):
        """rho(r) = phi(r)^T P phi(r) at the points xyz (n, 3), bohr (DfCalcGridX::gridDensity)."""
        P = np.ascontiguousarray(P, dtype=np.float64)
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(len(xyz))
        self._check(self.L.pdfxc_density(self.h, _ptr(P), len(xyz), _ptr(xyz), _ptr(out)), "pdfxc_density")
        return out

    def set_batch(self, mols):
        """mols: list of (ShellTable, xyzw (npts, 4), atom (npts,) or None)."""
        keep, structs = [], (Mol * len(mols))()
        for k, (sh, xyzw, atom) in enumerate(mols):
            arrs = [np.ascontiguousarray(a) for a in (
                sh.atom_xyz.astype(np.float64), sh.atom_z.astype(np.int32), sh.shell_atom.astype(np.int32),
                sh.shell_l.astype(np.int32), sh.shell_nprim.astype(np.int32), sh.prim_exp.astype(np.float64),
                sh.prim_coef.astype(np.float64), np.asarray(xyzw, dtype=np.float64).reshape(-1, 4))]
            at = None if atom is None else np.ascontiguousarray(atom, dtype=np.int32)
            keep.append((arrs, at))
            structs[k] = Mol(sh.natom, arrs[0].ctypes.data, arrs[1].ctypes.data, sh.nshell, arrs[2].ctypes.data,
                             arrs[3].ctypes.data, arrs[4].ctypes.data, arrs[5].ctypes.data, arrs[6].ctypes.data,
                             len(arrs[7]), arrs[7].ctypes.data, None if at is None else at.ctypes.data)
        self._check(self.L.pdfxc_set_batch(self.h, len(mols), ctypes.byref(structs)), "pdfxc_set_batch")
        self._batch_nao = [sh.nao for sh, _, _ in mols]
        self.nao = sum(self._batch_nao)
        self.natom = sum(sh.natom for sh, _, _ in mols)
        self.npts = sum(len(np.asarray(x).reshape(-1, 4)) for _, x, _ in mols)

    def build_vxc_batched(self, functional, PAs, incremental=False, Fs=None):
        """One build of every molecule of the batch. Returns (exc (nmol,), nelec_alpha (nmol,), Fs)."""
        nm = len(self._batch_nao)
        PAs = [np.ascontiguousarray(P, dtype=np.float64) for P in PAs]
        Fs = [np.zeros((n, n)) for n in self._batch_nao] if Fs is None else Fs
        pa = (ctypes.c_void_p * nm)(*[P.ctypes.data for P in PAs])
        fa = (ctypes.c_void_p * nm)(*[F.ctypes.data for F in Fs])
        exc, nel = np.zeros(nm), np.zeros(nm)
        self._check(self.L.pdfxc_build_vxc_batched(self.h, FUNCTIONALS[functional], pa, int(incremental), fa,
                                                   _ptr(exc), _ptr(nel)), "pdfxc_build_vxc_batched")
        return exc, nel, Fs

    def block_costs(self):
        nb = self.grid_stats()["nblocks"]
        out = np.zeros(nb)
        self._check(self.L.pdfxc_block_costs(self.h, _ptr(out)), "pdfxc_block_costs")
        return out

    def set_block_range(self, b_lo, b_hi):
        self._check(self.L.pdfxc_set_block_range(self.h, int(b_lo), int(b_hi)), "pdfxc_set_block_range")

    def grid_stats(self):
        nb, npad = ctypes.c_int64(), ctypes.c_int64()
        fl, mnb = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.pdfxc_grid_stats(self.h, ctypes.byref(nb), ctypes.byref(npad), ctypes.byref(fl),
                                            ctypes.byref(mnb)), "pdfxc_grid_stats")
        return {"nblocks": nb.value, "npts_padded": npad.value, "contraction_flops": fl.value, "mean_nb": mnb.value}

    def autotune(self, functional, d_PA_ptr=None):
        """pdfxc_autotune: time every candidate shape on the current grid, keep the fastest.
        Returns a list of dicts (group_blocks, vxc_stages, block_points, ms), the winner first."""
        out = (Tuning * 16)()
        n = ctypes.c_int(0)
        self._check(self.L.pdfxc_autotune(self.h, FUNCTIONALS[functional], _vp(d_PA_ptr or 0), out, 16,
                                          ctypes.byref(n)), "pdfxc_autotune")
        return [{k: getattr(out[i], k) for k, _ in Tuning._fields_} for i in range(n.value)]

    def tuning(self):
        t = Tuning()
        self._check(self.L.pdfxc_get_tuning(self.h, ctypes.byref(t)), "pdfxc_get_tuning")
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def selftest_wait(self, limit_seconds=1e-3):
        """Run the bounded-wait failure path (pdfxc_selftest_wait); returns (status, message)."""
        st = self.L.pdfxc_selftest_wait(self.h, float(limit_seconds))
        msg = self.L.pdfxc_last_error(self.h)
        return st, (msg.decode() if msg else "")

    def set_profiling(self, enable):
        """Stage-by-stage launches (per-stage times) instead of CUDA graph replay."""
        self._check(self.L.pdfxc_set_profiling(self.h, int(enable)), "pdfxc_set_profiling")

    def last_profile(self):
        p = Profile()
        self._check(self.L.pdfxc_last_profile(self.h, ctypes.byref(p)), "pdfxc_last_profile")
        return {k: getattr(p, k) for k, _ in Profile._fields_}
