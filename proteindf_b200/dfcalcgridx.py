"""Host mirror of ProteinDF's DfCalcGridX interface on top of libpdfxc.

The reference class (src/libpdf/DfCalcGridX.h:72-212) is constructed from
the parameter set (`coordinates`, `basis_set`, `xc-density-threshold`,
`xc-update`, ...), reads the grid matrix written by DfGenerateGrid, and is
called once per SCF iteration through

    double calcXCIntegForFockAndEnergy(const P_A, DfFunctional_{LDA,GGA}*, F_A*)

which accumulates Vxc into F_A and returns Exc (src/libpdf/DfCalcGridX.cpp:2280-2315).
This class keeps those names, argument meanings and side effects: F_A is
accumulated into (+=), the per-point rho columns of the grid matrix are
updated (and, with xc-update = yes, the next call adds rho(dP) to them), and
getWholeDensity returns sum_i w_i rho_A(r_i) (:2502-2537). Functionals are
named as the reference's xc-potential keyword (DfXCFunctional.cpp:70-104).

energyGradient(P_A, functional) mirrors the XC nuclear gradient
(src/libpdf/DfCalcGridX.cpp:1073-1415) on the current grid matrix (its atom
column says which atom each point moves with). The reference integrates it on
its own SG-1 grid; pass that grid's matrix here for the same result. With the
points' single-centre weights and the Becke radii the grid-weight term is
added, which the reference's own version evaluates to zero.

The open-shell overload calcXCIntegForFockAndEnergy(P_A, functional, F_A,
P_B, F_B) mirrors (P_A, P_B, functional, F_A, F_B) of the reference
(:2292-2303, :2317-2328); its grid matrix carries rho_A and rho_B columns.
"""
import numpy as np

from . import basis as _basis
from .xc import FUNCTIONALS, GGA, XcEngine

GM_X, GM_Y, GM_Z, GM_WEIGHT, GM_ATOM_INDEX = 0, 1, 2, 3, 4
GM_RHO_ALPHA = 5


class DfCalcGridX:
    def __init__(self, pdf_param, grid_matrix=None, device=0, precision="fp64"):
        """pdf_param: {"coordinates": [(symbol, (x, y, z) bohr), ...],
        "basis_set": name or {element: shells}, "xc-density-threshold": float,
        "xc-update": "yes"|"no", "xc-potential": name}."""
        self.param = dict(pdf_param)
        atoms = self.param["coordinates"]
        symbols = [a[0] for a in atoms]
        xyz = np.array([a[1] for a in atoms], dtype=np.float64)
        bs = self.param.get("basis_set", "cc-pVDZ")
        bdata = _basis.load_basis(bs) if isinstance(bs, str) else bs
        self.orbital_info = _basis.ShellTable(symbols, xyz, bdata)
        self.num_of_AOs = self.orbital_info.nao
        cut = self.param.get("xc-density-threshold", 1e-16)
        self.is_update_xc = str(self.param.get("xc-update", "yes")).lower() != "no"
        self._engine = XcEngine(device=device, precision=precision, rho_cutoff=float(cut))
        self._engine.set_system(self.orbital_info)
        self._iteration = 0
        self._grid = None
        self._functional_is_gga = None
        self._open_shell = False
        if grid_matrix is not None:
            self.setGridMatrix(grid_matrix)

    # grid matrix (DfObject::getGridMatrix / saveGridMatrix, src/libpdf/DfObject.h:955-972)
    def setGridMatrix(self, grid_matrix):
        g = np.ascontiguousarray(grid_matrix, dtype=np.float64)
        self._grid = g
        self._engine.set_grid(g[:, :4], g[:, GM_ATOM_INDEX].astype(np.int32))
        # rho columns by width (src/libpdf/DfCalcGridX.h:35-54): 6 LDA, 9 GGA closed shell;
        # 7 LDA, 13 GGA open shell
        ncol = g.shape[1]
        if ncol in (6, 9):
            gga = ncol == 9
            self._engine.set_rho(g[:, GM_RHO_ALPHA:ncol], gga)
            self._functional_is_gga, self._open_shell = gga, False
        elif ncol in (7, 13):
            gga = ncol == 13
            self._engine.set_rho_uks(g[:, GM_RHO_ALPHA:ncol], gga)
            self._functional_is_gga, self._open_shell = gga, True

    def getGridMatrix(self):
        """The grid matrix with the current rho (and grad rho) columns."""
        gga = bool(self._functional_is_gga)
        rho = self._engine.get_rho_uks(gga) if self._open_shell else self._engine.get_rho(gga)
        return np.concatenate([self._grid[:, :5], rho], axis=1)

    def calcXCIntegForFockAndEnergy(self, P_A, functional, F_A, P_B=None, F_B=None):
        """Closed shell: F_A += Vxc(P_A); open shell (P_B and F_B given): F_A += Vxc_A,
        F_B += Vxc_B. Returns Exc. With xc-update = yes the call after the first
        treats the densities as differences."""
        name = functional if isinstance(functional, str) else getattr(functional, "name")
        name = name.upper()
        if name not in FUNCTIONALS:
            raise ValueError(f"unknown functional {name}")
        gga = name in GGA
        open_shell = P_B is not None
        if open_shell != (F_B is not None):
            raise ValueError("the open-shell form needs both P_B and F_B")
        incremental = (self.is_update_xc and self._iteration > 0 and self._functional_is_gga == gga
                       and self._open_shell == open_shell)
        if open_shell:
            FA = np.ascontiguousarray(F_A, dtype=np.float64)
            FB = np.ascontiguousarray(F_B, dtype=np.float64)
            exc, na, nb, FA, FB = self._engine.build_vxc_uks(name, P_A, P_B, incremental=incremental, FA=FA, FB=FB)
            if FA is not F_A:
                F_A[...] = FA
            if FB is not F_B:
                F_B[...] = FB
            self._functional_is_gga = gga
            self._open_shell = True
            self._iteration += 1
            self._nelec_alpha, self._nelec_beta = na, nb
            return exc
        F = np.ascontiguousarray(F_A, dtype=np.float64)
        exc, nel, F = self._engine.build_vxc(name, P_A, incremental=incremental, F=F)
        if F is not F_A:
            F_A[...] = F
        self._functional_is_gga = gga
        self._open_shell = False
        self._iteration += 1
        self._nelec_alpha = nel
        return exc

    def energyGradient(self, P_A, functional, w_single=None, becke_radius=None, size_adjust=True):
        """XC nuclear gradient (natom, 3) at fixed P_A: the AO-centre term (the
        reference's result), plus the grid-weight term when w_single is given."""
        name = functional if isinstance(functional, str) else getattr(functional, "name")
        name = name.upper()
        if name not in FUNCTIONALS:
            raise ValueError(f"unknown functional {name}")
        go, gw, exc = self._engine.xc_gradient(name, P_A, w_single=w_single, becke_radius=becke_radius,
                                               size_adjust=size_adjust)
        self._gradient_exc = exc
        return go if gw is None else go + gw

    def getWholeDensity(self):
        """(sum w rho_A, sum w rho_B); the second is None after a closed-shell build."""
        return self._nelec_alpha, (self._nelec_beta if self._open_shell else None)

    def gridDensity(self, P, position):
        """rho(r) = phi(r)^T P phi(r) at one point (DfCalcGridX::gridDensity,
        src/libpdf/DfCalcGridX.cpp:1038-1044). gridDensities takes many points in one call."""
        return float(self.gridDensities(P, np.asarray(position, dtype=np.float64).reshape(1, 3))[0])

    def gridDensities(self, P, positions):
        """rho at every point of positions (n, 3), bohr: the loop of TlDensField::makeDensFld
        (src/tools/TlDensField.cpp:35-53) as one device call."""
        return self._engine.density(P, positions)

    def close(self):
        self._engine.close()
