"""torch.autograd wrapper of the XC energy Exc(P_A, R), for gradient checks.

Forward: the closed-shell FP64 build on the device (pdfxc_build_vxc) at the nuclear
coordinates R, on a grid that moves with the atoms: every point keeps its offset from
its owner atom and its single-centre weight, and the Becke partition weights are
recomputed at R (pdfxc_becke_weights). Backward: the hand-written adjoint kernel
(pdfxc_xc_backward), which recomputes the AO values per block and returns
dL/dP_A = 2 dL/dP and dL/dR (AO-centre term with the moving grid, plus the derivative
of the Becke partition), each scaled by the incoming dL/dExc.

Only the gradient tests use this module; the product path is the C ABI.
"""
import numpy as np
import torch

from . import basis as _basis


class MovingGridSystem:
    """A molecule, its basis and an atom-centred grid whose points move with their atoms."""

    def __init__(self, engine, symbols, xyz, basis_set, points, w_single, owner, becke_radius, functional):
        self.eng = engine
        self.symbols = list(symbols)
        self.basis_set = basis_set
        self.owner = np.ascontiguousarray(owner, dtype=np.int32)
        self.offsets = np.asarray(points) - np.asarray(xyz)[self.owner]
        self.w_single = np.ascontiguousarray(w_single, dtype=np.float64)
        self.brad = np.ascontiguousarray(becke_radius, dtype=np.float64)
        self.functional = functional

    def place(self, xyz):
        """Make R = xyz the engine's geometry: system, moved points, Becke weights."""
        xyz = np.asarray(xyz, dtype=np.float64)
        self.eng.set_system(_basis.ShellTable(self.symbols, xyz, self.basis_set))
        pts = xyz[self.owner] + self.offsets
        w = self.eng.becke_weights(pts, self.owner, self.w_single, self.brad)
        self.eng.set_grid(np.c_[pts, w], self.owner)

    def energy(self, PA, xyz):
        self.place(xyz)
        return self.eng.build_vxc(self.functional, PA)[0]


class XcEnergy(torch.autograd.Function):
    """Exc = XcEnergy.apply(PA, R, system): PA (n, n) and R (natom, 3) float64 CPU tensors."""

    @staticmethod
    def forward(ctx, PA, R, system):
        PA_np = PA.detach().cpu().numpy().astype(np.float64)
        R_np = R.detach().cpu().numpy().astype(np.float64)
        exc = system.energy(PA_np, R_np)
        ctx.system = system
        ctx.save_for_backward(PA, R)
        return torch.tensor(exc, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        PA, R = ctx.saved_tensors
        system = ctx.system
        system.place(R.detach().cpu().numpy().astype(np.float64))
        dP, go, gw, _ = system.eng.xc_backward(system.functional, PA.detach().cpu().numpy(), dexc=float(g),
                                               w_single=system.w_single, becke_radius=system.brad)
        # dL/dP_A = 2 dL/dP (P = 2 P_A); every element of P_A taken as independent
        return torch.from_numpy(2.0 * dP), torch.from_numpy(go + gw), None
