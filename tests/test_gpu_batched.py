"""Batched build (pdfxc_set_batch, pdfxc_build_vxc_batched): many independent
molecules in one context -- one launch per stage and one CUDA graph per build
for all of them -- against one context per molecule (FP64 and INT8), with the
molecules placed on top of each other in space, so that screening must keep each
molecule's blocks on its own shells."""
import numpy as np
import pytest

from proteindf_b200 import basis, grids, systems

pytestmark = pytest.mark.gpu


def _mols(n=6, seed=40):
    rng = np.random.default_rng(seed)
    b = basis.load_basis("cc-pVDZ")
    out = []
    for k in range(n):
        syms, xyz = systems.peptide_chain(int(rng.integers(4, 14)), seed=seed + k)
        Z = [int(z) for z in systems.nuclear_charges(syms)]
        pts, ws, own = grids.molecular_grid(xyz, Z, nrad=30, nang=110, radial="GC", mapping="TA", pruning=True)
        sh = basis.ShellTable(syms, xyz, b)
        PA = 0.5 * systems.density_matrix(sh.nao, max(1, sh.nao // 4), seed=seed + 100 + k)
        out.append((sh, np.c_[pts, ws], own, PA))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_one_context_per_molecule(precision):
    from proteindf_b200.xc import XcEngine
    mols = _mols()
    eng = XcEngine(device=0, precision=precision, split_terms=10)
    eng.set_batch([(sh, g, own) for sh, g, own, _ in mols])
    exc, nel, Fs = eng.build_vxc_batched("B3LYP", [P for *_, P in mols])
    # a second SCF-style call replays the captured graph
    exc2, _, Fs2 = eng.build_vxc_batched("B3LYP", [P for *_, P in mols])
    eng.close()
    tol = 1e-12 if precision == "fp64" else 1e-8
    for k, (sh, g, own, PA) in enumerate(mols):
        one = XcEngine(device=0, precision=precision, split_terms=10)
        one.set_system(sh)
        one.set_grid(g, own)
        e, n, V = one.build_vxc("B3LYP", PA)
        one.close()
        assert abs(exc[k] - e) < tol * abs(e) and abs(exc2[k] - e) < tol * abs(e)
        assert abs(nel[k] - n) < 1e-10 * abs(n)
        assert np.abs(Fs[k] - V).max() < tol * max(1.0, np.abs(V).max())
        assert np.abs(Fs2[k] - V).max() < tol * max(1.0, np.abs(V).max())
