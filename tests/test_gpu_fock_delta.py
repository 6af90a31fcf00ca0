"""The XC part of the Fock update on the device (pdfxc_build_vxc_delta_device; the reference's
DfFockMatrix::setXC_DIRECT, src/libpdf/DfFockMatrix.h:711-721: Fxc of this iteration, minus
Fxc of the previous iteration from the second one on) against separate builds."""
import numpy as np
import pytest

from conftest import shell_table

pytestmark = pytest.mark.gpu


def _engine(fx, precision):
    from proteindf_b200.xc import XcEngine
    e = XcEngine(device=0, precision=precision)
    e.set_system(shell_table(fx))
    e.set_grid(fx["grid"][:, :4], fx["grid"][:, 4].astype(np.int32))
    return e


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_delta_matches_separate_builds(water2, precision):
    import torch
    P1 = water2["PA"]
    rng = np.random.default_rng(3)
    E = rng.normal(scale=1e-3, size=P1.shape)
    P2 = P1 + 0.5 * (E + E.T)
    ref = _engine(water2, precision)
    exc1, nel1, V1 = ref.build_vxc("B3LYP", P1)
    exc2, _, V2 = ref.build_vxc("B3LYP", P2)
    ref.close()

    e = _engine(water2, precision)
    dP = torch.tensor(P1, device="cuda:0")
    dV = torch.empty_like(dP)
    dD = torch.empty_like(dP)
    x1, n1 = e.build_vxc_delta_device("B3LYP", 1, dP.data_ptr(), dD.data_ptr(), dV.data_ptr())
    # equal up to the summation order of the FP64 atomics
    assert abs(x1 - exc1) <= 1e-12 and abs(n1 - nel1) <= 1e-12
    assert np.abs(dV.cpu().numpy() - V1).max() <= 1e-13
    assert np.abs(dD.cpu().numpy() - V1).max() <= 1e-13  # iteration 1: Fxc itself
    dP.copy_(torch.tensor(P2))
    x2, _ = e.build_vxc_delta_device("B3LYP", 2, dP.data_ptr(), dD.data_ptr())  # no d_V this time
    assert abs(x2 - exc2) <= 1e-12
    assert np.abs(dD.cpu().numpy() - (V2 - V1)).max() <= 2e-13
    # iteration 3 from the same density: the difference vanishes up to the atomics' order
    e.build_vxc_delta_device("B3LYP", 3, dP.data_ptr(), dD.data_ptr())
    assert np.abs(dD.cpu().numpy()).max() <= 1e-13
    e.close()


def test_delta_history_errors(water2):
    import torch
    e = _engine(water2, "fp64")
    dP = torch.tensor(water2["PA"], device="cuda:0")
    dD = torch.empty_like(dP)
    with pytest.raises(RuntimeError, match="status 1"):  # PDFXC_ERR_ARG
        e.build_vxc_delta_device("B3LYP", 0, dP.data_ptr(), dD.data_ptr())
    with pytest.raises(RuntimeError, match="status 3"):  # no Fxc of iteration 1 yet
        e.build_vxc_delta_device("B3LYP", 2, dP.data_ptr(), dD.data_ptr())
    e.build_vxc_delta_device("B3LYP", 1, dP.data_ptr(), dD.data_ptr())
    with pytest.raises(RuntimeError, match="status 3"):  # iteration 2 skipped
        e.build_vxc_delta_device("B3LYP", 3, dP.data_ptr(), dD.data_ptr())
    e.build_vxc_delta_device("B3LYP", 2, dP.data_ptr(), dD.data_ptr())
    # a new system clears the history
    e.set_system(shell_table(water2))
    e.set_grid(water2["grid"][:, :4], water2["grid"][:, 4].astype(np.int32))
    with pytest.raises(RuntimeError, match="status 3"):
        e.build_vxc_delta_device("B3LYP", 3, dP.data_ptr(), dD.data_ptr())
    e.build_vxc_delta_device("B3LYP", 1, dP.data_ptr(), dD.data_ptr())
    e.close()
