"""The autotuner (pdfxc_autotune): every candidate shape of the INT8 path (groups of 4, 2, 1
blocks x 3 or 2 Vxc operand stages) is timed on the context's grid; the context keeps the
fastest, whose build still meets the INT8 tolerances against the reference; a later context of
the same workload class starts from the tuned shapes."""
import numpy as np
import pytest

from conftest import shell_table

pytestmark = pytest.mark.gpu

OZ_TOL = (2e-10, 5e-9)


@pytest.mark.parametrize("group,stages", [(1, 2), (2, 3)])
def test_explicit_shapes_meet_the_tolerances(chain12, group, stages):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(device=0, precision="mixed", split_terms=10, group_blocks=group, vxc_stages=stages)
    eng.set_system(shell_table(chain12))
    eng.set_grid(chain12["grid"][:, :4])
    assert eng.tuning()["group_blocks"] == group and eng.tuning()["vxc_stages"] == stages
    exc, _, V = eng.build_vxc("B3LYP", chain12["PA"])
    ref = chain12["B3LYP_exc"][0]
    assert abs(exc - ref) <= OZ_TOL[0] * abs(ref)
    assert np.abs(V - chain12["B3LYP_vxc"]).max() <= OZ_TOL[1] * np.abs(chain12["B3LYP_vxc"]).max()
    eng.close()


def test_autotune_keeps_the_fastest_and_caches_it(chain12):
    import torch
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(device=0, precision="mixed", split_terms=10)
    eng.set_system(shell_table(chain12))
    eng.set_grid(chain12["grid"][:, :4])
    dP = torch.tensor(chain12["PA"], device="cuda:0")
    res = eng.autotune("B3LYP", dP.data_ptr())
    print("autotune:", res)
    assert len(res) == 6
    assert res[0]["ms"] == min(r["ms"] for r in res) and all(r["ms"] > 0 for r in res)
    shapes = {(r["group_blocks"], r["vxc_stages"]) for r in res}
    assert shapes == {(g, s) for g in (4, 2, 1) for s in (3, 2)}
    t = eng.tuning()
    assert (t["group_blocks"], t["vxc_stages"]) == (res[0]["group_blocks"], res[0]["vxc_stages"])
    exc, _, V = eng.build_vxc("B3LYP", chain12["PA"])
    ref = chain12["B3LYP_exc"][0]
    assert abs(exc - ref) <= OZ_TOL[0] * abs(ref)
    # a new context of the same class starts from the tuned shapes
    e2 = XcEngine(device=0, precision="mixed", split_terms=10)
    e2.set_system(shell_table(chain12))
    e2.set_grid(chain12["grid"][:, :4])
    t2 = e2.tuning()
    assert (t2["group_blocks"], t2["vxc_stages"]) == (t["group_blocks"], t["vxc_stages"])
    e2.close()
    eng.close()
