"""Failure detection without a GPU fault: the bounded device waits of the tensor-core
kernels give up after their limit, record a code in the context's device error word,
and the host returns PDFXC_ERR_TIMEOUT; the context stays usable.

pdfxc_selftest_wait runs that path on purpose: one thread waits, through the same
bounded mbarrier wait as the contraction kernels, on an mbarrier that nothing ever
completes (a flag nothing sets), for 1 ms. No fault, trap or hang is involved."""
import time

import numpy as np
import pytest

from conftest import shell_table

pytestmark = pytest.mark.gpu


def test_bounded_wait_expires_and_context_stays_usable(water2):
    from proteindf_b200.xc import XcEngine
    eng = XcEngine(device=0, precision="mixed", split_terms=10)
    eng.set_system(shell_table(water2))
    g = water2["grid"]
    eng.set_grid(g[:, :4], g[:, 4].astype(np.int32))
    e0, _, V0 = eng.build_vxc("B3LYP", water2["PA"])
    t0 = time.perf_counter()
    st, msg = eng.selftest_wait(1e-3)
    dt = time.perf_counter() - t0
    print(f"self test: status {st} after {dt * 1e3:.2f} ms: {msg}")
    assert st == 4 and "expired" in msg  # PDFXC_ERR_TIMEOUT
    assert dt < 1.0
    # the error word was cleared: the next builds run and agree with the first
    for _ in range(2):
        e1, _, V1 = eng.build_vxc("B3LYP", water2["PA"])
        assert abs(e1 - e0) <= 1e-12 * abs(e0) and np.abs(V1 - V0).max() <= 1e-13
    assert eng.selftest_wait(0.0)[0] == 1  # PDFXC_ERR_ARG: no zero limit
    eng.close()
