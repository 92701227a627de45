"""The bounded waits of the persistent element kernels (GPU).

Every wait of k_element_tma / k_element_rows on a tile's bulk copies
(cp.async.bulk completing on an mbarrier) has a clock-cycle limit.  A test
hook (esdg_debug_bulk_wait_test) shortens the limit and names a tile whose
copies are never issued -- a failure made on the host side of the copy, no
GPU fault: that tile's wait runs out, its CTA records a time-out, lets its
other copies in flight land and returns, and the run reports ESDG_E_CUDA
with the engine's message.  The context stays usable: the same solver,
hook off and state re-uploaded, then runs to the oracle's result.
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import EsdgError, Solver
from oracle.oracle import OracleProblem
from tests.test_gpu_parity import rel_l2_per_var

pytestmark = pytest.mark.gpu

E_CUDA = -3


def _variants(s):
    ev = s.dc.element_variants() or {}
    return [v for v, c in enumerate(ev.get("ctas_per_sm", [])) if c > 0]


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_wait_runs_out_and_context_stays_usable(variant):
    pr = problems.curved_lake(N=4, nel=16, seed=2, ripple=0.03, steps=5)
    s = Solver(pr)
    try:
        s.run(T=1e9, max_steps=1)  # builds the variants' grids and the graph
        if variant not in _variants(s):
            pytest.skip(f"element variant {variant} not available here")
        s.dc.set_element_variant(variant)
        s.dc.copy_q_from_host(pr.q0)
        # about 1 ms of clock at most for any wait; tile 0 is never copied
        s.dc.debug_bulk_wait_test(2_000_000, 0)
        with pytest.raises(EsdgError) as ei:
            s.run(T=1e9, max_steps=2)
        assert ei.value.code == E_CUDA
        assert "bounded wait" in str(ei.value)
        # hook off, state re-uploaded: the same solver runs as the oracle
        s.dc.debug_bulk_wait_test(0, -1)
        s.dc.copy_q_from_host(pr.q0)
        t, steps = s.run(T=1e9, max_steps=5)
        q = s.q()
    finally:
        s.close()
    ref = OracleProblem(pr).run(T=1e9, max_steps=5)
    assert steps == ref["steps"] == 5
    assert max(rel_l2_per_var(q, ref["q"], pr.K, pr.ngl ** 2)) <= 1e-12
