"""A device wait that runs out ends its kernel normally with an error status
that the host reads (no fault, no hang), and the context stays usable.

The wait is the one-right-hand-side solve's chain-flag wait, made to run out
on purpose: cad_wait_timeout_probe starts the chain's order counter past
block 0, so every block waits for a flag that nothing sets, with a short
limit set by cad_set_wait_limit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_chain_wait_runs_out_and_the_context_survives(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    try:
        _lib.check(L.cad_set_wait_limit(ctx, 2000), ctx)
        for n in (640, 1000):
            rc = L.cad_wait_timeout_probe(ctx, n)
            assert rc == _lib.CAD_ERR_TIMEOUT
            assert b"wait ran out" in L.cad_last_error(ctx)
    finally:
        _lib.check(L.cad_set_wait_limit(ctx, 1 << 22), ctx)
    # the same context solves correctly afterwards
    rng = np.random.default_rng(0)
    A = rng.standard_normal((300, 300)) + 300 * np.eye(300)
    b = rng.standard_normal(300)
    x = cad.solve(A, b)
    assert np.linalg.norm(A @ x - b) <= 1e-12 * np.linalg.norm(b)


def test_wait_limit_arguments(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    assert L.cad_set_wait_limit(ctx, 0) == _lib.CAD_ERR_ARG
    assert L.cad_wait_timeout_probe(ctx, 64) == _lib.CAD_ERR_ARG
