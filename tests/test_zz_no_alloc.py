"""GPU test of cad_td_sum_eval_noalloc, the summing-overload entry point for
callers that cannot let a library allocate device memory (hosts whose device
memory belongs to their own pool and budget, or services with a fixed
per-tenant memory slice).  It must give the same results as the regular
device entry point, cad_td_sum_eval_dev, on consecutive calls that reuse its
static scratch array, without changing the device's free memory.

Kept in a file that sorts last so that a run stopping at the first failure has
run every other test first; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from helpers import assert_parity, random_points, random_triangles

pytestmark = pytest.mark.gpu


def _case(seed, n, m, hs):
    rng = np.random.default_rng(seed)
    P1, P2, P3 = random_triangles(rng, n)
    pts = random_points(rng, m) if hs else random_points(rng, m, lo=(-4, -4, -5), hi=(4, 4, 3))
    sl = rng.uniform(-1e-3, 1e-3, (3, n))
    return pts, P1, P2, P3, sl


def _device_inputs(torch, pts, P1, P2, P3, sl):
    dev = torch.device("cuda", 0)

    def t(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)

    cols = [t(np.asfortranarray(p).ravel(order="F")) for p in (P1, P2, P3)]
    return [t(pts[:, k]) for k in range(3)], cols, [t(sl[k]) for k in range(3)]


def _outputs(torch, m):
    dev = torch.device("cuda", 0)
    return (torch.empty(6 * m, dtype=torch.float64, device=dev), torch.empty(3 * m, dtype=torch.float64, device=dev))


def _run_noalloc(L, torch, xyz, cols, slips, hs, m, out):
    S, U = out
    S.fill_(np.nan)
    U.fill_(np.nan)
    stream = torch.cuda.current_stream(torch.device("cuda", 0))
    rc = L.cad_td_sum_eval_noalloc(ctypes.c_void_p(stream.cuda_stream), xyz[0].data_ptr(), xyz[1].data_ptr(),
                                   xyz[2].data_ptr(), m, cols[0].data_ptr(), cols[1].data_ptr(), cols[2].data_ptr(),
                                   len(slips[0]), slips[0].data_ptr(), slips[1].data_ptr(), slips[2].data_ptr(),
                                   0.25, 1, 1, hs, S.data_ptr(), U.data_ptr())
    assert rc == 0, rc
    torch.cuda.synchronize()
    return S.view(6, m).cpu().numpy(), U.view(3, m).cpu().numpy()


def _run_regular(L, ctx, torch, xyz, cols, slips, hs, m):
    dev = torch.device("cuda", 0)
    S = torch.empty(6 * m, dtype=torch.float64, device=dev)
    U = torch.empty(3 * m, dtype=torch.float64, device=dev)
    rc = L.cad_td_sum_eval_dev(ctx, xyz[0].data_ptr(), xyz[1].data_ptr(), xyz[2].data_ptr(), m, cols[0].data_ptr(),
                               cols[1].data_ptr(), cols[2].data_ptr(), len(slips[0]), slips[0].data_ptr(),
                               slips[1].data_ptr(), slips[2].data_ptr(), 0.25, 1, 1, hs, S.data_ptr(), U.data_ptr())
    assert rc == 0, rc
    torch.cuda.synchronize()
    return S.view(6, m).cpu().numpy(), U.view(3, m).cpu().numpy()


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    from cutanddisplacejulia_b200 import _lib, build
    build.build()
    L = _lib.load()
    ctx = _lib.context(0)
    cases = [_case(101, 40, 700, 1), _case(202, 17, 1500, 0), _case(303, 64, 333, 1)]
    prepared = [(_device_inputs(torch, *c[:5]), c[0].shape[0], hs) for c, hs in zip(cases, (1, 0, 1))]
    expected = [_run_regular(L, ctx, torch, *inp, hs, m) for inp, m, hs in prepared]
    outs = [_outputs(torch, m) for _, m, _ in prepared]
    # first call on this device: looks up the scratch address (and loads code)
    _run_noalloc(L, torch, *prepared[0][0], prepared[0][2], prepared[0][1], outs[0])
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    for (inp, m, hs), (So, Uo), out in zip(prepared, expected, outs):
        S, U = _run_noalloc(L, torch, *inp, hs, m, out)
        assert_parity(S, So)
        assert_parity(U, Uo)
    # the same case again after a different one: stale scratch must not leak in
    S, U = _run_noalloc(L, torch, *prepared[0][0], prepared[0][2], prepared[0][1], outs[0])
    assert_parity(S, expected[0][0])
    assert_parity(U, expected[0][1])
    assert torch.cuda.mem_get_info(0)[0] == free_before


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from cutanddisplacejulia_b200 import _lib, build
    build.build()
    L = _lib.load()
    dev = torch.device("cuda", 0)
    big = torch.zeros(16385, dtype=torch.float64, device=dev)
    one = torch.zeros(3, dtype=torch.float64, device=dev)
    out = torch.zeros(9 * 16385, dtype=torch.float64, device=dev)
    rc = L.cad_td_sum_eval_noalloc(None, big.data_ptr(), big.data_ptr(), big.data_ptr(), 16385, one.data_ptr(),
                                   one.data_ptr(), one.data_ptr(), 1, one.data_ptr(), one.data_ptr(), one.data_ptr(),
                                   0.25, 1, 1, 0, out.data_ptr(), out.data_ptr())
    assert rc == _lib.CAD_ERR_TOO_LARGE
    tri = torch.zeros(3 * 1025, dtype=torch.float64, device=dev)
    rc = L.cad_td_sum_eval_noalloc(None, one.data_ptr(), one.data_ptr(), one.data_ptr(), 1, tri.data_ptr(),
                                   tri.data_ptr(), tri.data_ptr(), 1025, tri.data_ptr(), tri.data_ptr(), tri.data_ptr(),
                                   0.25, 1, 1, 0, out.data_ptr(), out.data_ptr())
    assert rc == _lib.CAD_ERR_TOO_LARGE


def test_noalloc_checks_half_space_triangles_without_points():
    # no observation points but a triangle above z = 0: both entry points
    # reject it in half space (src/TD.jl:606-619), and accept it in full space
    torch = pytest.importorskip("torch")
    from cutanddisplacejulia_b200 import _lib, build
    build.build()
    L = _lib.load()
    ctx = _lib.context(0)
    dev = torch.device("cuda", 0)
    col = (lambda p: torch.tensor(np.asfortranarray(np.array([p], dtype=np.float64)).ravel(order="F"), device=dev))
    P1, P2, P3 = col([0.0, 0.0, 0.5]), col([1.0, 0.0, -1.0]), col([0.0, 1.0, -1.0])
    sl = torch.full((1,), 1e-3, dtype=torch.float64, device=dev)
    pt = torch.zeros(1, dtype=torch.float64, device=dev)
    out = torch.zeros(9, dtype=torch.float64, device=dev)
    for hs, want in ((1, _lib.CAD_ERR_HS_ABOVE_SURFACE), (0, 0)):
        rc = L.cad_td_sum_eval_noalloc(None, pt.data_ptr(), pt.data_ptr(), pt.data_ptr(), 0, P1.data_ptr(),
                                       P2.data_ptr(), P3.data_ptr(), 1, sl.data_ptr(), sl.data_ptr(), sl.data_ptr(),
                                       0.25, 1, 1, hs, out.data_ptr(), out.data_ptr())
        rc_dev = L.cad_td_sum_eval_dev(ctx, pt.data_ptr(), pt.data_ptr(), pt.data_ptr(), 0, P1.data_ptr(),
                                       P2.data_ptr(), P3.data_ptr(), 1, sl.data_ptr(), sl.data_ptr(), sl.data_ptr(),
                                       0.25, 1, 1, hs, out.data_ptr(), out.data_ptr())
        assert rc == want and rc_dev == want, (hs, rc, rc_dev)
