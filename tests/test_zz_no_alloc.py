"""gs_batch_eval_at_point_noalloc (static device scratch, no allocation) against
gs_batch_eval_at_point (context scratch pool): identical results on two calls
in a row with different sizes and points, so a stale word left in the shared
array by the first call would show in the second. Collected last, so that it
runs both alone and after every other test in the session."""
import numpy as np
import pytest

import pyoracle as O

P = O.P
GS_ERR_INVALID = 1  # include/gpustark.h


def rand(rng, *shape):
    return rng.integers(0, P, shape, dtype=np.int64).astype(np.uint32)


def test_noalloc_rejects_oversize_before_any_launch():
    """Limits are checked on the host before any CUDA call (no GPU needed)."""
    from gpustark import _lib as L
    lib = L.lib()
    pp, keep = L.ptr_array([8] * 257)
    out = (L.QM31 * 257)()
    pt = L.PointQM31()
    assert lib.gs_batch_eval_at_point_noalloc(None, pp, 257, 4, pt, out) == GS_ERR_INVALID
    assert b"256" in lib.gs_last_error()
    pp, keep = L.ptr_array([8] * 2)
    assert lib.gs_batch_eval_at_point_noalloc(None, pp, 2, 28, pt, out) == GS_ERR_INVALID
    assert b"2^18" in lib.gs_last_error()
    assert lib.gs_batch_eval_at_point_noalloc(None, pp, 2, 31, pt, out) == GS_ERR_INVALID


@pytest.mark.gpu
def test_noalloc_matches_context_entry_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark.backend import GpuBackend as B, to_device
    rng = np.random.default_rng(2024)
    # call 1: the largest case the static scratch holds (256 x 2^10 chunks)
    big = [rand(rng, 1 << 20) for _ in range(256)]
    pt1 = rand(rng, 8)
    # call 2: fewer, smaller polynomials at another point
    small = [rand(rng, 1 << 13) for _ in range(37)]
    pt2 = rand(rng, 8)
    d_big = [to_device(p) for p in big]
    d_small = [to_device(p) for p in small]
    got1 = B.batch_eval_at_point_noalloc(d_big, pt1)
    got2 = B.batch_eval_at_point_noalloc(d_small, pt2)
    assert got1 == B.batch_eval_at_point(d_big, pt1)
    assert got2 == B.batch_eval_at_point(d_small, pt2)
    # and once more in the opposite order, on a side stream
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    assert B.batch_eval_at_point_noalloc(d_small, pt2, stream=s) == got2
    assert B.batch_eval_at_point_noalloc(d_big[:5], pt1, stream=s) == got1[:5]
    # spot-check against the oracle (independent of both entry points)
    for i in (0, 36):
        assert [int(x) for x in O.eval_at_point(small[i], pt2)] == got2[i]
