"""FFT pass-split tuning: every split computes the same values. Evaluate +
interpolate under each tile geometry (specialised and generic pass kernels)
must give bit-identical evaluations to the default split and to the oracle,
and the autotuner must install only valid splits. The default 13 / 4 is put
back afterwards."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = O.P

SPLITS = [(13, 4), (12, 4), (11, 4), (10, 4), (13, 3), (13, 5), (12, 5), (11, 5), (10, 5), (8, 3), (6, 0), (13, 0)]


@pytest.fixture(scope="module")
def B():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpustark.backend import GpuBackend
    yield GpuBackend
    GpuBackend.fft_set_tuning(0, 13, 4)


def _round_trip(B, coeffs, log, tw, blowup):
    ev = B.evaluate_polynomials(coeffs, log + blowup, tw)
    back = [e.clone() for e in ev]
    B.interpolate_columns(back, log + blowup, tw)
    torch.cuda.synchronize()
    return ev, back


@pytest.mark.parametrize("log,n_cols,blowup", [(11, 3, 1), (14, 2, 0), (17, 2, 2), (18, 3, 2), (21, 1, 1), (24, 1, 0)])
def test_every_split_gives_the_same_values(B, log, n_cols, blowup):
    from gpustark.backend import to_device
    rng = np.random.default_rng(log * 7 + blowup)
    tw = B.precompute_twiddles(log + blowup - 1)
    host = [rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.uint32) for _ in range(n_cols)]
    coeffs = [to_device(h) for h in host]
    B.fft_set_tuning(0, 13, 4)
    want, _ = _round_trip(B, coeffs, log, tw, blowup)
    if log <= 14:
        for h, w in zip(host, want):
            assert np.array_equal(O.evaluate(h, log + blowup), w.cpu().numpy().view(np.uint32))
    for tile, coal in SPLITS:
        B.fft_set_tuning(0, tile, coal)
        ev, back = _round_trip(B, coeffs, log, tw, blowup)
        for e, w in zip(ev, want):
            assert torch.equal(e, w), (tile, coal)
        for b, c in zip(back, coeffs):
            padded = torch.zeros_like(b)
            padded[: c.numel()] = c
            assert torch.equal(b, padded), (tile, coal)
    B.fft_set_tuning(0, 13, 4)


def test_autotune_installs_valid_splits(B):
    from gpustark.backend import to_device
    picks = B.fft_autotune(8, 22, 2)
    assert sorted(picks) == [(n, e) for n in range(8, 23) for e in range(3)]
    for (log, ext), (tile, coal) in picks.items():
        assert 6 <= tile <= 13 and coal <= 5 and coal + 5 <= tile
        assert B.fft_get_tuning(log, ext) == (tile, coal)
    rng = np.random.default_rng(5)
    tw = B.precompute_twiddles(21)
    coeffs = [to_device(rng.integers(0, P, 1 << 21, dtype=np.int64).astype(np.uint32))]
    ev, back = _round_trip(B, coeffs, 21, tw, 1)
    B.fft_set_tuning(0, 13, 4)
    want, _ = _round_trip(B, coeffs, 21, tw, 1)
    assert torch.equal(ev[0], want[0])
    assert torch.equal(back[0][: 1 << 21], coeffs[0]) and not back[0][1 << 21:].any()
