"""FFT pass geometry checked on the CPU for every pass split the tuning
interface accepts: an emulation of the index arithmetic of fft_pass_kernel
and fft_tile_kernel as run_passes launches them (nitroozk-stwo_b200/csrc/
fft.cu) asserts that every global load and store lies in the column, that
vector accesses are 16-byte aligned and cover exactly the elements the
scalar mapping names, that every element is loaded and stored once per pass,
that twiddle reads stay inside the tree with the alignment of their vector
width, that shared-memory indices stay inside the launch's allocation, and
that no block exceeds 256 threads. Mirrors the kernels' formulas; a change
to either side must change both."""
import numpy as np
import pytest


def partition(layers, T, C):
    if layers <= T:
        return [(0, layers)]
    np_ = 1 + (layers - T + (T - C) - 1) // (T - C)
    lr = min(T - C, (layers + np_ - 1) // np_)
    l0 = layers - lr * (np_ - 1)
    parts = [(0, l0)]
    lo = l0
    for _ in range(1, np_):
        parts.append((lo, lr)); lo += lr
    return parts


def specialised(R, c, L):
    return R == 5 and ((c == 0 and 5 <= L <= 13) or (c == 4 and 5 <= L <= 9) or (c == 5 and 5 <= L <= 8))


def padw(e):
    return e + (e >> 5)


def check_split(n, layers, T, C, INV, src_mask, tw_len):
    parts = partition(layers, T, C)
    if not INV:
        parts = parts[::-1]
    N = 1 << n
    for p, (lo, L) in enumerate(parts):
        c = min(C, lo); t = c + L; R = min(5, L); K = (L + R - 1) // R
        tpt_log = t - R; tiles_log = n - t
        assert tiles_log >= 0, ("tile larger than domain", n, t)
        shift = 7 - tpt_log if tpt_log < 7 else 0
        shift = min(shift, tiles_log)
        threads = 1 << (tpt_log + shift); gx = 1 << (tiles_log - shift)
        assert threads <= 256, threads
        spec = specialised(R, c, L)
        words = 1 << (t + shift)
        smem_words = words + (words >> 5) if spec else words
        mask = src_mask if p == 0 else 0xffffffff
        bx = np.repeat(np.arange(gx, dtype=np.int64), threads)
        tid = np.tile(np.arange(threads, dtype=np.int64), gx)
        ltid = tid & ((1 << tpt_log) - 1)
        sub = tid >> tpt_log
        tile = (bx << shift) | sub
        ml = lo - c
        midlow = tile & ((1 << ml) - 1)
        hi = tile >> ml
        basev = (hi << (lo + L)) | (midlow << c)
        cmask = (1 << c) - 1
        NQ = 1 << R
        loads = []; stores = []
        for k in range(K):
            if INV:
                if k + 1 < K: s0, ja, jb = c + k * R, 0, R
                else: s0 = t - R; ja = c + k * R - s0; jb = R
            else:
                if k + 1 < K: s0, ja, jb = t - (k + 1) * R, 0, R
                else: s0 = c; ja = 0; jb = t - k * R - c
            ebase = ((ltid >> s0) << (s0 + R)) | (ltid & ((1 << s0) - 1))
            gbase = basev | ((ebase >> c) << lo) | (ebase & cmask)
            q = np.arange(NQ, dtype=np.int64)
            e = ebase[:, None] | (q[None, :] << s0)
            v = basev[:, None] | ((e >> c) << lo) | (e & cmask)
            # shared memory index
            smb = (sub << t)[:, None] | e
            sidx = (padw(sub << t)[:, None] + padw(ebase)[:, None] + padw(q << s0)[None, :]) if spec else smb
            assert sidx.min() >= 0 and sidx.max() < smem_words, ("smem", sidx.max(), smem_words)
            vec_cond = (s0 == 0 and c == 0 and lo == 0 and NQ >= 4)
            if k == 0:
                if vec_cond and mask == 0xffffffff:
                    assert (gbase % 4 == 0).all(), "vec load misaligned"
                    la = gbase[:, None] + q[None, :]
                    assert (la == v).all(), "vec load != element addresses"
                else:
                    la = v & mask
                assert la.min() >= 0 and la.max() < N, "load oob"
                loads.append(la.ravel())
            # twiddles
            vth = gbase
            for jj in range(R):
                j = jj if INV else R - 1 - jj
                if j < ja or j >= jb: continue
                i = lo + s0 + j - c
                assert 0 <= i < n
                hth = vth >> (i + 1)
                COUNT = 1 << (R - 1 - j)
                if i >= 1:
                    off = tw_len - (1 << (n - i)) + hth
                    assert off.min() >= 0 and (off + COUNT).max() <= tw_len, "tw oob"
                    if COUNT >= 4: assert (off % 4 == 0).all(), ("tw uint4 misaligned", i, COUNT)
                    elif COUNT == 2: assert (off % 2 == 0).all(), "tw uint2 misaligned"
                else:
                    base = tw_len - (1 << (n - 1))
                    if COUNT >= 4:
                        assert (hth % 4 == 0).all(), "circle tw group misaligned"
                        off = base + 2 * ((hth >> 2))
                        assert base % 2 == 0 and off.min() >= 0 and (off + 2 * (COUNT // 4)).max() <= tw_len
                    else:
                        for g in range(COUNT):
                            h = hth + g
                            o = base + 2 * (h >> 2) + np.where((h & 3) < 2, 1, 0)
                            assert o.min() >= 0 and o.max() < tw_len
            if k + 1 == K:
                if vec_cond:
                    assert (gbase % 4 == 0).all(), "vec store misaligned"
                    sa = gbase[:, None] + q[None, :]
                    assert (sa == v).all(), "vec store != element addresses"
                else:
                    stride = 1 << (s0 - c + lo)
                    sa = gbase[:, None] + q[None, :] * stride
                    assert (sa == v).all(), "strided store != element addresses"
                assert sa.min() >= 0 and sa.max() < N, "store oob"
                stores.append(sa.ravel())
        st = np.sort(np.concatenate(stores))
        assert (st == np.arange(N)).all(), "stores not a permutation"
        if mask == 0xffffffff:
            ld = np.sort(np.concatenate(loads))
            assert (ld == np.arange(N)).all(), "loads not a permutation"
        if spec:
            assert (c, L) in [(0, l) for l in range(5, 14)] + [(4, l) for l in range(5, 10)] + [(5, l) for l in range(5, 9)]


SPLITS = [(T, C) for T in range(6, 14) for C in range(0, 6) if C + 5 <= T]


@pytest.mark.parametrize("T,C", SPLITS)


def test_pass_geometry_in_bounds_and_aligned(T, C):
    for n in range(3, 17):
        for blow in range(0, 3):
            layers = n - blow
            if layers < 1:
                continue
            check_split(n, layers, T, C, False, (1 << layers) - 1, 1 << (n - 1))
            if blow == 0:
                check_split(n, layers, T, C, True, 0xffffffff, 1 << (n - 1))
