"""The bound on |column - row| that decides a level's 2-byte column deltas and the solver's vector
window.

``ngs_grid_band_bound`` (behind ``Reconstruction._row_span_bound``) works from the rank bitmap alone:
the first rank of every (x, y) column.  Its rule is restated here in numpy; on CPU the restatement,
over bitmaps built from the oracle's voxel sets, must cover every entry of the oracle's matrices of
the same levels and stay close to the largest one; on the GPU the kernel must give the restatement's
value exactly.
"""
import numpy as np
import pytest
import torch

from oracle import fast as F


def _bitmap_words(coords, stride):
    """int64 [nwords * 2] rank-bitmap words (the libngs layout: {u32 rank, u32 pad, u64 bits}) of a
    level whose voxel min-corners are ``coords``, and a Grid-like description."""
    lo = coords.min(0) // stride * stride
    dims = (coords.max(0) - lo) // stride + 1
    zwords = (int(dims[2]) + 63) // 64
    ijk = (coords - lo) // stride
    w = (ijk[:, 0] * dims[1] + ijk[:, 1]) * zwords + ijk[:, 2] // 64
    nwords = int(dims[0] * dims[1] * zwords)
    bits = np.zeros(nwords, np.uint64)
    np.bitwise_or.at(bits, w, (np.uint64(1) << (ijk[:, 2] % 64).astype(np.uint64)))
    cnt = np.array([bin(int(b)).count("1") for b in bits], np.int64)
    rank = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    words = np.zeros((nwords, 2), np.int64)
    words[:, 0] = rank
    words[:, 1] = bits.view(np.int64)

    class G:
        pass
    g = G()
    g.dims, g.zwords = [int(v) for v in dims], zwords
    return torch.from_numpy(words.reshape(-1)), g


def band_bound(words, g, n):
    """The kernel's rule: per (x, y) column the larger of (first rank of column (x+2, y+2) + 1 -
    first rank of the column) and (first rank of the next column - first rank of column (x-2, y-2)),
    the maximum over columns; the first rank past the last column is n."""
    d0, d1, zw = g.dims[0], g.dims[1], g.zwords
    first = words.numpy().reshape(-1, 2)[::zw, 0][:d0 * d1].astype(np.int64)
    starts = np.concatenate([first, [n]])
    x = np.arange(d0)[:, None]
    y = np.arange(d1)[None, :]
    own = x * d1 + y
    lo = np.clip(x - 2, 0, None) * d1 + np.clip(y - 2, 0, None)
    hi = np.clip(x + 2, None, d0 - 1) * d1 + np.clip(y + 2, None, d1 - 1) + 1
    return int(max((starts[hi] - starts[own]).max(), (starts[own + 1] - starts[lo]).max()))


def oracle_levels():
    from jspsr import synthetic
    xyz, nrm, _ = synthetic.superquadrics(20000, k=2, seed=3)
    r = F.reconstruct(xyz, nrm, 1 / 256, 3, 0.7, 4.0, cg_tol=1e-6, mesh=False)
    for d in range(3):
        yield d, r[f"coords{d}"].astype(np.int64), r[f"rowptr{d}"], r[f"cols{d}"]


def test_row_span_bound_covers_every_column():
    for d, coords, rp, cols in oracle_levels():
        words, g = _bitmap_words(coords, 1 << d)
        bound = band_bound(words, g, coords.shape[0])
        rows = np.repeat(np.arange(coords.shape[0]), np.diff(rp))
        actual = int(np.abs(cols - rows).max())
        assert actual <= bound, (d, actual, bound)
        assert bound <= 1.25 * actual + 64, (d, actual, bound)    # and it is tight enough to use


@pytest.mark.gpu
def test_band_bound_kernel_equals_the_rule():
    from jspsr import _lib as L
    from jspsr.core.pipeline import Level, Reconstruction
    dev = torch.device("cuda", 0)
    for d, coords, _, _ in oracle_levels():
        words, g = _bitmap_words(coords, 1 << d)
        stride = 1 << d
        lo = coords.min(0) // stride * stride
        grid, dwords = L.make_grid(lo, g.dims, stride, dev)
        dwords.copy_(words.to(dev))
        lv = Level(stride=stride, grid=grid, words=dwords, n=coords.shape[0])
        got = int(Reconstruction._row_span_bound(lv))
        assert got == band_bound(words, g, coords.shape[0]), d
