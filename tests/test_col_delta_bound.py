"""The bound on |column - row| that decides whether a level's solver reads 2-byte column deltas.

``Reconstruction._row_span_bound`` works from the rank bitmap alone (the first rank of every (x, y)
column);
here it runs on CPU over bitmaps built from the oracle's voxel sets and must cover every entry of
the oracle's matrices of the same levels.
"""
import numpy as np
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


def test_row_span_bound_covers_every_column():
    from jspsr import synthetic
    from jspsr.core.pipeline import Level, Reconstruction
    xyz, nrm, _ = synthetic.superquadrics(20000, k=2, seed=3)
    r = F.reconstruct(xyz, nrm, 1 / 256, 3, 0.7, 4.0, cg_tol=1e-6, mesh=False)
    for d in range(3):
        coords, rp, cols = r[f"coords{d}"], r[f"rowptr{d}"], r[f"cols{d}"]
        words, g = _bitmap_words(coords.astype(np.int64), 1 << d)
        lv = Level(stride=1 << d, grid=g, words=words, n=coords.shape[0])
        bound = int(Reconstruction._row_span_bound(lv))
        rows = np.repeat(np.arange(coords.shape[0]), np.diff(rp))
        actual = int(np.abs(cols - rows).max())
        assert actual <= bound, (d, actual, bound)
        assert bound <= 1.25 * actual + 64, (d, actual, bound)    # and it is tight enough to use
