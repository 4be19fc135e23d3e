"""Vertex de-duplication through the C ABI against numpy, at every bucket size its kernels switch on.

The reference de-duplicates the triangle corners with ``torch.unique(dim=0, return_inverse=True)``
over (vid0, vid1) pairs (``jspsr/core/reconstructor.py:380-383``): vertex ids in sorted pair order,
faces = the inverse.  ``ngs_vdedup_*`` buckets the keys by vid0 and sorts each bucket: buckets of
2..8 keys by one lane's sorting network, 9..512 by a warp, larger ones by a block.  The synthetic
keys here give buckets of 1..700 keys with repeated pairs, and the positions of a vertex are those
of the pair's first occurrence.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def synthetic_keys(seed=0):
    rng = np.random.default_rng(seed)
    sizes = [1, 2, 3, 7, 8, 9, 16, 31, 32, 33, 127, 128, 129, 511, 512, 513, 700]
    sizes += list(rng.integers(1, 12, size=3000))          # many small buckets, as a mesh has
    n_primal = len(sizes) + 500                             # some buckets stay empty
    owners = rng.permutation(n_primal)[:len(sizes)]
    vid0, vid1 = [], []
    for b, c in zip(owners, sizes):
        # vid1 < vid0 in a mesh; here any value, with repeats (the same edge from several cubes)
        distinct = rng.integers(0, 1 << 20, size=max(1, (c + 1) // 2))
        vid1.append(rng.choice(distinct, size=c))
        vid0.append(np.full(c, b))
    vid0 = np.concatenate(vid0).astype(np.int32)
    vid1 = np.concatenate(vid1).astype(np.int32)
    perm = rng.permutation(vid0.size)
    vids = np.stack([vid0[perm], vid1[perm]], 1)
    tris = rng.standard_normal((vids.shape[0], 3)).astype(np.float32)
    return vids, tris, n_primal


def numpy_dedup(vids, tris):
    keys = vids[:, 0].astype(np.int64) << 32 | vids[:, 1].astype(np.int64)
    uniq, first_idx, inverse = np.unique(keys, return_index=True, return_inverse=True)
    return inverse.astype(np.int64), tris[first_idx]


@pytest.mark.parametrize("seed", [0, 1])
def test_vertex_dedup_matches_unique_at_every_bucket_size(seed):
    from jspsr import _lib as L
    vids, tris, n_primal = synthetic_keys(seed)
    n = vids.shape[0]
    st = L.stream()
    dv, dt = torch.from_numpy(vids).to(DEV).contiguous(), torch.from_numpy(tris).to(DEV).contiguous()
    bcount = torch.zeros(n_primal, dtype=torch.int32, device=DEV)
    L.call("ngs_vdedup_count", L.ptr(dv), n, L.ptr(bcount), st)
    bstart, _ = L.scan(bcount)
    fill = torch.zeros(n_primal, dtype=torch.int32, device=DEV)
    sorted_keys = torch.empty(n, dtype=torch.int64, device=DEV)
    first = torch.empty(n, dtype=torch.int32, device=DEV)
    L.call("ngs_vdedup_sort", L.ptr(dv), n, L.ptr(bstart), n_primal, L.ptr(fill), L.ptr(sorted_keys), L.ptr(first), st)
    vid_of, nvert = L.scan(first)
    nv = int(nvert.item())
    faces = torch.empty(n, dtype=torch.int64, device=DEV)
    verts = torch.empty((nv, 3), dtype=torch.float32, device=DEV)
    L.call("ngs_vdedup_emit", L.ptr(dv), L.ptr(dt), n, L.ptr(bstart), L.ptr(fill), L.ptr(sorted_keys), L.ptr(vid_of),
           L.ptr(faces), L.ptr(verts), st)
    ref_faces, ref_verts = numpy_dedup(vids, tris)
    assert nv == ref_verts.shape[0]
    np.testing.assert_array_equal(faces.cpu().numpy(), ref_faces)
    np.testing.assert_array_equal(verts.cpu().numpy(), ref_verts)
    # the buckets come out sorted by (vid1, key index)
    sk = sorted_keys.cpu().numpy()
    bs, bc = bstart.cpu().numpy(), bcount.cpu().numpy()
    for b in np.nonzero(bc)[0][:200]:
        seg = sk[bs[b]:bs[b] + bc[b]]
        assert np.all(np.diff(seg) > 0)


@pytest.mark.parametrize("m", [1, 31, 32, 33, 1000, 4099])
def test_dual_mc_emit_with_counts_matches_the_oracle(m):
    """Dual MC over an uncompacted accumulation (cnt != 8 cubes emit nothing) through the count,
    scan and emit entry points -- the emit runs a warp per 32 cubes, so the cube count is varied
    around multiples of 32, and the last cube always emits -- against the oracle's dual MC of the
    complete cubes (``dual_mc.cu:33-189``)."""
    from jspsr import _lib as L
    rng = np.random.default_rng(m)
    n_primal = 3 * m + 50
    pos = rng.standard_normal((n_primal, 3)).astype(np.float32)
    vals = rng.standard_normal(n_primal).astype(np.float32)
    acc = rng.integers(0, n_primal, size=(m, 8)).astype(np.int32)
    cnt = np.where(rng.random(m) < 0.8, 8, rng.integers(1, 12, size=m)).astype(np.int32)
    cnt[-1] = 8
    acc[-1] = [0, 1, 2, 3, 4, 5, 6, 7]
    vals[:8] = [-1.0, 0.5, 0.7, 0.9, 1.1, 1.3, 1.5, 1.7]      # one corner inside: the last cube emits
    st = L.stream()
    dacc, dcnt = torch.from_numpy(acc).to(DEV), torch.from_numpy(cnt).to(DEV)
    dpos, dval = torch.from_numpy(pos).to(DEV), torch.from_numpy(vals).to(DEV)
    vcount = torch.empty(m, dtype=torch.int32, device=DEV)
    L.call("ngs_dual_mc_count", L.ptr(dacc), 1, L.ptr(dcnt), m, L.ptr(dval), L.ptr(vcount), st)
    voff, vtot = L.scan(vcount)
    nv = int(vtot.item())
    tris = torch.empty((nv, 3), dtype=torch.float32, device=DEV)
    vids = torch.empty((nv, 2), dtype=torch.int32, device=DEV)
    L.call("ngs_dual_mc_emit", L.ptr(dacc), 1, L.ptr(dcnt), m, L.ptr(dpos), L.ptr(dval), L.ptr(voff), L.ptr(tris),
           L.ptr(vids), st)
    from oracle import ops as O
    acc3 = np.stack([acc, np.zeros_like(acc)], -1)              # the oracle's (primal id, depth) pairs
    rt, rv = O.dual_marching_cubes_sparse(acc3[cnt == 8], pos, vals)
    assert nv == rv.reshape(-1, 2).shape[0] and nv > 0
    np.testing.assert_array_equal(vids.cpu().numpy(), rv.reshape(-1, 2))
    np.testing.assert_allclose(tris.cpu().numpy(), rt.reshape(-1, 3), atol=1e-5)
