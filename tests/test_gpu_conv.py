"""Sparse convolution (gather-GEMM on tcgen05) against a torch restatement of the reference's op.

The reference (``csrc/sparse_op/convolution_cuda.cu:52-282``, ``models/ascn/utils.py:108-190``)
gathers, multiplies and scatters per kernel offset; its CPU branch (``utils.py:153-165``) is the
loop ``output[o] += input[i] @ weight[k]`` over the pairs of every offset, restated here in FP32
on the same (16-bit-rounded) inputs.  Tolerances: FP32 outputs of 16-bit inputs 1e-5 relative L2
(the products are exact in FP32, only the summation order differs); 16-bit outputs 2^-8 (bf16) and
2^-11 (fp16) relative per element, as one rounding of the FP32 sum; FP32 features (CUDA cores) 1e-5.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def voxel_maps(n_side=24, keep=0.35, ksize=3, seed=0, stride=1):
    """A random sparse voxel set and its neighbour map (pairs (input, output) per offset of a ksize^3
    kernel, input = output + offset), grouped by offset: nbmaps int32 [P, 2], nbsizes int32 [K]."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    r = np.linalg.norm(g - n_side / 2, axis=1)
    shell = g[(np.abs(r - n_side / 3) < 3) & (rng.random(len(g)) < keep)]
    index = {tuple(c): i for i, c in enumerate(shell)}
    half = ksize // 2
    offs = [(dx, dy, dz) for dx in range(-half, ksize - half) for dy in range(-half, ksize - half)
            for dz in range(-half, ksize - half)]
    maps, sizes = [], []
    for d in offs:
        pairs = [(index[t], o) for o, c in enumerate(shell) if (t := (c[0] + d[0], c[1] + d[1], c[2] + d[2])) in index]
        maps += pairs
        sizes.append(len(pairs))
    nbmaps = torch.tensor(np.array(maps, np.int32).reshape(-1, 2), device=DEV)
    return len(shell), nbmaps, torch.tensor(sizes, dtype=torch.int32)


def ref_forward(x, w, nbmaps, nbsizes, n_out, transposed):
    out = torch.zeros(n_out, w.shape[-1], dtype=torch.float32, device=x.device)
    a = 0
    for k in range(w.shape[0]):
        b = a + int(nbsizes[k])
        i, o = (nbmaps[a:b, 1], nbmaps[a:b, 0]) if transposed else (nbmaps[a:b, 0], nbmaps[a:b, 1])
        out.index_add_(0, o.long(), x[i.long()].float() @ w[k].float())
        a = b
    return out


def rel(a, b):
    return float(torch.linalg.norm(a.double() - b.double()) / max(float(torch.linalg.norm(b.double())), 1e-30))


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
@pytest.mark.parametrize("cin,cout", [(32, 32), (64, 64), (16, 128), (128, 256), (96, 48), (64, 320)])
def test_forward_matches_reference_loop(dtype, cin, cout):
    from jspsr import ext
    n, nbmaps, nbsizes = voxel_maps()
    gen = torch.Generator(device="cpu").manual_seed(cin * 1000 + cout)
    x = torch.randn(n, cin, generator=gen).to(DEV, dtype)
    w = (torch.randn(27, cin, cout, generator=gen) / cin ** 0.5).to(DEV, dtype)
    ref = ref_forward(x, w, nbmaps, nbsizes, n, False)
    out = torch.zeros(n, cout, dtype=dtype, device=DEV)
    ext.sparse_op.convolution_forward_cuda(x, out, w, nbmaps, nbsizes, False, True)     # no_acc: the map's own centre
    eps = 2.0 ** -8 if dtype == torch.bfloat16 else 2.0 ** -11
    assert float(((out.float() - ref).abs() / (ref.abs() + 1e-2)).max()) <= 2 * eps
    # FP32 accumulator out, through the raw kernel
    out32 = torch.empty(n, cout, dtype=torch.float32, device=DEV)
    from jspsr import _lib as L
    starts, _ = ext._offset_starts(nbsizes, 27, DEV)
    table = ext._conv_table(nbmaps, starts, 27, 1, n, -1)
    wt = w.transpose(1, 2).contiguous()
    assert L.load().ngs_conv_tensor_core_ok(cin, cout, ext._conv_dtype(x)) == 1
    err = ext._gather_gemm(x, table, wt, cout, out32)
    assert int(err) == 0
    assert rel(out32, ref) <= 1e-5


@pytest.mark.parametrize("transposed", [False, True])
def test_forward_centre_identity_and_transposed(transposed):
    """The reference's forward takes the centre offset as one dense product over all rows when the kernel
    is odd, the sets agree and no_acc is false; transposed maps read the pairs the other way round."""
    from jspsr import ext
    n, nbmaps, nbsizes = voxel_maps(seed=1)
    gen = torch.Generator(device="cpu").manual_seed(5)
    x = torch.randn(n, 64, generator=gen).to(DEV, torch.bfloat16)
    w = (torch.randn(27, 64, 64, generator=gen) / 8).to(DEV, torch.bfloat16)
    ref = ref_forward(x, w, nbmaps, nbsizes, n, transposed)
    out = torch.zeros(n, 64, dtype=torch.float32, device=DEV)
    ext.sparse_op.convolution_forward_cuda(x, out, w, nbmaps, nbsizes, transposed, False)
    assert rel(out, ref) <= 1e-5


def test_strided_kernel_between_two_sets():
    """A 2^3 kernel from a fine set to a coarse one (the U-Net's down-sampling shape): n_in != n_out."""
    from jspsr import ext
    n, nbmaps_f, _ = voxel_maps(seed=2)
    rng = np.random.default_rng(3)
    n_out = n // 4
    K = 8
    sizes = rng.integers(n // 10, n // 4, size=K)
    maps = np.concatenate([np.stack([rng.integers(0, n, s), rng.integers(0, n_out, s)], 1) for s in sizes]).astype(np.int32)
    # at most one input per (output, offset), as a neighbour map has
    keep, seen, a = [], set(), 0
    for k, s in enumerate(sizes):
        for j in range(a, a + s):
            key = (k, int(maps[j, 1]))
            if key not in seen:
                seen.add(key)
                keep.append(j)
        a += s
    keep = np.array(keep)
    ks = np.repeat(np.arange(K), sizes)[keep]
    nbmaps = torch.tensor(maps[keep], device=DEV)
    nbsizes = torch.tensor(np.bincount(ks, minlength=K), dtype=torch.int32)
    gen = torch.Generator(device="cpu").manual_seed(9)
    x = torch.randn(n, 32, generator=gen).to(DEV, torch.float16)
    w = (torch.randn(K, 32, 64, generator=gen) / 6).to(DEV, torch.float16)
    ref = ref_forward(x, w, nbmaps, nbsizes, n_out, False)
    out = torch.zeros(n_out, 64, dtype=torch.float32, device=DEV)
    ext.sparse_op.convolution_forward_cuda(x, out, w, nbmaps, nbsizes, False, False)
    assert rel(out, ref) <= 1e-5


@pytest.mark.parametrize("dtype,cin,cout", [(torch.bfloat16, 64, 48), (torch.float32, 64, 48),
                                            (torch.bfloat16, 64, 64), (torch.float16, 128, 256),
                                            (torch.bfloat16, 192, 64)])
def test_backward_matches_autograd_of_reference_loop(dtype, cin, cout):
    """Channels in multiples of 64 take the weight gradient's MN-major stages (pair rows copied as
    they are), others the transposing K-major stages; FP32 the CUDA cores."""
    from jspsr.sparse_conv import ConvolutionFunction
    n, nbmaps, nbsizes = voxel_maps(seed=4)
    gen = torch.Generator(device="cpu").manual_seed(11)
    x = torch.randn(n, cin, generator=gen).to(DEV, dtype).requires_grad_(True)
    w = (torch.randn(27, cin, cout, generator=gen) / cin ** 0.5).to(DEV, dtype).requires_grad_(True)
    y = ConvolutionFunction.apply(x, w, nbmaps, nbsizes, (n, n), False, False)
    g = torch.randn(y.shape, generator=gen).to(DEV, dtype)
    gx, gw = torch.autograd.grad(y, (x, w), g)
    xr = x.detach().float().requires_grad_(True)
    wr = w.detach().float().requires_grad_(True)
    yr = ref_forward(xr, wr, nbmaps, nbsizes, n, False)
    gxr, gwr = torch.autograd.grad(yr, (xr, wr), g.float())
    tol = 1e-5 if dtype == torch.float32 else 2.0 ** -7
    assert rel(y, yr) <= tol
    assert rel(gx, gxr) <= tol
    assert rel(gw, gwr) <= tol


def test_fp32_and_unaligned_channels_take_the_cuda_cores():
    from jspsr import ext, _lib as L
    assert L.load().ngs_conv_tensor_core_ok(3, 32, L.NGS_BF16) == 0
    assert L.load().ngs_conv_tensor_core_ok(64, 24, L.NGS_BF16) == 0
    assert L.load().ngs_conv_tensor_core_ok(64, 64, L.NGS_F32) == 0
    n, nbmaps, nbsizes = voxel_maps(seed=6)
    gen = torch.Generator(device="cpu").manual_seed(13)
    for cin, cout, dt in [(3, 32, torch.bfloat16), (64, 24, torch.float16), (16, 16, torch.float32)]:
        x = torch.randn(n, cin, generator=gen).to(DEV, dt)
        w = torch.randn(27, cin, cout, generator=gen).to(DEV, dt)
        out = torch.zeros(n, cout, dtype=torch.float32, device=DEV)
        ext.sparse_op.convolution_forward_cuda(x, out, w, nbmaps, nbsizes, False, True)
        assert rel(out, ref_forward(x, w, nbmaps, nbsizes, n, False)) <= 1e-5


def test_empty_offsets_and_rows_without_pairs():
    """Offsets without pairs cost nothing and rows without any pair come out zero."""
    from jspsr import ext
    n, nbmaps, nbsizes = voxel_maps(seed=7)
    # keep only offsets 0 and 26, so most tiles have two active offsets and some rows none
    starts = np.concatenate([[0], np.cumsum(nbsizes.numpy())])
    keep = np.concatenate([np.arange(starts[0], starts[1]), np.arange(starts[26], starts[27])])
    sizes = torch.zeros(27, dtype=torch.int32)
    sizes[0], sizes[26] = nbsizes[0], nbsizes[26]
    maps = nbmaps[torch.from_numpy(keep).to(DEV)]
    gen = torch.Generator(device="cpu").manual_seed(17)
    x = torch.randn(n, 32, generator=gen).to(DEV, torch.bfloat16)
    w = torch.randn(27, 32, 32, generator=gen).to(DEV, torch.bfloat16)
    out = torch.full((n, 32), 7.0, dtype=torch.float32, device=DEV)
    ext.sparse_op.convolution_forward_cuda(x, out, w, maps, sizes, False, True)     # adds to out
    ref = ref_forward(x, w, maps, sizes, n, False) + 7.0
    assert rel(out, ref) <= 1e-5
