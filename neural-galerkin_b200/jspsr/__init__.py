"""jspsr -- sparse screened-Poisson surface reconstruction on NVIDIA B200.

Drop-in for the reconstruction path of neural-galerkin's ``jspsr`` package:
``reconstruct`` keeps the reference's signature (``jspsr/__init__.py:8-61``);
``jspsr.ext`` re-exposes its op modules and ``CuckooHashTable``;
``jspsr.core`` / ``jspsr.bases`` keep its class names.  All compute runs in
hand-written sm_100a kernels (libngs.so); there is no CPU fallback.
"""
from typing import Tuple

__version__ = "1.0.0"
__version_info__ = (1, 0, 0)


def _to_device(a, device):
    """Input -> float32 CUDA tensor; returns (tensor, kind) with kind "cuda", "cpu" (torch) or "numpy"."""
    import numpy as np
    import torch
    if isinstance(a, torch.Tensor):
        kind = "cuda" if a.is_cuda else "cpu"
        return a.to(device=device, dtype=torch.float32, non_blocking=True).contiguous(), kind
    if hasattr(a, "numpy") and not isinstance(a, np.ndarray):     # jittor Var and friends
        a = a.numpy()
    host = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))
    return host.to(device), "numpy"


def reconstruct(xyz, normal, voxel_size: float, depth: int = 4, min_density: float = 32.0,
                screen_alpha: float = 4.0, solver: str = "pcg-mixed@tol=1e-7", n_upsample: int = 2,
                return_reconstruction: bool = False) -> Tuple:
    """Reconstruct a triangle mesh from oriented points.

    :param xyz: (N, 3) float32 positions (numpy array, torch tensor or any object with ``.numpy()``)
    :param normal: (N, 3) float32 normals
    :param voxel_size: size of a voxel at the finest level
    :param depth: number of levels of the tree
    :param min_density: density for determining point layering
    :param screen_alpha: weight of the screening term
    :param solver: per-level linear solver (``"pcg"`` reproduces the reference's FP32 PCG with
        tol 1e-5; the default is FP32 PCG with FP64 dots and FP64 residual replacement)
    :return: vertices (V, 3) float32, triangles (T, 3) int64 -- torch tensors on the inputs'
        device when the inputs were torch tensors (CPU inputs are copied in and the mesh copied
        back), numpy arrays otherwise
    """
    import torch
    from .core.pipeline import Reconstruction

    assert xyz.shape[0] == normal.shape[0] and xyz.shape[1] == normal.shape[1] == 3, \
        "Input positions and normals should have same size (N, 3)!"
    if not torch.cuda.is_available():
        raise RuntimeError("jspsr.reconstruct needs a CUDA device (libngs has no CPU path)")
    dev = torch.device("cuda", torch.cuda.current_device())
    xyz_d, kind = _to_device(xyz, dev)
    nrm_d, _ = _to_device(normal, dev)
    rec = Reconstruction(xyz_d, nrm_d, voxel_size, depth, min_density, screen_alpha, solver=solver)
    v, f = rec.run(n_upsample)
    if kind != "cuda":
        # pinned host buffers: the copies run at DMA speed instead of through a pageable bounce
        vh = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
        fh = torch.empty(f.shape, dtype=f.dtype, pin_memory=True)
        vh.copy_(v, non_blocking=True)
        fh.copy_(f, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        v, f = (vh, fh) if kind == "cpu" else (vh.numpy(), fh.numpy())
    return (v, f, rec) if return_reconstruction else (v, f)
