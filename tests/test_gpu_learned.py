"""Learned-basis (Neural Galerkin) form on the GPU: the reference-API classes (HashTree,
Reconstructor, AdditiveHermite) on libngs, against the reference's own autograd run
(``tests/golden/learned_sq.npz``) and central finite differences."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

pytestmark = pytest.mark.gpu

G = np.load(ROOT / "tests" / "golden" / "learned_sq.npz")
DEPTH = int(G["params"][1])


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def step():
    from jspsr.core.learned import LearnedStep
    dev = torch.device("cuda:0")
    s = LearnedStep(torch.from_numpy(G["xyz"]).to(dev), torch.from_numpy(G["nrm"]).to(dev),
                    torch.from_numpy(G["query"]).to(dev), torch.from_numpy(G["target"]).to(dev),
                    voxel_size=float(G["params"][0]), depth=DEPTH, min_density=float(G["params"][2]),
                    screen_alpha=float(G["params"][3]))
    s.build()
    feats = {d: torch.from_numpy(G[f"feat{d}"]).to(dev) for d in range(DEPTH)}
    loss, gn, gf, chi, rec = s.loss_and_grad(s.normal, feats)
    return s, feats, loss, gn, gf, chi, rec


def test_learned_structure_bit_exact(step):
    s = step[0]
    assert np.array_equal(s.tree.xyz_depth.cpu().numpy(), G["levels"])
    for d in range(DEPTH):
        assert np.array_equal(s.tree.get_coords(s.tree.DECODER, d).cpu().numpy(), G[f"coords{d}"]), d


TOL = 1e-5          # solutions and chi against the reference's run (relative L2)
TOL_GRAD = 1e-4     # gradients against the reference's FP32 autograd (relative L2)


def test_learned_forward_matches_reference(step):
    s, feats, loss, gn, gf, chi, rec = step
    for d in range(DEPTH):
        e = rel(rec.solutions[d].detach().cpu().numpy(), G[f"x{d}"])
        print(f"level {d} solution error {e:.2e}")
        assert e < TOL, d
    e = rel(chi.cpu().numpy(), G["chi"])
    print(f"chi error {e:.2e}")
    assert e < TOL
    assert abs(loss - float(G["loss"])) <= TOL * float(G["loss"])


def test_learned_gradients_match_reference_autograd(step):
    s, feats, loss, gn, gf, chi, rec = step
    e = rel(gn.cpu().numpy(), G["grad_nrm"])
    print(f"normal gradient error {e:.2e}")
    assert e < TOL_GRAD
    for d in range(DEPTH):
        e = rel(gf[d].cpu().numpy(), G[f"grad_feat{d}"])
        print(f"level {d} feature gradient error {e:.2e}")
        assert e < TOL_GRAD, d


def test_learned_batch_equals_single_shapes(step):
    """The batched form (all shapes through one GalerkinSolve, level solves batched) gives every
    shape the loss and gradients of its own single-shape run."""
    from jspsr.core.learned import LearnedBatch, LearnedStep
    from jspsr import synthetic
    s0 = step[0]
    dev = s0.xyz.device
    steps = []
    for seed in range(3):
        xyz, nrm, q, tgt = synthetic.learned_problem(n=2000, n_query=5000, seed=seed)
        T = lambda a: torch.from_numpy(a).to(dev)          # noqa: E731
        steps.append(LearnedStep(T(xyz), T(nrm), T(q), T(tgt), min_density=None).build())
    feats = [st.init_features(0.1, seed=k) for k, st in enumerate(steps)]
    singles = [st.loss_and_grad(st.normal, f) for st, f in zip(steps, feats)]
    batch = LearnedBatch(steps)
    normals = [st.normal.detach().clone().requires_grad_(True) for st in steps]
    fl = [{d: v.detach().clone().requires_grad_(True) for d, v in f.items()} for f in feats]
    total, losses, _ = batch.forward(normals, fl)
    total.backward()
    # the same systems and solves (a batched solve is bit-identical to a solo one); the FP32 scatter
    # sums of the assembly run on atomics, whose order varies, hence a 1e-5 tolerance
    for k, (loss, gn, gf, _, _) in enumerate(singles):
        assert abs(float(losses[k]) - loss) <= 1e-5 * loss, k
        assert rel(normals[k].grad.cpu().numpy(), gn.cpu().numpy()) < 1e-5, k
        for d in gf:
            assert rel(fl[k][d].grad.cpu().numpy(), gf[d].cpu().numpy()) < 1e-5, (k, d)


def _loss64(s, normal, feats):
    with torch.no_grad():
        chi = s.forward(normal, feats)[1].double()
    # the loss reduction in FP64 so that the difference quotient resolves 2h * grad
    return float(torch.mean((chi - s.target.double()) ** 2))


def _central_fd(s, normal, feats, which, direction, h=1e-3):
    """(L(theta + h v) - L(theta - h v)) / 2h for the direction v on one input."""
    def shifted(sign):
        n = normal.clone()
        f = {d: v.clone() for d, v in feats.items()}
        if which == "normal":
            n += sign * h * direction
        else:
            f[which] += sign * h * direction
        return _loss64(s, n, f)
    return (shifted(1.0) - shifted(-1.0)) / (2 * h)


def test_learned_gradients_match_central_differences_coordinates(step):
    """Central differences, h = 1e-3, on the ten normal coordinates with the largest gradients."""
    s, feats, loss, gn, gf, chi, rec = step
    flat = gn.reshape(-1)
    for idx in torch.topk(flat.abs(), 10).indices.tolist():
        e = torch.zeros_like(flat)
        e[idx] = 1.0
        fd = _central_fd(s, s.normal, feats, "normal", e.view_as(gn))
        an = float(flat[idx])
        assert abs(fd - an) <= 2e-2 * abs(an), (idx, fd, an)


def test_learned_gradients_match_central_differences_directional(step):
    """Central differences, h = 1e-3, along v = g / max|g| (all coordinates of one input at once:
    a single feature's loss change is below the FP32 assembly's rounding floor)."""
    s, feats, loss, gn, gf, chi, rec = step
    gen = torch.Generator(device="cpu").manual_seed(5)
    for which, g in [("normal", gn)] + [(d, gf[d]) for d in range(DEPTH)]:
        v = g / g.abs().max()
        noise = torch.randn(g.shape, generator=gen).to(g.device) * 0.1
        v = v + noise * (v.abs() > 0).float()
        fd = _central_fd(s, s.normal, feats, which, v)
        an = float(torch.sum(g.double() * v.double()))
        assert abs(fd - an) <= 2e-2 * abs(an), (which, fd, an)
