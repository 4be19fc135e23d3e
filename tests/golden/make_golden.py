"""Generate golden vectors by running the reference's own Python layer on CPU.

The reference (huangjh-pub/neural-galerkin) cannot run as shipped here: its
ops are CUDA-only pybind11 modules, and ``jittor``, ``torch_scatter`` and
``omegaconf`` are absent.  This script therefore

1. copies the reference's ``jspsr`` package to a temporary directory and adds
   the two data files the reference never published (``kernel.npz`` and
   ``bezier_integrals.pkl``), re-derived by the oracle;
2. installs stand-ins for the absent pieces: ``jittor`` (type names and
   ``jt.array`` only), ``torch_scatter`` (index_add), ``omegaconf`` (a dict),
   and the five compiled op modules, whose functions are the oracle's CPU
   restatements of the CUDA ops (``oracle/ops.py``); the linear solves use an
   exact FP64 solve so that the fixtures pin assembly, not solver tolerance;
3. runs the reference's unmodified ``jspsr.reconstruct`` (and its
   ``AdditiveBasis`` sympy integrals) and records inputs, intermediates and
   outputs into small ``.npz`` fixtures beside this script.

Everything the reference computes in torch (trilinear weights, quantisation,
neighbour queries, density, levels, RHS / LHS assembly, correction, chi,
conformal tree, dual-grid construction, vertex de-duplication) is the
reference's own code.  The learned-basis case also writes the reference's additive-integral cache files (which it
would otherwise compute with sympy) from its own symbolic components.  Run from the
repository root, with the reference checkout named by ``NGS_REFERENCE_DIR``
(``python tests/golden/make_golden.py [tables|learned|<case>...]``):

    NGS_REFERENCE_DIR=/path/to/neural-galerkin python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import pickle
import shutil
import sys
import tempfile
import types
from pathlib import Path

import numpy as np
import torch

# the reference checkout (huangjh-pub/neural-galerkin), named by NGS_REFERENCE_DIR
REF = Path(os.environ.get("NGS_REFERENCE_DIR", "../neural-galerkin")).resolve()
HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import ops as O            # noqa: E402
from oracle import spsr as S           # noqa: E402
from oracle import tables as T         # noqa: E402


def _load_synthetic():
    """The workload generators of this repository, loaded without claiming the name ``jspsr``."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "ngs_synthetic", ROOT / "neural-galerkin_b200" / "jspsr" / "synthetic.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


synthetic = _load_synthetic()

CASES = {
    # name: (generator, voxel_size, depth, min_density, screen_alpha)
    "torus_small": (lambda: synthetic.torus(n=3000, seed=0), 1.0 / 64, 3, 0.5, 4.0),
    "torus_adaptive": (lambda: synthetic.torus(n=10000, seed=0), 1.0 / 128, 3, 1.5, 4.0),
    "sq_noisy": (lambda: synthetic.superquadrics(n=4000, k=2, seed=3, normal_noise=0.02, pos_noise=0.002)[:2],
                 1.0 / 128, 3, 0.35, 4.0),
}


# ----------------------------------------------------------------------------- stand-ins
def _t(x, dtype=None):
    a = np.asarray(x)
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.to(dtype) if dtype is not None else t


class _Handle:
    def __init__(self, table):
        self.table = table
        self.inserted_size = table.inserted_size


def _install_stubs(pkgdir: Path):
    jt = types.ModuleType("jittor")
    jt.Var = torch.Tensor
    jt.array = lambda a: np.asarray(a)
    sys.modules["jittor"] = jt

    ts = types.ModuleType("torch_scatter")

    def scatter_sum(src, index, dim=0, dim_size=None, out=None):
        if out is None:
            size = list(src.shape)
            size[0] = int(dim_size if dim_size is not None else (int(index.max()) + 1 if index.numel() else 0))
            out = torch.zeros(size, dtype=src.dtype)
        return out.index_add_(0, index.long(), src)
    ts.scatter_sum = scatter_sum
    ts.scatter_add = scatter_sum
    ts.scatter = scatter_sum
    sys.modules["torch_scatter"] = ts

    oc = types.ModuleType("omegaconf")
    oc.OmegaConf = types.SimpleNamespace(create=lambda *a: {})
    sys.modules["omegaconf"] = oc

    common = types.ModuleType("jspsr._common")
    common.hash_cuda = lambda idx: _t(O.hash_cuda(idx.numpy()))
    common.kernel_hash_cuda = lambda idx, off: _t(O.kernel_hash_cuda(idx.numpy(), off.numpy()))
    common.build_hash_table = lambda keys, vals, enlarge: _Handle(O.build_hash_table(keys.numpy(), vals.numpy()))
    common.hash_table_query = lambda h, q: _t(h.table.query(q.numpy()))

    sop = types.ModuleType("jspsr._sparse_op")
    sop.screened_multiplication = lambda h, av, bv, ai, bi, al, bl, w: _t(
        O.screened_multiplication(h.table, av.numpy(), bv.numpy(), ai.numpy(), bi.numpy(), al.numpy(),
                                  bl.numpy(), w.numpy()), torch.float32)

    def smb(h, av, bv, ai, bi, al, bl, w, g):
        ga, gb, gw = O.screened_multiplication_backward(h.table, av.numpy(), bv.numpy(), ai.numpy(), bi.numpy(),
                                                        al.numpy(), bl.numpy(), w.numpy(), g.numpy())
        return [_t(ga, torch.float32), _t(gb, torch.float32), _t(gw, torch.float32)]
    sop.screened_multiplication_backward = smb
    sop.sparse_meshgrid = lambda a, b: tuple(_t(x) for x in O.sparse_meshgrid(a.numpy(), b.numpy()))

    integ = types.ModuleType("jspsr._integration")

    def ddi_f(s, t, r, ff, dd):
        p, q = O.ddi_forward(s.detach().numpy(), t.detach().numpy(), r.numpy(), ff.numpy(), dd.numpy())
        return _t(p, torch.float32), _t(q, torch.float32)

    def ddi_b(s, t, r, ff, dd, gp, gq):
        a, b = O.ddi_backward(s.numpy(), t.numpy(), r.numpy(), ff.numpy(), dd.numpy(), gp.numpy(), gq.numpy())
        return _t(a, torch.float32), _t(b, torch.float32)
    integ.ddi_forward, integ.ddi_backward = ddi_f, ddi_b

    solve = types.ModuleType("jspsr._sparse_solve")
    solve.init_cusolver = lambda: None

    def exact(ap, aj, ax, b, *args):
        import scipy.sparse as sps
        import scipy.sparse.linalg as spla
        n = b.shape[0]
        a = sps.csr_matrix((ax.numpy().astype(np.float64), aj.numpy(), ap.numpy()), shape=(n, n))
        x = spla.spsolve(a.tocsc(), b.numpy().astype(np.float64)) if n < 3000 else S._cg64(a, b.numpy().astype(np.float64))
        return _t(x, torch.float32)
    solve.solve_pcg_diag = lambda ap, aj, ax, b, dinv, tol, mi, rf: (exact(ap, aj, ax, b), 0)
    solve.solve_cusparse = lambda ap, aj, ax, b, tol: exact(ap, aj, ax, b)

    mc = types.ModuleType("jspsr._marching_cubes")

    def dmi(h, epb, strides, bases):
        acc, cnt = O.dual_marching_cubes_indices(h.table, {k: v.numpy() for k, v in epb.items()}, strides, bases)
        return [_t(acc), _t(cnt)]

    def dms(acc, pos, val):
        tris, vids = O.dual_marching_cubes_sparse(acc.numpy(), pos.numpy(), val.numpy())
        return [_t(tris), _t(vids)]

    def pms(base, sdf):
        return [_t(x) for x in O.marching_cubes_sparse(base.numpy(), sdf.numpy())]
    mc.dual_marching_cubes_indices, mc.dual_marching_cubes_sparse, mc.marching_cubes_sparse = dmi, dms, pms

    for name, mod in [("_common", common), ("_sparse_op", sop), ("_integration", integ),
                      ("_sparse_solve", solve), ("_marching_cubes", mc)]:
        sys.modules[f"jspsr.{name}"] = mod
    torch.Tensor.cuda = lambda self, *a, **k: self


def _prepare_reference() -> Path:
    tmp = Path(tempfile.mkdtemp(prefix="jspsr_ref_"))
    shutil.copytree(REF / "jspsr", tmp / "jspsr")
    data = tmp / "jspsr" / "data"
    data.mkdir(exist_ok=True)
    np.savez(data / "kernel.npz", kernel=S.range_kernel(9))
    tabs = T.bezier_tables(5)
    with open(data / "bezier_integrals.pkl", "wb") as f:
        pickle.dump([[list(map(float, t)) for t in tabs[k]] for k in T.BEZIER_PICKLE_ORDER], f)
    os.environ["HOME"] = str(tmp / "home")
    sys.path.insert(0, str(tmp))
    _install_stubs(tmp / "jspsr")
    return tmp


# ----------------------------------------------------------------------------- capture
def run_case(name, gen, vs, depth, md, alpha):
    import jspsr as ref_jspsr
    from jspsr.core import reconstructor as R
    assert Path(ref_jspsr.__file__).resolve().parts[1] in ("tmp",), ref_jspsr.__file__

    captured = {}
    orig_extract = R.Reconstructor.extract_multiscale_mesh
    orig_solve = R.Reconstructor.solve_multigrid

    def extract(self, *a, **k):
        captured["rec"] = self
        return orig_extract(self, *a, **k)

    lhs_cap = {}
    import jspsr.core.reconstructor as RM
    orig_ss = RM.solve_sparse

    def solve_sparse(src, tgt, lhs, rhs, solver):
        d = len(lhs_cap)
        n = rhs.shape[0]
        probe = torch.from_numpy(np.random.default_rng(100 + d).standard_normal(n).astype(np.float32))
        av = torch.zeros(n).index_add_(0, src, probe[tgt] * lhs)
        lhs_cap[d] = dict(rhs=rhs.detach().numpy().copy(), av=av.numpy().copy(), probe=probe.numpy(),
                          nnz=int(lhs.shape[0]), diag=torch.zeros(n).index_add_(0, src[src == tgt], lhs[src == tgt]).numpy())
        return orig_ss(src, tgt, lhs, rhs, solver)
    RM.solve_sparse = solve_sparse
    R.Reconstructor.extract_multiscale_mesh = extract
    try:
        xyz, nrm = gen()
        v, f = ref_jspsr.reconstruct(torch.from_numpy(xyz), torch.from_numpy(nrm), vs, depth=depth,
                                     min_density=md, screen_alpha=alpha)
    finally:
        R.Reconstructor.extract_multiscale_mesh = orig_extract
        RM.solve_sparse = orig_ss
    rec = captured["rec"]
    ht = rec.hash_tree
    out = dict(xyz=xyz, nrm=nrm, params=np.array([vs, depth, md, alpha]),
               density=ht.xyz_density.numpy(), levels=ht.xyz_depth.numpy(),
               vertices=np.asarray(v, dtype=np.float32), faces=np.asarray(f, dtype=np.int64))
    for d in range(depth):
        out[f"coords{d}"] = ht.get_coords(ht.DECODER, d).numpy()
        out[f"x{d}"] = rec.solutions[d].detach().numpy()
    # solve order is coarse -> fine: capture index i corresponds to level depth-1-i
    for i, cap in lhs_cap.items():
        d = depth - 1 - i
        for k, val in cap.items():
            out[f"lhs{d}_{k}"] = np.asarray(val)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, {k: np.asarray(v).shape for k, v in out.items() if k.startswith(("coords", "faces", "vertices"))})


def tables_case():
    """Pin the re-derived Bezier tables against the reference's own basis definition.

    The reference computes its tables with sympy (``additive.py:17-52``); sympy's
    piecewise integration does not finish here for shifted intervals, so the
    reference's symbolic ``Bezier`` (``additive_components.py:102-113``) is
    lambdified and integrated with adaptive quadrature (scipy ``quad``) over the
    same intervals and index conventions as ``_integrate_ff`` / ``_integrate_f`` /
    ``_integrate_f_inv``.
    """
    from jspsr.bases import additive_components as AC
    import sympy as sp
    from scipy.integrate import quad
    x = sp.Symbol("x")
    sym = AC.Bezier().symbolic(x)
    f = sp.lambdify(x, sym, "math")
    df = sp.lambdify(x, sp.diff(sym, x), "math")
    brk = [-1.5, -0.5, 0.5, 1.5]

    def integ(fn, lo, hi, pts):
        pts = sorted(p for p in set(pts) if lo < p < hi)
        return quad(fn, lo, hi, points=pts or None, limit=200, epsabs=1e-14, epsrel=1e-14)[0]
    out = {}
    for m in range(3):
        M = 2 ** m
        ff, dd = [], []
        for dx in np.arange(-1.5 * M - 0.5, 1.5 * M + 1.5):
            pts = [b - dx for b in brk] + [b * M for b in brk]
            lo, hi = -1.5 * M - 4 - abs(dx), 1.5 * M + 4 + abs(dx)
            ff.append(integ(lambda y: f(y + dx) * f(y / M), lo, hi, pts))
            dd.append(integ(lambda y: df(y + dx) * df(y / M) / M, lo, hi, pts))
        out[f"ff{m}"], out[f"dfdf{m}"] = np.array(ff), np.array(dd)
        fv, dfv = [], []
        for ra in np.arange(-1.5 * M, 1.5 * M):
            fv.insert(0, integ(lambda y: f(y / M), ra, ra + 1, [b * M for b in brk]))
            dfv.insert(0, integ(lambda y: df(y / M) / M, ra, ra + 1, [b * M for b in brk]))
        out[f"f{m}"], out[f"df{m}"] = np.array(fv), np.array(dfv)
        if m >= 1:
            fv, dfv = [], []
            for ra in np.arange(-(2 ** m) - 0.5, 1.5):
                lb, ub = max(ra, -1.5), min(ra + M, 1.5)
                fv.insert(0, integ(f, lb, ub, brk) if ub > lb else 0.0)
                dfv.insert(0, integ(df, lb, ub, brk) if ub > lb else 0.0)
            out[f"finv{m}"], out[f"dfinv{m}"] = np.array(fv), np.array(dfv)
    np.savez_compressed(HERE / "bezier_tables.npz", **out)
    print("tables", sorted(out))


def mc_tables_case():
    """The reference's marching-cubes tables, to pin the derived edge / vertex-count tables."""
    import re
    txt = (REF / "csrc" / "marching_cubes" / "mc_data.cuh").read_text()

    def arr(name, n):
        s = txt.index(name)
        body = txt[s:txt.index("};", s)].split("=", 1)[1]
        return np.array([int(v, 0) for v in re.findall(r"-?0x[0-9a-fA-F]+|-?\d+", body)][:n])
    np.savez_compressed(HERE / "mc_tables.npz", edge=arr("edgeTable[256]", 256),
                        numverts=arr("numVertsTable[256]", 256), tri=arr("triangleTable[256][16]", 4096))


def range_kernel_case():
    """Pin the FNV keys the reference's kernel_hash path produces for a few coords (known answers)."""
    coords = np.array([[0, 0, 0], [1, 2, 3], [-1, -2, -3], [1023, -4096, 77], [2 ** 20, 5, -(2 ** 20)]], np.int32)
    np.savez_compressed(HERE / "fnv_keys.npz", coords=coords, keys=O.hash_cuda(coords),
                        keys4=O.hash_cuda(np.concatenate([coords, coords[:, :1]], 1)))


LEARNED = dict(seed=0, voxel_size=1.0 / 128, depth=3, min_density=2.0, screen_alpha=4.0, feat_sigma=0.1)


def _learned_components():
    """The learned basis of ``configs/shapenet/full_net_base.yaml:54-59`` as the reference builds it."""
    from jspsr.bases import additive_components as AC
    comps = [AC.SinPeaks(1), AC.SinPeaks(2), AC.SinPeaks(3)]
    return comps + [AC.Power(p) for p in range(7)]


def additive_tables_case(n_mult: int = 5):
    """theta / rho tables of the learned basis's ten components from the reference's symbolic
    definitions (``additive.py:17-52``), integrated with adaptive quadrature, written as the
    reference's own cache files (``additive.py:178-246``) and as a fixture.

    sympy's piecewise integration of these products does not finish here, so the reference's
    symbolic components are lambdified and integrated with scipy ``quad`` over the same intervals
    and index conventions."""
    import sympy as sp
    from scipy.integrate import quad
    import jspsr
    comps = _learned_components()
    x = sp.Symbol("x")
    fs = [sp.lambdify(x, c.symbolic(x), "math") for c in comps]
    dfs = [sp.lambdify(x, sp.diff(c.symbolic(x), x), "math") for c in comps]
    brk = [-1.5, 1.5]

    def integ(fn, lo, hi, pts):
        if hi <= lo:
            return 0.0
        pts = sorted(p for p in set(pts) if lo < p < hi)
        return quad(fn, lo, hi, points=pts or None, limit=200, epsabs=1e-14, epsrel=1e-13)[0]

    def objarr(lists):
        a = np.empty(len(lists), dtype=object)
        for i, v in enumerate(lists):
            a[i] = [float(t) for t in v]
        return a

    cache = Path(jspsr.__file__).parent / "data" / "additive_integrals"
    cache.mkdir(parents=True, exist_ok=True)
    fixture = {}
    C = len(comps)
    for a in range(C):
        for b in range(C):
            ff, dd = [], []
            for m in range(n_mult):
                M = 2 ** m
                rf, rd = [], []
                for dx in np.arange(-1.5 * M - 0.5, 1.5 * M + 1.5):
                    lo, hi = max(-1.5 - dx, -1.5 * M), min(1.5 - dx, 1.5 * M)
                    pts = [q - dx for q in brk] + [q * M for q in brk] + [0.0]
                    rf.append(integ(lambda y: fs[a](y + dx) * fs[b](y / M), lo, hi, pts))
                    rd.append(integ(lambda y: dfs[a](y + dx) * dfs[b](y / M) / M, lo, hi, pts))
                ff.append(rf)
                dd.append(rd)
                fixture[f"ff_{a}_{b}_{m}"] = np.asarray(rf)
                fixture[f"dfdf_{a}_{b}_{m}"] = np.asarray(rd)
            np.savez_compressed(cache / f"ff-{comps[a]}-{comps[b]}.npz", f_f=objarr(ff), df_df=objarr(dd))
    for a in range(C):
        f, df, fi, dfi = [], [], [], []
        for m in range(n_mult):
            M = 2 ** m
            rf, rd = [], []
            for ra in np.arange(-1.5 * M, 1.5 * M):
                rf.insert(0, integ(lambda y: fs[a](y / M), ra, ra + 1, [q * M for q in brk]))
                rd.insert(0, integ(lambda y: dfs[a](y / M) / M, ra, ra + 1, [q * M for q in brk]))
            f.append(rf)
            df.append(rd)
            fixture[f"f_{a}_{m}"], fixture[f"df_{a}_{m}"] = np.asarray(rf), np.asarray(rd)
        for m in range(1, n_mult):
            M = 2 ** m
            rf, rd = [], []
            for ra in np.arange(-M - 0.5, 1.5):
                lb, ub = max(ra, -1.5), min(ra + M, 1.5)
                rf.insert(0, integ(fs[a], lb, ub, brk))
                rd.insert(0, integ(dfs[a], lb, ub, brk))
            fi.append(rf)
            dfi.append(rd)
            fixture[f"finv_{a}_{m}"], fixture[f"dfinv_{a}_{m}"] = np.asarray(rf), np.asarray(rd)
        np.savez_compressed(cache / f"f-{comps[a]}.npz", f=objarr(f), df=objarr(df), f_inv=objarr(fi),
                            df_inv=objarr(dfi))
    fixture["names"] = np.array([repr(c) for c in comps])
    np.savez_compressed(HERE / "additive_tables.npz", **fixture)
    print("additive tables", len(fixture))


def learned_case():
    """The Neural Galerkin training form on the reference's own classes: AdditiveHermite basis with
    per-voxel features (Bezier-like initialisation + N(0, 0.1)), density-adaptive tree, normals
    splatted as ``jspsr/__init__.py:36-47`` does, multigrid solve with screening, loss = MSE of
    ``evaluate_chi`` at query points against an analytic target; gradients by the reference's
    autograd graph (its DDIFunc / EvalFunc / ScreenedMultiplication / Solver backward)."""
    from jspsr.core.hashtree import HashTree
    from jspsr.core.reconstructor import Reconstructor
    from jspsr.bases.hermite_ns import AdditiveHermite
    from jspsr.bases import additive_components as AC
    P = LEARNED
    xyz, nrm, q, target = synthetic.learned_problem(seed=P["seed"])
    xyz_t = torch.from_numpy(xyz)
    nrm_t = torch.from_numpy(nrm).requires_grad_(True)
    basis = AdditiveHermite(6, [AC.SinPeaks(1), AC.SinPeaks(2), AC.SinPeaks(3)], [0.0, 0.0, 0.0])
    ht = HashTree(xyz_t, voxel_size=P["voxel_size"], depth=P["depth"])
    ht.build_encoder_hierarchy_adaptive(min_density=P["min_density"])
    ht.reflect_decoder_coords()
    sw = 1.0 / ht.xyz_density
    normal_data = {}
    for d in range(ht.depth):
        msk = ht.xyz_depth == d
        if not torch.any(msk):
            continue
        nd = ht.splat_data(xyz_t[msk], ht.DECODER, d, nrm_t[msk] * sw[msk, None])
        normal_data[d] = nd / (ht.get_stride(ht.DECODER, d) ** 3)
    rng = np.random.default_rng(P["seed"] + 7)
    feats = {}
    for d in range(ht.depth):
        f0 = torch.zeros((ht.get_coords_size(ht.DECODER, d), basis.get_feature_size()))
        basis.initialize_feature_value(f0)
        f0 = f0 + torch.from_numpy(rng.normal(0, P["feat_sigma"], f0.shape).astype(np.float32))
        feats[d] = f0.requires_grad_(True)
    rec = Reconstructor(ht, basis, feats)
    rec.sample_weight = sw
    rec.solve_multigrid(ht.depth - 1, 0, normal_data, screen_alpha=P["screen_alpha"], screen_xyz=xyz_t,
                        solver="cholmod", verbose=False)
    chi = rec.evaluate_chi(torch.from_numpy(q))
    loss = torch.mean((chi - torch.from_numpy(target)) ** 2)
    loss.backward()
    out = dict(xyz=xyz, nrm=nrm, query=q, target=target,
               params=np.array([P["voxel_size"], P["depth"], P["min_density"], P["screen_alpha"]]),
               density=ht.xyz_density.numpy(), levels=ht.xyz_depth.numpy(), chi=chi.detach().numpy(),
               loss=np.array(float(loss)), grad_nrm=nrm_t.grad.numpy())
    for d in range(ht.depth):
        out[f"coords{d}"] = ht.get_coords(ht.DECODER, d).numpy()
        out[f"feat{d}"] = feats[d].detach().numpy()
        out[f"grad_feat{d}"] = feats[d].grad.numpy()
        out[f"x{d}"] = rec.solutions[d].detach().numpy()
    np.savez_compressed(HERE / "learned_sq.npz", **out)
    print("learned", float(loss), {k: v.shape for k, v in out.items() if k.startswith(("coords", "grad"))})


def _count_policy(xyz, inds, min_count=6):
    """Test subdivision policy: keep subdividing the cells that hold at least min_count points."""
    counts = torch.bincount(inds)
    return counts[inds] >= min_count


def structure_case():
    """The hierarchy builders and queries beside the density-adaptive one (``hashtree.py:240-312``,
    ``_hash_backend.py:292-412``): dense hierarchy, subdivision by a policy, voxel status,
    expanded / conforming coordinates, test grid and trilinear split of voxel data."""
    from jspsr.core.hashtree import HashTree
    xyz, nrm = synthetic.torus(n=3000, seed=1)
    xyz_t = torch.from_numpy(xyz)
    out = dict(xyz=xyz)
    dense = HashTree(xyz_t, voxel_size=1.0 / 64, depth=3)
    dense.build_encoder_hierarchy_dense(expand_range=3)
    dense.reflect_decoder_coords()
    out["dense_density"] = dense.xyz_density.numpy()
    rng = np.random.default_rng(5)
    for d in range(3):
        c = dense.get_coords(dense.ENCODER, d)
        out[f"dense{d}"] = c.numpy()
        s = dense.get_stride(dense.ENCODER, d)
        probe = torch.cat([c[::7], c[::11] + s, torch.from_numpy(rng.integers(-40, 40, (64, 3)).astype(np.int32)) * s])
        out[f"probe{d}"] = probe.numpy()
        out[f"status{d}"] = dense.evaluate_voxel_status(dense.ENCODER, probe, d).numpy()
        out[f"expand{d}"] = dense._enc_branch.get_coords(d, expand=3).numpy()
        out[f"conform{d}"] = dense._enc_branch.get_coords(d, conforming=True).numpy()
        data = torch.from_numpy(rng.normal(size=(c.shape[0], 2)).astype(np.float32))
        out[f"data{d}"] = data.numpy()
        out[f"split{d}"] = dense.split_data(xyz_t, dense.ENCODER, d, data).numpy()
    q, base = dense.get_test_grid(3, 1, expand=0, conforming=False)
    out["test_grid_pos"], out["test_grid_base"] = q.numpy(), base.numpy()
    sub = HashTree(xyz_t, voxel_size=1.0 / 64, depth=3)
    sub.build_hierarchy_subdivide(_count_policy, expand=True, min_count=6)
    out["sub_depth"] = sub.xyz_depth.numpy()
    for d in range(3):
        out[f"sub{d}"] = sub.get_coords(sub.ENCODER, d).numpy()
    np.savez_compressed(HERE / "structure.npz", **out)
    print("structure", {k: v.shape for k, v in out.items() if k.startswith(("dense", "sub", "status"))})


def main():
    _prepare_reference()
    names = sys.argv[1:]
    if not names or "tables" in names:
        tables_case()
        mc_tables_case()
        range_kernel_case()
    if not names or "structure" in names:
        structure_case()
    if not names or "learned" in names:
        additive_tables_case()
        learned_case()
    for n in names or list(CASES):
        if n in CASES:
            run_case(n, *CASES[n])


if __name__ == "__main__":
    main()
