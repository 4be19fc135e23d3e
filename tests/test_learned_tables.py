"""CPU: the learned basis's component integral tables against the reference's symbolic
definitions integrated by adaptive quadrature (``tests/golden/additive_tables.npz``)."""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

from jspsr.bases import tables as T                         # noqa: E402
from jspsr.bases.additive_components import SinPeaks, Power  # noqa: E402

Z = np.load(ROOT / "tests" / "golden" / "additive_tables.npz")
COMPS = [SinPeaks(1), SinPeaks(2), SinPeaks(3)] + [Power(p) for p in range(7)]


def test_component_names_match_reference_cache_names():
    assert [repr(c) for c in COMPS] == [str(n) for n in Z["names"]]


def test_single_component_tables():
    for a, c in enumerate(COMPS):
        f, df, fi, dfi = T.component_tables(c, 5)
        for m in range(5):
            np.testing.assert_allclose(f[m], Z[f"f_{a}_{m}"], atol=1e-10)
            np.testing.assert_allclose(df[m], Z[f"df_{a}_{m}"], atol=1e-10)
        for m in range(1, 5):
            np.testing.assert_allclose(fi[m - 1], Z[f"finv_{a}_{m}"], atol=1e-10)
            np.testing.assert_allclose(dfi[m - 1], Z[f"dfinv_{a}_{m}"], atol=1e-10)


def test_pair_tables():
    for a in (0, 2, 3, 9):
        for b in (1, 2, 5, 9):
            ff, dd = T.component_pair_tables(COMPS[a], COMPS[b], 5)
            for m in range(5):
                np.testing.assert_allclose(ff[m], Z[f"ff_{a}_{b}_{m}"], atol=1e-9)
                np.testing.assert_allclose(dd[m], Z[f"dfdf_{a}_{b}_{m}"], atol=1e-9)
