"""CPU-side checks of the native library: it loads and exports every symbol include/ngs.h declares."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "ngs.h").read_text()
    return sorted(set(re.findall(r"\b(ngs_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    from jspsr import _lib
    lib = _lib.load()
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    from jspsr import _lib
    assert set(header_symbols()) == set(_lib.exported_symbols())


def header_arities():
    """Number of parameters of every function the header declares (comments stripped)."""
    text = (ROOT / "include" / "ngs.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for m in re.finditer(r"\b(ngs_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_binding_arities_match_header():
    """The ctypes prototypes take as many arguments as the C declarations (an ABI change that the
    binding missed would pass garbage silently)."""
    from jspsr import _lib
    arity = header_arities()
    wrong = {name: (len(sig[0]), arity[name]) for name, sig in _lib._SIGS.items()
             if name in arity and len(sig[0]) != arity[name]}
    assert not wrong, wrong
    unchecked = set(_lib._SIGS) - set(arity)
    assert not unchecked, unchecked


def test_status_strings():
    from jspsr import _lib
    lib = _lib.load()
    assert lib.ngs_status_string(0) == b"ok"
    assert b"tolerance" in lib.ngs_status_string(4)
    assert lib.ngs_version() >= 10000


def test_solver_spec_grammar():
    from jspsr.core.pipeline import parse_solver
    s = parse_solver("pcg@tol=1e-7@maxiter=300")
    assert (s.name, s.tol, s.maxiter) == ("pcg", 1e-7, 300)
    s = parse_solver("pcg")
    assert (s.tol, s.maxiter) == (1e-5, -1)
    s = parse_solver("pcg-mixed@tol=1e-9@replace=25")
    assert (s.mode, s.tol, s.replace) == (1, 1e-9, 25)
    with pytest.raises(ValueError):
        parse_solver("pcg@tol=__import__('os')")
    with pytest.raises(NotImplementedError):
        parse_solver("cg-magic")


def test_product_tables_match_oracle():
    import numpy as np
    from jspsr.bases import tables as P
    from oracle import tables as T
    t = T.bezier_tables(5)
    for m in range(5):
        M = 2 ** m
        s, d = P.shifted(m)
        np.testing.assert_allclose(s, t["SHIFTED_SELF_INTEGRAL"][m], rtol=1e-10, atol=1e-11)
        np.testing.assert_allclose(d, t["SHIFTED_DERIVATIVE_INTEGRAL"][m], rtol=1e-10, atol=1e-11)
        f, g = P.partial(m)
        np.testing.assert_allclose(f, t["DERIVATIVE_PARTIAL_INTEGRAL"][m], atol=1e-11)
        np.testing.assert_allclose(g, t["PARTIAL_INTEGRAL"][m], atol=1e-11)
        if m:
            f, g = P.inverse_partial(m)
            np.testing.assert_allclose(f, t["INV_DERIVATIVE_PARTIAL_INTEGRAL"][m - 1], atol=1e-11)
            np.testing.assert_allclose(g, t["INV_PARTIAL_INTEGRAL"][m - 1], atol=1e-11)


def test_product_tables_beyond_reference_ratios():
    """Level ratios 32 .. 1024 (m = 5 .. 10), outside the reference's tables (n_multiples = 5), used by
    hierarchies deeper than 5 levels: every entry against the oracle's piecewise Gauss-Legendre
    quadrature (exact for the polynomial pieces), relative to the entry itself.  The smallest
    entries at m = 10 are ~3e-8 while the integration range spans 1.5 * 1024 voxels."""
    import numpy as np
    from jspsr.bases import tables as P
    from oracle import tables as T
    t = T.bezier_tables(11)
    for m in range(5, 11):
        s, d = P.shifted(m)
        np.testing.assert_allclose(s, t["SHIFTED_SELF_INTEGRAL"][m], rtol=1e-11, atol=1e-22, err_msg=f"m={m}")
        np.testing.assert_allclose(d, t["SHIFTED_DERIVATIVE_INTEGRAL"][m], rtol=1e-11, atol=1e-14, err_msg=f"m={m}")
        f, g = P.partial(m)
        np.testing.assert_allclose(f, t["DERIVATIVE_PARTIAL_INTEGRAL"][m], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(g, t["PARTIAL_INTEGRAL"][m], rtol=1e-11, atol=1e-14)
        f, g = P.inverse_partial(m)
        np.testing.assert_allclose(f, t["INV_DERIVATIVE_PARTIAL_INTEGRAL"][m - 1], atol=1e-14)
        np.testing.assert_allclose(g, t["INV_PARTIAL_INTEGRAL"][m - 1], atol=1e-14)


def test_stencil_is_symmetric_and_annihilates_nothing():
    import numpy as np
    from jspsr.bases import tables as P
    st = P.stencil125(1).reshape(5, 5, 5)
    np.testing.assert_allclose(st, st[::-1, ::-1, ::-1], atol=1e-14)
    assert st[2, 2, 2] > 0
    # the stiffness annihilates constants on a full lattice: its stencil sums to zero
    assert abs(st.sum()) < 1e-12


def test_ctypes_structures_match_the_header_layout(tmp_path):
    """Every structure the Python side passes through the C ABI has the header's size and field
    offsets: a C program built from include/ngs.h prints them, the ctypes mirrors are compared."""
    import ctypes
    import shutil
    import subprocess
    import sys
    sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))
    from jspsr import _lib as L
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"ngs_grid": L.Grid, "ngs_hash_table": L.HashTable, "ngs_pcg_operator": L.PcgOperator,
               "ngs_pcg_system": L.PcgSystem, "ngs_pcg_config": L.PcgConfig, "ngs_pcg_batch_item": L.PcgBatchItem}
    lines = ['#include <stdio.h>', '#include "ngs.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    want = {}
    for line in filter(None, out):
        cname, field, value = line.split()
        want[(cname, field)] = int(value)
    for cname, py in mirrors.items():
        assert ctypes.sizeof(py) == want[(cname, "size")], cname
        for fname, _ in py._fields_:
            assert getattr(py, fname).offset == want[(cname, fname)], (cname, fname)
