"""Marching-cubes case tables for the oracle (data file shared with the CUDA build).

TEST INFRASTRUCTURE ONLY.  ``TRI_TABLE`` is read from the data file
``neural-galerkin_b200/csrc/mc_tables.inc`` (the Lorensen/Bourke table, numbers
only); ``EDGE_TABLE`` and ``NUM_VERTS_TABLE`` are derived from the corner sign
pattern and from ``TRI_TABLE``.  The golden script checks all three against the
reference's ``csrc/marching_cubes/mc_data.cuh:38-199``.
"""
import re
from pathlib import Path

import numpy as np

_INC = Path(__file__).resolve().parent.parent / "neural-galerkin_b200" / "csrc" / "mc_tables.inc"
_EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def _load():
    text = _INC.read_text().split("*/", 1)[1]
    nums = [int(x) for x in re.findall(r"-?\d+", text)]
    return np.asarray(nums, dtype=np.int64).reshape(256, 16)


TRI_TABLE = _load()
# Edge e is crossed when its two corners fall on opposite sides of the iso level.
EDGE_TABLE = np.asarray([sum(1 << e for e, (a, b) in enumerate(_EDGES) if ((c >> a) & 1) != ((c >> b) & 1))
                         for c in range(256)], dtype=np.int64)
NUM_VERTS_TABLE = (TRI_TABLE != -1).sum(1)
