"""Regenerate ``mc_tables.inc``: the marching-cubes triangle table as plain data.

The table is the classic Lorensen / Bourke case table (256 cases x 16 edge
indices, -1 terminated).  Mesh topology must match the reference bit for bit,
so the table has to be the identical data; it is taken, numbers only, from the
reference's ``csrc/marching_cubes/mc_data.cuh`` (MIT licence, table originally
published by Paul Bourke).  The edge-crossing mask and the vertex-count table
are *derived* from it in code (``edge_mask`` / ``num_verts`` below and in the
CUDA sources), not copied.

Usage (only needed when the table file is missing):
    python gen_mc_tables.py /path/to/neural-galerkin/csrc/marching_cubes/mc_data.cuh
"""
import re
import sys
from pathlib import Path

OUT = Path(__file__).with_name("mc_tables.inc")


def parse_tri_table(header_text: str):
    start = header_text.index("triangleTable[256][16]")
    body = header_text[start:header_text.index("};", start)]
    nums = [int(x) for x in re.findall(r"-?\d+", body.split("=", 1)[1])]
    assert len(nums) == 256 * 16, len(nums)
    return [nums[i * 16:(i + 1) * 16] for i in range(256)]


def main(src: str):
    rows = parse_tri_table(Path(src).read_text())
    lines = ["/* Marching-cubes triangle table (Lorensen/Bourke), 256 x 16, -1 terminated. Data only.",
             " * Taken as data from huangjh-pub/neural-galerkin csrc/marching_cubes/mc_data.cuh,",
             " * Copyright 2022 Jiahui Huang, Hao-Xiang Chen, Shi-Min Hu, MIT licence (permission notice:",
             " * the LICENSE file of that project); table originally published by Paul Bourke. */"]
    lines += ["{" + ", ".join(f"{v:2d}" for v in r) + "}," for r in rows]
    OUT.write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
