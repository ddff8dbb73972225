"""Generate the Dual Marching Cubes lookup tables used by the extractor.

The extractor must produce the reference's mesh topology bit for bit, so it
needs the reference's DMC case tables (the FlexiCubes tables: per 8-bit
corner-sign case, up to four dual vertices each listing up to seven cube
edges; the number of dual vertices per case; the C16/C19 ambiguity check
table; the tetrahedra table kept for state-dict compatibility).  They are
data, not code: this script reads them from a reference checkout once and
writes two compact encodings:

  atom3d_b200/csrc/dmc_tables.inc            int8 C arrays for the CUDA kernels
  atom3d_b200/mesh_extractor/dmc_tables.py   hex strings decoded into torch tensors

Usage: python tests/golden/gen_dmc_tables.py <path to the reference's
atom3d/mesh_extractor/tables.py>
"""

from __future__ import annotations

import ast
import os
import sys

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "atom3d_b200",
                    "mesh_extractor")


def load(path: str) -> dict:
    tree = ast.parse(open(path).read())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name):
            out[node.targets[0].id] = np.array(ast.literal_eval(node.value), dtype=np.int16)
    return out


def main(path: str) -> None:
    t = load(path)
    shapes = {"dmc_table": (256, 4, 7), "num_vd_table": (256,), "check_table": (256, 5), "tet_table": (256, 6)}
    for k, s in shapes.items():
        assert t[k].shape == s, (k, t[k].shape)
    # check_table's last column holds a case id (0..255): store it as uint8
    lines = ["// Generated by tests/golden/gen_dmc_tables.py -- DMC lookup tables.", "#pragma once", ""]
    # Threads of one warp index these tables with different case ids, so they
    # live in global memory (cached loads) rather than constant memory (one
    # serialised access per distinct address).
    lines.append("// kDmcPacked[c][j]: the up to 7 cube edges of dual vertex j of case c,")
    lines.append("// edge k in bits 4k..4k+3, 0xF = no edge")
    lines.append("__device__ const unsigned int kDmcPacked[256][4] = {")
    for c in range(256):
        words = []
        for j in range(4):
            w = 0
            for k in range(7):
                e = int(t["dmc_table"][c, j, k])
                w |= (0xF if e < 0 else e) << (4 * k)
            words.append(f"0x{w:07x}u")
        lines.append("  {" + ", ".join(words) + "},")
    lines.append("};")
    lines.append("__device__ const unsigned char kNumVd[256] = {" +
                 ", ".join(str(int(x)) for x in t["num_vd_table"]) + "};")
    lines.append("// check: [flag, dx, dy, dz, replacement case]")
    lines.append("__device__ const short kCheck[256][5] = {")
    for c in range(256):
        lines.append("  {" + ", ".join(str(int(x)) for x in t["check_table"][c]) + "},")
    lines.append("};")
    with open(os.path.join(HERE, "..", "csrc", "dmc_tables.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")
    py = ['"""DMC lookup tables (generated by tests/golden/gen_dmc_tables.py; hex-encoded int16 data)."""', "",
          "import numpy as np", "", "_SHAPES = " + repr(shapes), "", "_HEX = {"]
    for k in shapes:
        py.append(f"    {k!r}: {t[k].astype('<i2').tobytes().hex()!r},")
    py += ["}", "", "",
           "def table(name: str) -> np.ndarray:",
           "    return np.frombuffer(bytes.fromhex(_HEX[name]), dtype='<i2').astype(np.int64).reshape(_SHAPES[name])", ""]
    with open(os.path.join(HERE, "dmc_tables.py"), "w") as f:
        f.write("\n".join(py))
    print("tables written")


if __name__ == "__main__":
    main(sys.argv[1])
