"""Cube topology conventions shared with the reference (atom3d/constants.py:11-111).

Corner i of a unit cube sits at (i & 1, (i >> 1) & 1, (i >> 2) & 1) (x
fastest); these tables are conventions of the public API, so they are kept
identical, generated here from that rule.
"""

import torch

CUBE_CORNERS = torch.tensor([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=torch.int64)

# 12 edges as corner pairs: x-aligned, then y-aligned, then z-aligned
CUBE_EDGES = torch.tensor(
    [[0, 1], [2, 3], [4, 5], [6, 7], [0, 2], [1, 3], [4, 6], [5, 7], [0, 4], [1, 5], [2, 6], [3, 7]],
    dtype=torch.int64,
)

# faces as 4 corners, counter-clockwise seen from outside: -X, +X, -Y, +Y, -Z, +Z
CUBE_FACES = torch.tensor(
    [[0, 4, 6, 2], [1, 3, 7, 5], [0, 1, 5, 4], [2, 6, 7, 3], [0, 2, 3, 1], [4, 5, 7, 6]], dtype=torch.int64
)

EDGE_TO_FACES = torch.tensor(
    [[0, 2], [0, 5], [0, 3], [0, 4], [1, 2], [1, 5], [1, 3], [1, 4], [2, 4], [2, 5], [3, 5], [3, 4]],
    dtype=torch.int64,
)

CUBE_CORNER_SIGNS = (CUBE_CORNERS * 2 - 1).float()

NEIGHBOR_OFFSETS_6 = torch.tensor(
    [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=torch.int32
)

# 26-neighbourhood, dz slowest, dx fastest, centre excluded
NEIGHBOR_OFFSETS_26 = torch.tensor(
    [[dx, dy, dz] for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dx, dy, dz) != (0, 0, 0)],
    dtype=torch.int32,
)

SIGN_WATER = 1
SIGN_DRY = -1
SIGN_DAM_DEFAULT = -1

# Neighbours sharing edge e of a cell (4 edges per axis, x-, y-, then
# z-aligned).  The two axes p < q perpendicular to the edge get a + or -
# offset by bit 0 and bit 1 of e % 4; the neighbours are p, q and p+q.
def _edge_neighbours():
    rows = []
    for e in range(12):
        axis, k = divmod(e, 4)
        p, q = [a for a in range(3) if a != axis]
        op, oq = [0, 0, 0], [0, 0, 0]
        op[p] = -1 if k & 1 else 1
        oq[q] = -1 if k & 2 else 1
        rows.append([op, oq, [op[a] + oq[a] for a in range(3)]])
    return rows


EDGE_NEIGHBOR_OFFSETS = torch.tensor(_edge_neighbours(), dtype=torch.int32)

# Neighbours sharing corner c: with s = CUBE_CORNER_SIGNS[c], the faces
# (sx,0,0), (0,sy,0), (0,0,sz), the edges (sx,sy,0), (sx,0,sz), (0,sy,sz) and
# the corner (sx,sy,sz).
CORNER_NEIGHBOR_OFFSETS = torch.tensor(
    [[[sx, 0, 0], [0, sy, 0], [0, 0, sz], [sx, sy, 0], [sx, 0, sz], [0, sy, sz], [sx, sy, sz]]
     for sx, sy, sz in CUBE_CORNER_SIGNS.int().tolist()],
    dtype=torch.int32,
)
