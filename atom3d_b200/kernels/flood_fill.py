"""Mirror of atom3d.kernels.flood_fill: flood_fill_3d_sparse runs the native
bit-volume flood fill (see atom3d_b200.apps.sparse_flood_fill)."""

from ..apps.sparse_flood_fill import flood_fill_3d_sparse

__all__ = ["flood_fill_3d_sparse"]
