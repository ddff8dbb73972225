from .sparse_flood_fill import flood_fill_3d_sparse, sparse_flood_fill

__all__ = ["sparse_flood_fill", "flood_fill_3d_sparse"]
