from .sparse_flood_fill import (construct_surface_dual_graph, flood_fill_3d_sparse, get_dam_wet_corners,
                                get_dam_neighborhood_signs, get_dam_wet_edges, get_dam_wet_faces,
                                sparse_flood_fill)
