"""Module path mirror of the reference's atom3d.kernels for the flood fill."""
