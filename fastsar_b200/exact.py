"""Exact backprojection (the oracle family of the former): ExactFormer and backproject on the GPU, and the grid points
of form_image."""
import numpy as np

C = 299792458.0


def plane_points(nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), height=None):
    """Points [nx, ny, 3] of the form_image grid: pixel (i, j) at (i - nx/2) spx e1 + (j - ny/2) spy e2, optionally
    displaced along the plane normal (pointing up) by height [nx, ny] (fastsar/bp.py:351-361)."""
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    X, Y = np.meshgrid((np.arange(nx) - nx / 2.0) * spx, (np.arange(ny) - ny / 2.0) * spy, indexing='ij')
    p = X[..., None] * e1 + Y[..., None] * e2
    if height is not None:
        n = np.cross(e1, e2)
        n = n / np.linalg.norm(n) * np.sign(n[2] if abs(n[2]) > 1e-12 else 1.0)
        p = p + np.asarray(height, np.float64)[..., None] * n
    return p
