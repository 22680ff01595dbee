"""fastsar_b200: factorized-backprojection (FFBP) spotlight SAR image formation on the NVIDIA B200.

A drop-in for the factorized-backprojection former of saulpingerman/FastSAR 0.3.1 (fastsar.ImageFormer,
fastsar.form_image, fastsar.ExactFormer, fastsar.backproject): the same arguments and the same complex64 image,
formed by hand-written sm_100a CUDA kernels behind a C ABI (include/ffbp_b200.h)."""
__version__ = '0.1.0'

from .sim import Collect, make_collect  # noqa: F401
from .plan import make_plan, choose_T, final_phase_error, collection_arrays, final_weights  # noqa: F401
from .exact import plane_points  # noqa: F401


def __getattr__(name):
    # the formers import torch and load the CUDA library: only when asked for
    if name in ('ImageFormer', 'form_image', 'BatchFormer'):
        from . import api
        return getattr(api, name)
    if name in ('ExactFormer', 'backproject'):
        from . import exact
        return getattr(exact, name)
    raise AttributeError(name)
