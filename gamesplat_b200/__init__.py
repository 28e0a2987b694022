"""gamesplat_b200 - the per-frame Gaussian-splatting path of gamesplat
(cull/SH/project, radix depth sort, sorted alpha compositing, stochastic and
Gaussian Point Splatting passes) as hand-written CUDA for sm_100a behind a
C ABI (include/gs_api.h, libgs_cuda.so).

The CUDA library is required: importing works without it, but every render
call raises if libgs_cuda.so is missing.  There is no CPU fallback.
"""
from ._lib import GsError, LIB_PATH  # noqa: F401
from .denoiser import Denoiser  # noqa: F401
from .gsanim import GSAnim, load_gsanim  # noqa: F401
from .renderer import (  # noqa: F401
    MODE_NAMES,
    Renderer,
    camera_from_array,
    camera_to_array,
    camera_uniforms,
    load_ply,
    load_scene,
    load_sog,
    pack_raw,
    sort_pairs,
    sort_pairs_scratch_bytes,
    webp_decode,
)
