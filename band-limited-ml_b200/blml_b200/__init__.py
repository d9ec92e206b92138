"""blml_b200: BLML's binned fitting path on one NVIDIA B200.

Host code mirrors the reference's Python surface (rahuljhu/band-limited-ml: blml_binned.BLMLBinned,
blml_trivial.make_modes / with_lattice, blml_local_gpu.rows / cols); every array operation runs in libblml_b200.so
(hand-written sm_100a CUDA behind a C ABI, include/blml_b200.h). There is no CPU fallback."""
from .spec import make_modes, parse_modes, with_lattice, with_fc, modes_fc, modes_trainable   # noqa: F401
from . import workloads                                           # noqa: F401


def __getattr__(name):
    # the GPU classes import torch and load the library on first use
    if name == 'BLMLBinned':
        from .binned import BLMLBinned
        return BLMLBinned
    if name == 'BLMLBinnedStreaming':
        from .streaming import BLMLBinnedStreaming
        return BLMLBinnedStreaming
    if name in ('rows', 'cols', 'ProductKernel', 'rank_coords', 'BLMLQuickLattice'):
        from . import local_gpu
        return getattr(local_gpu, name)
    raise AttributeError(name)
