"""begputhinning_b200 -- B200-native directional-subiteration thinning of
binary 2D images and 3D volumes and centreline segment extraction, a drop-in
for the Thinning2D / Thinning3D / CenterlineExtraction entry points of
BEGPUThinning.  The compute path is libbgt.so (hand-written sm_100a CUDA
behind a C ABI, include/bgt_capi.h); this package is the Python host side."""
from ._lib import BGTError, lib
from .api import (Batch, CenterlineExtraction, Context, ExtractSegmentsV, PipelinedBatch, Segments, Thinning2D,
                  Thinning3D, cfg_describe, cfg_list, default_context, matlab_segments, thin_device)

__all__ = ["BGTError", "lib", "Batch", "CenterlineExtraction", "Context", "ExtractSegmentsV", "PipelinedBatch",
           "Segments", "Thinning2D", "Thinning3D", "cfg_describe", "cfg_list", "default_context", "matlab_segments",
           "thin_device"]
