"""imgrecsrc_b200 -- a B200-native X-ray CT projection engine.

Drop-in for the projector of anindyabijoydas/imgRecSrc (prj/): parallel- and
fan-beam forward projection, the matched backprojection and FBP, behind the
reference's own interface (setup / gpuPrj / mPrj), with every compute step in
hand-written sm_100a CUDA kernels reached through the C ABI of
include/ctprj.h.
"""
from ._lib import (BWD_BIT, FBP_BIT, FWD_BIT, CtprjError, Geometry, check, lib)  # noqa: F401
from .projector import Projector  # noqa: F401
