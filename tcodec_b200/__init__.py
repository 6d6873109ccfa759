"""B200-native TCodec v2 pixel pipeline.

`tcodec_b200.api` binds the include/tcodec.h C ABI of libtcodec_b200.so
(hand-written sm_100a kernels behind the reference's encoder API);
`tcodec_b200.kernels` binds the batched standalone kernels of
include/tcodec_b200.h; `tcodec_b200.synth` makes the seeded synthetic
benchmark sources.
"""
from .api import LIB_PATH, load_library  # noqa: F401
