"""B200-native TCodec pixel pipeline (v2 quadtree and legacy v0 / v1 block
bitstreams).

`tcodec_b200.api` binds the C ABI of libtcodec_b200.so: the reference's
include/tcodec.h encoder / decoder entry points and the additions of
include/tcodec_b200.h (batched and served forms, the standalone CTU-engine
frame entry points and the frame kernels), all backed by hand-written sm_100a
kernels.  `tcodec_b200.serving` replays a served-session schedule through
the server entry points, and `tcodec_b200.synth` makes the seeded synthetic
benchmark sources.
"""
from .api import LIB_PATH, load_library  # noqa: F401
