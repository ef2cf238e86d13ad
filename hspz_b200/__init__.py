"""hspz_b200: hspZ's seed-and-filter hot path (spaced-seed lookup, hit
expansion, ungapped X-drop extension with entropy correction, diagonal dedup)
as hand-written CUDA kernels for the B200 (sm_100a) behind a C ABI
(include/hspz_b200.h).  This package is the Python host mirror of the
reference's Engine interface; it does no sequence arithmetic itself."""
from .engine import Engine, EngineConfig, dedup_and_order, shape_info  # noqa: F401
from .scoring import build_sub_mat  # noqa: F401
