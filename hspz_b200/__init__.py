"""hspz_b200: hspZ's seed-and-filter hot path (spaced-seed lookup, hit
expansion, ungapped X-drop extension with entropy correction, diagonal dedup)
as hand-written CUDA kernels for the B200 (sm_100a) behind a C ABI
(include/hspz_b200.h).  This package is the Python host mirror of the
reference's Engine interface (``engine``), plus the host steps either side
of the path: input readers and packing (``sequence``), the .segments records,
renderer and file naming (``hsp``), the -D partition (``partition``) and the
synthetic workloads (``synth``).  Extension and scoring run in the library."""
from .engine import Engine, EngineConfig, dedup_and_order, shape_info  # noqa: F401
from .scoring import build_sub_mat  # noqa: F401
from .sequence import load_genome  # noqa: F401
