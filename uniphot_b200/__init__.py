"""uniphot_b200: B200-native per-island forced-photometry solve.

A drop-in for uniphot's (``tract7dt``) ``fit/grid_gpu/island_solver`` entry
points (``island_fit``, ``make_class_kernels``, ``run_class_chunk``) whose
arithmetic runs in hand-written sm_100a CUDA kernels behind the C ABI in
``include/uniphot_b200.h``.
"""

import os as _os

# The solver runs up to 32 chunks concurrently on separate CUDA streams; the
# driver's default of 8 hardware work queues would serialise most of them.
# The setting is read when the process creates its CUDA context, so it only
# takes effect if this package is imported before CUDA is first used.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

__version__ = "0.1.0"
