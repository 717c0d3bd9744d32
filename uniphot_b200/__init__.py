"""uniphot_b200: B200-native per-island forced-photometry solve.

A drop-in for uniphot's (``tract7dt``) ``fit/grid_gpu/island_solver`` entry
points (``island_fit``, ``make_class_kernels``, ``run_class_chunk``) whose
arithmetic runs in hand-written sm_100a CUDA kernels behind the C ABI in
``include/uniphot_b200.h``.
"""

__version__ = "0.1.0"
