"""B200-native (sm_100a) per-island UV parameterization and validation.

Drop-in modules for the reference's engine/param.py, engine/gpu.py,
engine/validate.py and engine/metrics.py live in ``ultimate_uv_artist_b200.engine``;
the CUDA kernels are in ``csrc/`` behind the C ABI of ``include/uva_b200.h``.
"""
__version__ = "0.1.0"
