"""field_b200: a B200-native (sm_100a) block-sparse SDF field engine.

The hot path of the reference field engine -- block classification, stream compaction into a
leaf pool, leaf-tile evaluation fused with min/max CSG (milling and drilling as tool
subtraction), the exact integer squared EDT and SDF value/gradient point queries -- as
hand-written CUDA behind a thin C ABI (``libfield_b200.so``), with Python host code that keeps
the reference's call signatures.  There is no CPU fallback: every compute call goes to the GPU
and raises if the CUDA library or a device is missing.
"""
__version__ = "0.1.0"
