"""Drop-in modules with the call signatures of the reference's engine/param.py,
engine/gpu.py, engine/validate.py and engine/metrics.py, computed by the
uva_b200 CUDA kernels. Importing a module that needs the GPU does not touch
the device; the first computation does, and raises without CUDA."""
