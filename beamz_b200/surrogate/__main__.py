"""python -m beamz_b200.surrogate [batch] [steps] [warmup]: milliseconds per training
step of the default FNO surrogate (forward, backward, Adam) on random densities."""
import sys

from .fno import bench_step

args = [int(v) for v in sys.argv[1:4]]
print(f"training step: {bench_step(*args):.3f} ms")
