"""python -m beamz_b200.surrogate [batch] [steps] [warmup]: milliseconds per training
step of the default FNO surrogate (forward, backward, Adam) on random densities.
python -m beamz_b200.surrogate mixing: microseconds and bytes per second of the 1x1
channel-mixing GEMMs on the tcgen05 kernel and on the mma.sync kernel."""
import json
import sys

from .fno import bench_mixing, bench_step

if sys.argv[1:2] == ["mixing"]:
    for row in bench_mixing():
        print(json.dumps(row))
else:
    args = [int(v) for v in sys.argv[1:4]]
    print(f"training step: {bench_step(*args):.3f} ms")
