"""Thread-block shape autotuner for the stencil kernels.

The box kernels (one thread per grid point) and the column kernels (one
thread per column) take their block shape from a process-wide setting of
the library (``fv3b_set_launch_shape``).  The shape changes no result, only
speed, and the best one depends on the grid size (how many blocks fill the
148 SMs, how a tile's i rows map onto warps).  ``tune`` times a caller's
workload for each candidate shape with CUDA events and keeps the fastest.
"""
import torch

from . import _lib

# (box_x, box_y, column block): box_x covers i (warp-contiguous)
CANDIDATES = (
    (32, 4, 128), (32, 8, 128), (64, 2, 128), (64, 4, 128), (32, 16, 128),
    (128, 1, 128), (32, 2, 128), (32, 4, 64), (32, 4, 256), (64, 4, 64),
)


def tune(run, precision="f64", candidates=CANDIDATES, repeats=2):
    """Time ``run()`` (which enqueues work on the current stream) for each
    candidate shape and set the fastest.  Returns (best shape, {shape: ms})."""
    timings = {}
    stream = torch.cuda.current_stream()
    for shape in candidates:
        _lib.set_launch_shape(*shape, precision=precision)
        run()  # warm-up with this shape
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(repeats):
            run()
        stop.record(stream)
        torch.cuda.synchronize()
        timings[shape] = start.elapsed_time(stop) / repeats
    best = min(timings, key=timings.get)
    _lib.set_launch_shape(*best, precision=precision)
    return best, timings
