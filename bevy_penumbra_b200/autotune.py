"""Launch-shape autotuner for a view's trace kernels.

Times candidate LuxTunings (traversal scheduling mode of each trace kernel,
persistent blocks per SM -- the warps-per-SM choice --, the tile of rays a
warp takes from the work queue per fetch, traversal stack depth, and whether
interval rays / visibility queries are put in coherence order before
tracing) on the caller's own frame with the library's per-stage CUDA-event
timings, and keeps the fastest.  The winner depends on the scene,
receivers and settings, so a host engine runs this once per view
configuration (untimed), like a convolution-algorithm search.
"""
from __future__ import annotations

import itertools

DEFAULT_SPACE = {
    "closest_mode": (0, 1),
    "shadow_mode": (0, 1),
    "blocks_per_sm": (8, 16, 32),
    "tile_rays": (32, 64, 128),
    "stack_depth": (32, 64),
    "sort_rays": (0, 1),
    "sort_queries": (0, 1),
}

START = dict(closest_mode=0, shadow_mode=0, blocks_per_sm=16, tile_rays=32, stack_depth=64, sort_rays=0,
             sort_queries=1)


def tuning_of(point: dict) -> dict:
    """A LuxTuning field dict of a search point (one blocks-per-SM axis for
    both persistent kernels)."""
    return dict(closest_mode=point["closest_mode"], shadow_mode=point["shadow_mode"],
                closest_blocks_per_sm=point["blocks_per_sm"], shadow_blocks_per_sm=point["blocks_per_sm"],
                tile_rays=point.get("tile_rays", 32), stack_depth=point["stack_depth"], sort_rays=point["sort_rays"],
                sort_queries=point["sort_queries"])


def candidates(space=None):
    """Every point of the space (the exhaustive search)."""
    space = space or DEFAULT_SPACE
    keys = list(space)
    for values in itertools.product(*(space[k] for k in keys)):
        yield tuning_of(dict(zip(keys, values)))


def autotune(view, run_frame, space=None, repeats: int = 2, sweeps: int = 2) -> dict:
    """run_frame() must issue one lux_view_trace_merge on `view`.

    Coordinate search: starting from START, each sweep tries every value of
    one axis at a time with the others at the best point so far (the axes
    interact little: scheduling, occupancy, tile, stack size, ray and query order),
    `sweeps` times over all axes; every distinct point is timed once (its
    first frame untimed, then the minimum of `repeats` frames).  The time is
    the frame's seed + trace + merge + pack stages: a choice that speeds the
    trace can slow the merge (the ray sort's histogram takes L2 the merge
    reads from).  Returns {"best": tuning, "frame_ms": best time,
    "trials": [(tuning, ms), ...]}."""
    space = space or DEFAULT_SPACE
    view.set_timing(True)
    timed = {}

    def measure(point):
        key = tuple(sorted(point.items()))
        if key not in timed:
            view.set_tuning(**tuning_of(point))
            run_frame()  # the first frame with a new shape is not timed
            times = []
            for _ in range(repeats):
                run_frame()
                t = view.timings()
                times.append(t.seed_ms + t.trace_ms + t.merge_ms + t.pack_ms)
            timed[key] = min(times)
        return timed[key]

    best = {k: (START[k] if START[k] in space[k] else space[k][0]) for k in space}
    best_ms = measure(best)
    for _ in range(sweeps):
        for axis in space:
            for value in space[axis]:
                point = dict(best, **{axis: value})
                ms = measure(point)
                if ms < best_ms:
                    best, best_ms = point, ms
    view.set_tuning(**tuning_of(best))
    trials = [(tuning_of(dict(k)), ms) for k, ms in timed.items()]
    return {"best": tuning_of(best), "frame_ms": best_ms, "trials": trials}
