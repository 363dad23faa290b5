"""Launch-shape autotuner for a view's trace kernels.

Times each candidate LuxTuning (traversal scheduling mode, persistent blocks
per SM -- the warps-per-SM choice --, traversal stack depth, and whether
interval rays / visibility queries are put in coherence order before tracing)
on the caller's own frame with the library's per-stage CUDA-event timings,
and keeps the fastest.  The winner depends on the scene,
receivers and settings, so a host engine runs this once per view
configuration (untimed), like a convolution-algorithm search.
"""
from __future__ import annotations

import itertools

DEFAULT_SPACE = {
    "closest_mode": (0,),
    "shadow_mode": (0,),
    "blocks_per_sm": (16, 32),
    "stack_depth": (32, 64),
    "sort_rays": (0,),
    "sort_queries": (0, 1),
}


def candidates(space=None):
    space = space or DEFAULT_SPACE
    for cm, sm, bps, depth, sr, sq in itertools.product(space["closest_mode"], space["shadow_mode"],
                                                        space["blocks_per_sm"], space.get("stack_depth", (64,)),
                                                        space["sort_rays"], space["sort_queries"]):
        yield dict(closest_mode=cm, shadow_mode=sm, closest_blocks_per_sm=bps, shadow_blocks_per_sm=bps,
                   stack_depth=depth, sort_rays=sr, sort_queries=sq)


def autotune(view, run_frame, space=None, repeats: int = 2) -> dict:
    """run_frame() must issue one lux_view_trace_merge on `view`.

    Returns {"best": {...}, "trace_ms": best time, "trials": [(tuning, ms), ...]}."""
    view.set_timing(True)
    trials = []
    for cand in candidates(space):
        view.set_tuning(**cand)
        run_frame()  # the first frame with a new shape is not timed
        times = []
        for _ in range(repeats):
            run_frame()
            times.append(view.timings().trace_ms)
        trials.append((cand, min(times)))
    best, best_ms = min(trials, key=lambda t: t[1])
    view.set_tuning(**best)
    return {"best": best, "trace_ms": best_ms, "trials": trials}
