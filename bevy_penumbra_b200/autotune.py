"""Launch-shape autotuner for a view's trace kernels.

Times each candidate LuxTuning (traversal scheduling mode and persistent
blocks per SM for the closest-hit and visibility kernels) on the caller's
own frame with the library's per-stage CUDA-event timings, and keeps the
fastest.  The winner is a property of the scene, receivers and settings, so
a host engine runs this once per view configuration (untimed), like a
convolution-algorithm search.
"""
from __future__ import annotations

import itertools


DEFAULT_SPACE = {
    "closest_mode": (0, 1),
    "shadow_mode": (0, 1),
    "blocks_per_sm": (4, 8, 16),
}


def autotune(view, run_frame, space=None, repeats: int = 2) -> dict:
    """run_frame() must issue one lux_view_trace_merge on `view`.

    Returns {"best": {...}, "trace_ms": best time, "trials": [(tuning, ms), ...]}."""
    space = space or DEFAULT_SPACE
    view.set_timing(True)
    trials = []
    for cm, sm, bps in itertools.product(space["closest_mode"], space["shadow_mode"], space["blocks_per_sm"]):
        cand = dict(closest_mode=cm, shadow_mode=sm, closest_blocks_per_sm=bps, shadow_blocks_per_sm=bps)
        view.set_tuning(**cand)
        run_frame()  # first frame with a new shape is not timed
        times = []
        for _ in range(repeats):
            run_frame()
            times.append(view.timings().trace_ms)
        trials.append((cand, min(times)))
    best, best_ms = min(trials, key=lambda t: t[1])
    view.set_tuning(**best)
    return {"best": best, "trace_ms": best_ms, "trials": trials}
