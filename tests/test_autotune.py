"""The autotuner's search on a fake view (host logic only): a separable cost
over the tuning axes is minimised, every timed point is distinct, and the
view is left at the best point."""
from types import SimpleNamespace

from bevy_penumbra_b200 import autotune as at


class FakeView:
    def __init__(self, cost):
        self.cost, self.tuning, self.frames = cost, None, 0

    def set_timing(self, on):
        pass

    def set_tuning(self, **t):
        self.tuning = t

    def timings(self):
        return SimpleNamespace(seed_ms=0.0, trace_ms=self.cost(self.tuning), merge_ms=0.0, pack_ms=0.0)


def cost(t):
    return (3.0 * (t["closest_mode"] == 1) + 1.0 * (t["shadow_mode"] == 0) + abs(t["closest_blocks_per_sm"] - 8) / 8
            + 0.5 * (t["stack_depth"] == 64) + 2.0 * (t["sort_queries"] == 0) + 0.25 * (t["sort_rays"] == 1)
            + 0.125 * (t["tile_rays"] != 64) + 5.0)


def test_coordinate_search_finds_the_separable_minimum():
    view = FakeView(cost)
    frames = []
    out = at.autotune(view, lambda: frames.append(1))
    best = out["best"]
    assert best == dict(closest_mode=0, shadow_mode=1, closest_blocks_per_sm=8, shadow_blocks_per_sm=8,
                        tile_rays=64, stack_depth=32, sort_rays=0, sort_queries=1)
    assert out["frame_ms"] == cost(best) == 5.0
    assert view.tuning == best
    keys = [tuple(sorted(t.items())) for t, _ in out["trials"]]
    assert len(keys) == len(set(keys)) < len(list(at.candidates()))
    assert len(frames) == 3 * len(keys)  # one untimed + two timed frames per point
