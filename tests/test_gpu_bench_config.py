"""Parity at the benchmarked configuration.

The bench frame is the seed-2 atrium of 262,144 triangles seen by a
1280x720 camera, receivers at 4x4 px, 36 interval rays per receiver, 16
emissive samples (8 visibility queries per shaded hit), 8 cascades of 32
base directions, world history on, and the trace kernels under the tuning
the autotuner picks there (16 persistent blocks per SM, a 64-entry stack,
visibility queries counting-sorted over 8 emitter buckets x 128^3 origin
cells).  The GPU frame and the oracle frame run on the same receiver subset
(every 64th receiver, as the CPU baseline samples), two frames in a row so
the second blends the first's records:

* interval-ray hits (triangle, instance, error bits, distance bits) are
  bit-exact against the oracle's closest hits of the same rays;
* per-record sample counts are exact; raw and merged records are within
  rtol 1e-4 / atol 1e-6 (float atomics sum samples in arbitrary order);
* the resolve of a few thousand primary hits of the full-resolution camera
  is within 1e-4 relative.
"""
import functools

import numpy as np
import pytest

import bench
import bevy_penumbra_b200 as bp
import oracle
from bevy_penumbra_b200 import scenes
from tests.helpers import empty_device, from_device, to_device
from tests.test_gpu_cascades import ATOL, RTOL, compare_levels

pytestmark = pytest.mark.gpu

RECEIVER_STRIDE = 64   # the CPU baseline's receiver sample
POINT_STRIDE = 256     # resolve points: every 256th primary hit of the full-resolution camera
BENCH_TUNING = dict(closest_mode=0, shadow_mode=0, closest_blocks_per_sm=16, shadow_blocks_per_sm=16,
                    stack_depth=64, sort_rays=0, sort_queries=1)


@functools.lru_cache(maxsize=1)
def workload():
    w = bench.build_workload(0)
    rpos = np.ascontiguousarray(w["rpos"][::RECEIVER_STRIDE])
    rnrm = np.ascontiguousarray(w["rnrm"][::RECEIVER_STRIDE])
    ppos = np.ascontiguousarray(w["ppos"][::POINT_STRIDE])
    pnrm = np.ascontiguousarray(w["pnrm"][::POINT_STRIDE])
    camera = bp.camera_struct(scenes.clip_from_world(bench.EYE, bench.TARGET, 60.0, bench.WIDTH, bench.HEIGHT),
                              bench.EYE, bench.HEIGHT, 1)
    oscene = oracle.OracleScene.from_packed(w["packed"])
    return w, rpos, rnrm, ppos, pnrm, camera, oscene


def settings_at(frame):
    s = bench.settings_for_workload()
    s.frame_index = frame
    return s


@pytest.mark.parametrize("stack_depth", [64, 32])
def test_bench_config_matches_oracle(stack_depth):
    w, rpos, rnrm, ppos, pnrm, camera, oscene = workload()
    ctx, scene = w["ctx"], w["scene"]
    assert w["desc"].world_triangles() == 262_144
    first = settings_at(0)
    assert (first.levels, first.base_columns * first.base_rows, first.rays_per_receiver,
            first.emissive_samples) == (8, 32, 36, 16)
    n = len(rpos)
    rays = n * first.rays_per_receiver
    view = bp.SplitView(ctx, max_receivers=n, max_cells=1 << 16, max_entries=1 << 24, max_rays=rays)
    view.set_camera(scenes.clip_from_world(bench.EYE, bench.TARGET, 60.0, bench.WIDTH, bench.HEIGHT), bench.EYE,
                    bench.HEIGHT, 1)
    view.set_tuning(**dict(BENCH_TUNING, stack_depth=stack_depth))
    d_pos, d_nrm = to_device(rpos), to_device(rnrm)
    prev = None
    for frame in (0, 1):
        s = settings_at(frame)
        view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), n)
        st = view.stats()
        assert st.error_flags == 0
        ofr = oracle.OracleFrame(oscene, s.to_c(), rpos, rnrm, previous=prev, camera=camera)
        ost = ofr.stats()
        assert st.interval_rays == ost.interval_rays == rays
        assert st.shadow_rays == ost.shadow_rays
        assert st.deposits == ost.deposits and st.unsupported == ost.unsupported
        got = view.read_hits(rays)
        want = ofr.hits(rays)
        assert len(want) == rays
        np.testing.assert_array_equal(got["triangle"], want["triangle"], err_msg=f"frame {frame} triangle")
        np.testing.assert_array_equal(got["instance"], want["instance"], err_msg=f"frame {frame} instance")
        np.testing.assert_array_equal(got["errors"], want["errors"], err_msg=f"frame {frame} errors")
        np.testing.assert_array_equal(got["distance"].view(np.uint32), want["distance"].view(np.uint32),
                                      err_msg=f"frame {frame} distance")
        assert np.mean(got["triangle"] != 0xFFFFFFFF) > 0.5
        compare_levels(s, [view.read_level(l) for l in range(s.levels)], ofr, exact=False)
        prev = ofr
    d_p, d_n, d_o = to_device(ppos), to_device(pnrm), empty_device(len(ppos) * 16)
    view.resolve(s, d_p.data_ptr(), d_n.data_ptr(), len(ppos), d_o.data_ptr())
    ctx.synchronize()
    out = from_device(d_o, np.float32, (len(ppos), 4))
    expected = prev.resolve(ppos, pnrm)
    np.testing.assert_allclose(out, expected, rtol=RTOL, atol=ATOL)
    assert np.mean(out[:, 3] >= 1.0) > 0.01  # sparse receivers: most points see no cascade-0 probe

