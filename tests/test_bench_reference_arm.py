"""The bench's CPU arm: the same workload configuration as the GPU arm,
built and run by the oracle alone (no part of liblux is loaded).  No GPU
needed."""
import subprocess
import sys

from tests.test_abi import ROOT

SCRIPT = r"""
import sys
sys.path.insert(0, {root!r})
import bench
w = bench.build_workload(0, host_only=True)
sample = bench.cpu_sample(w, 512, 4)
config = bench.workload_config(w)
assert config["resolve_points"] > 800000 and config["receivers"] > 50000, config
assert sample["rays"] > 0 and sample["points"] > 0, sample
maps = open("/proc/self/maps").read()
assert "liblux_oracle.so" in maps
assert "bevy_penumbra_b200/liblux.so" not in maps
print("ok", config["records"])
"""


def test_reference_arm_runs_without_the_library():
    out = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.startswith("ok")


def test_unsanitized_workload_settings_are_already_sanitized():
    import bench
    a, b = bench.settings_for_workload(sanitize=False).to_c(), bench.settings_for_workload().to_c()
    assert bytes(a) == bytes(b)
    s = bench.settings_for_workload()
    assert [bench.direction_count(s, l) for l in range(s.levels)] == [s.direction_count(l) for l in range(s.levels)]


def test_emitter_distance_matches_dense_sampling():
    """The bench's distance from a point to the nearest emitter triangle
    (used to band the error against the path-traced reference) equals the
    minimum over a dense barycentric sampling of the triangles, to within the
    sampling's resolution."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import bench

    class Packed:
        conventional = 0

    rec = np.zeros((2, 24), np.float32)
    rec[0, 0:3], rec[0, 12:15], rec[0, 16:19] = (0.0, 2.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0)
    rec[1, 0:3], rec[1, 12:15], rec[1, 16:19] = (3.0, 1.0, 1.0), (0.0, 1.0, 0.0), (1.0, 0.5, 0.0)
    Packed.lights = rec.view(np.uint32)
    rng = np.random.default_rng(5)
    pts = rng.uniform(-2.0, 5.0, (400, 3))
    got = bench.emitter_distance(Packed, pts)
    k = 200
    u, v = np.meshgrid(np.arange(k + 1) / k, np.arange(k + 1) / k)
    keep = u + v <= 1.0
    u, v = u[keep], v[keep]
    samples = np.concatenate([r[0:3] + u[:, None] * r[12:15] + v[:, None] * r[16:19] for r in rec.astype(np.float64)])
    want = np.min(np.linalg.norm(pts[:, None, :] - samples[None, :, :], axis=2), axis=1)
    assert np.all(got <= want + 1e-9)
    assert np.all(want - got < 0.02)
    assert bench.emitter_distance(Packed, np.array([[0.25, 2.0, 0.25]]))[0] == 0.0
