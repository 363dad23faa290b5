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
