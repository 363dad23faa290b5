"""The allocation-free interval-radiance entry point.

Some hosts may not allocate device memory while they run: a real-time render
thread where cudaMalloc/cudaFree can synchronise the device and stall a frame,
or an engine that reserves its device budget up front through its own
allocator.  lux_interval_radiance_noalloc serves them from a fixed scratch
array inside the library (at most 8192 rays per call).  These tests call it
through the C ABI and check it against lux_interval_radiance, which uses
scratch owned by the context, on two calls in a row.  This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import _native as N
from tests.helpers import empty_device, from_device, packed, to_device

pytestmark = pytest.mark.gpu

MAX_RAYS = 8192


def rays_in_box(n, seed):
    rng = np.random.default_rng(seed)
    rays = np.zeros(n, dtype=bp.RAY_DTYPE)
    rays["origin"] = rng.uniform((-0.95, 0.05, -0.95), (0.95, 1.95, 0.95), size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["direction"] = d.astype(np.float32)
    rays["limit"] = 1e20
    return rays


def test_no_alloc_matches_allocating_entry_on_two_calls():
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    lib = N.lib()
    for call, (n, frame) in enumerate([(5000, 3), (MAX_RAYS, 4)]):
        settings = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=16, frame_index=frame).sanitized()
        s = settings.to_c()
        rays = rays_in_box(n, seed=call)
        d_rays = to_device(rays)
        d_expected = empty_device(n * 16)
        d_out = empty_device(n * 16)
        ctx.check(lib.lux_interval_radiance(ctx.handle, scene.handle, C.byref(s), d_rays.data_ptr(), n,
                                            d_expected.data_ptr()))
        ctx.check(lib.lux_interval_radiance_noalloc(ctx.handle, scene.handle, C.byref(s), d_rays.data_ptr(), n,
                                                    d_out.data_ptr()))
        ctx.synchronize()
        expected = from_device(d_expected, np.float32, (n, 4))
        got = from_device(d_out, np.float32, (n, 4))
        # The same kernels on the same inputs: bit-identical, like the oracle parity tests.
        np.testing.assert_array_equal(got.view(np.uint32), expected.view(np.uint32), err_msg=f"call {call}")
        assert np.mean(got[:, 3] > 0) > 0.9
        assert np.mean(got[:, :3].sum(1) > 0) > 0.2


def test_no_alloc_rejects_batches_above_its_capacity():
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    s = bp.RadianceCascades().sanitized().to_c()
    d_rays = empty_device((MAX_RAYS + 1) * 32)
    d_out = empty_device((MAX_RAYS + 1) * 16)
    status = N.lib().lux_interval_radiance_noalloc(ctx.handle, scene.handle, C.byref(s), d_rays.data_ptr(),
                                                   MAX_RAYS + 1, d_out.data_ptr())
    assert status == 4  # LUX_ERR_CAPACITY, refused before any launch
    assert b"8192" in N.lib().lux_last_error_message(ctx.handle)


def test_no_alloc_calls_leave_free_device_memory_unchanged():
    """The property the entry point exists for: once its kernels are loaded,
    a call takes no device memory.  Every buffer the calls use is allocated
    before the first reading; the allocating entry point is not called
    between the readings."""
    import torch

    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    lib = N.lib()
    s = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=16, frame_index=7).sanitized().to_c()
    rays = rays_in_box(MAX_RAYS, seed=11)
    d_rays = to_device(rays)
    d_out = empty_device(MAX_RAYS * 16)
    # Warm-up: loads the kernels and looks up the scratch array's address.
    ctx.check(lib.lux_interval_radiance_noalloc(ctx.handle, scene.handle, C.byref(s), d_rays.data_ptr(), 64,
                                                d_out.data_ptr()))
    ctx.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for n in (MAX_RAYS, 1000):
        ctx.check(lib.lux_interval_radiance_noalloc(ctx.handle, scene.handle, C.byref(s), d_rays.data_ptr(), n,
                                                    d_out.data_ptr()))
    ctx.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
