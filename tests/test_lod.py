"""Distance LODs (splitLodBlendForParameters, shaders/common.slang:431-461)
in the oracle: the reference's LOD regressions of src/lod_tests.rs
(gpu_split_lod_grows_beyond_four_cascades_and_preserves_keys :180-229,
gpu_split_lod_overlap_is_continuous_beyond_lod_three :232-264,
gpu_split_lod_orthographic_uses_projected_spacing_not_camera_distance
:267-300; tolerance 2e-5 x max(1, |expected|) as their close()), and a Split
frame whose receivers span several LODs."""
import math

import numpy as np

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import packed


def close(actual, expected):
    assert abs(actual - expected) <= max(abs(expected), 1.0) * 2e-5, (actual, expected)


def perspective_infinite_reverse(fov_y, aspect, near):
    f = 1.0 / math.tan(0.5 * fov_y)
    m = np.zeros((4, 4))
    m[0, 0], m[1, 1], m[2, 3], m[3, 2] = f / aspect, f, near, -1.0
    return m


def orthographic(left, right, bottom, top, near, far):
    m = np.eye(4)
    m[0, 0], m[1, 1], m[2, 2] = 2.0 / (right - left), 2.0 / (top - bottom), 1.0 / (near - far)
    m[0, 3], m[1, 3], m[2, 3] = -(right + left) / (right - left), -(top + bottom) / (top - bottom), near / (near - far)
    return m


def view_from_world(camera, target):
    """Inverse of a transform at `camera` whose -Z looks at `target` (Y up)."""
    camera = np.asarray(camera, np.float64)
    back = camera - np.asarray(target, np.float64)
    back /= np.linalg.norm(back)
    right = np.cross((0.0, 1.0, 0.0), back)
    right /= np.linalg.norm(right)
    up = np.cross(back, right)
    world_from_view = np.eye(4)
    world_from_view[:3, 0], world_from_view[:3, 1], world_from_view[:3, 2] = right, up, back
    world_from_view[:3, 3] = camera
    return np.linalg.inv(world_from_view)


def lod_camera(projection, camera, target):
    clip = (projection @ view_from_world(camera, target)).astype(np.float32)
    # viewport 512 x 512 (src/lod_tests.rs:163), 8 target pixels (:165).
    return bp.camera_struct(clip, camera, 512, 8)


def settings():
    # tuning (1.0, 1.6, 0, 1): spacing 1, interval 1.6 (src/lod_tests.rs:164).
    return bp.RadianceCascades(probe_spacing=1.0, interval_length=1.6).sanitized().to_c()


def test_lod_grows_beyond_four_cascades():
    projection = perspective_infinite_reverse(math.pi / 2, 1.0, 0.1)
    camera = np.array([3.0, -5.0, 7.0])
    cam = lod_camera(projection, camera, camera - np.array([0.0, 0.0, 1.0]))
    base = 32.0  # focal pixels x spacing / target pixels = 256 / 8
    for radius, lod in zip([4.0, 8.0, 16.0, 32.0, 2.0 ** 30], [2, 3, 4, 5, 24]):
        low, high, blend = oracle.lod_blend(settings(), cam, camera + np.array([radius * base, 0.0, 0.0]))
        assert (low, high) == (lod, lod)
        close(blend, 0.0)
    # Chebyshev, not Euclidean distance, sets perspective bands.
    low, high, _ = oracle.lod_blend(settings(), cam, camera + 7.0 * base)
    assert (low, high) == (2, 2)


def test_lod_overlap_is_continuous():
    projection = perspective_infinite_reverse(math.pi / 2, 1.0, 0.1)
    cam = lod_camera(projection, np.zeros(3), np.array([0.0, 0.0, -1.0]))
    for next_lod in range(1, 8):
        boundary = np.float32(32.0 * 2.0 ** next_lod)
        previous = 0.0
        for step, (fraction, expected) in enumerate(zip([0.9, 0.95, 0.999999, 1.0, 1.00001],
                                                        [0.0, 0.5, 0.99999, 0.0, 0.0])):
            x = np.float32(boundary * np.float32(fraction))
            low, high, blend = oracle.lod_blend(settings(), cam, (x, 0.0, 0.0))
            assert low == (next_lod - 1 if step < 3 else next_lod)
            close(blend, expected)
            # The blended spacing grows monotonically through the overlap.
            scale = 2.0 ** low * (1.0 - blend) + 2.0 ** high * blend
            assert scale >= previous
            previous = scale
            if step >= 2:
                close(scale, 2.0 ** next_lod)


def test_lod_orthographic_uses_projected_spacing():
    projection = orthographic(-1152.0, 1152.0, -1152.0, 1152.0, 0.1, 100000.0)
    target = np.array([-3.0, 2.0, 1.0])
    direction = np.array([2.0, 1.0, 3.0]) / np.linalg.norm([2.0, 1.0, 3.0])
    for distance in (10.0, 1000.0, 20000.0):
        cam = lod_camera(projection, target + direction * distance, target)
        for p in (target, target + np.array([-7.0, 5.0, 12.0])):
            low, high, blend = oracle.lod_blend(settings(), cam, p)
            assert (low, high) == (5, 5)  # 8 px target = 36 x the projected spacing
            close(blend, 0.0)
    zoom = orthographic(-288.0, 288.0, -288.0, 288.0, 0.1, 100000.0)
    low, _, _ = oracle.lod_blend(settings(), lod_camera(zoom, target + direction * 1000.0, target), target)
    assert low == 3


def test_split_frame_spans_lods():
    """Receivers along a line away from a perspective camera fall into
    increasing LODs; each LOD's cells use spacing x 2^lod and the frame's
    records exist at several LODs."""
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=2,
                            emissive_samples=4).sanitized()
    n = 256
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = np.linspace(-0.95, 0.95, n, dtype=np.float32)
    pos[:, 2] = np.linspace(-0.95, 0.95, n, dtype=np.float32)
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    eye = np.array([0.9, 0.4, 0.9])
    projection = perspective_infinite_reverse(math.radians(60.0), 16 / 9, 0.1)
    # base = max(focal 27.7 px x 0.25 / 16 px, 0.25) = 0.43 m: LODs 0-2 across the floor.
    cam = bp.camera_struct((projection @ view_from_world(eye, (0.0, 0.0, 0.0))).astype(np.float32), eye, 32, 16)
    scene = oracle.OracleScene.from_packed(packed("cornell"))
    f = oracle.OracleFrame(scene, s.to_c(), pos, nrm, camera=cam)
    keys = f.level(0, s.direction_count(0))[0]
    lods = {(int(k[3]) >> 18) & 31 for k in keys}
    assert len(lods) >= 2, lods
    for i in range(0, n, 17):
        low, high, _ = oracle.lod_blend(s.to_c(), cam, pos[i, :3])
        cell = np.floor(pos[i, :3] / np.float32(0.25 * 2.0 ** low)).astype(np.int64)
        assert any((k[:3] == cell).all() and ((int(k[3]) >> 18) & 31) == low for k in keys)
