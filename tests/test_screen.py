"""Screen reconstruction (the reference's temporal + denoise passes,
shaders/cascades.slang:310-690) in the oracle: invariants of the temporal
history and the a-trous filter on an analytic G-buffer."""
import numpy as np

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import synthetic_screen

W, H = 96, 64
EYE, TARGET = (0.0, 1.2, 2.5), (0.0, 0.3, 0.0)


def settings(**kw):
    return bp.RadianceCascades(probe_spacing=0.25, normal_bias=0.005, **kw).sanitized().to_c()


def test_static_camera_accumulates_history():
    irr, pos, nrm, ident, clip = synthetic_screen(W, H, EYE, TARGET, seed=1)
    st = settings(history_frames=24)
    h1, out1 = oracle.screen_filter(st, irr, pos, nrm, ident, clip, spatial_filter_steps=0)
    supported = irr[..., 3] > 0
    fresh = np.clip((irr[..., 3] - np.floor(irr[..., 3])) * 4.0, 0, 1)
    np.testing.assert_array_equal(h1[..., 4][supported], fresh[supported].astype(np.float32))
    np.testing.assert_array_equal(out1[..., :3][supported], irr[..., :3][supported])
    # The same frame again: every supported pixel reprojects onto itself.
    h2, out2 = oracle.screen_filter(st, irr, pos, nrm, ident, clip, history=h1, spatial_filter_steps=0)
    interior = supported.copy()
    interior[[0, -1], :] = interior[:, [0, -1]] = False
    grew = h2[..., 4][interior] > h1[..., 4][interior]
    assert grew.mean() > 0.95
    assert np.all(h2[..., 4] <= 24.0)
    # Unsupported pixels keep validated history unchanged.
    lost = (irr[..., 3] < 0) & (h1[..., 4] > 0)
    assert not lost.any() or np.all(h2[..., 4][lost] <= h1[..., 4][lost])


def test_history_off_dirty_box_and_moved_camera():
    irr, pos, nrm, ident, clip = synthetic_screen(W, H, EYE, TARGET, seed=2)
    h1, _ = oracle.screen_filter(settings(), irr, pos, nrm, ident, clip, spatial_filter_steps=0)
    fresh_only, _ = oracle.screen_filter(settings(), irr, pos, nrm, ident, clip, spatial_filter_steps=0)
    for kw in (dict(st=settings(history_frames=0)), dict(st=settings(), dirty=[-9, -9, -9, 9, 9, 9])):
        h2, _ = oracle.screen_filter(kw["st"], irr, pos, nrm, ident, clip, history=h1,
                                     dirty=kw.get("dirty"), spatial_filter_steps=0)
        np.testing.assert_array_equal(h2[..., 4], fresh_only[..., 4])
    # A moved camera reprojects part of the history.
    irr2, pos2, nrm2, ident2, clip2 = synthetic_screen(W, H, (0.05, 1.2, 2.5), TARGET, seed=3)
    h2, _ = oracle.screen_filter(settings(), irr2, pos2, nrm2, ident2, clip, history=h1, spatial_filter_steps=0)
    fresh2, _ = oracle.screen_filter(settings(), irr2, pos2, nrm2, ident2, clip2, spatial_filter_steps=0)
    more = h2[..., 4] > fresh2[..., 4]
    assert 0.5 < more[pos2[..., 3] > 0].mean() < 1.0


def test_denoise_smooths_within_surfaces():
    irr, pos, nrm, ident, clip = synthetic_screen(W, H, EYE, TARGET, seed=4)
    st = settings()
    _, raw = oracle.screen_filter(st, irr, pos, nrm, ident, clip, spatial_filter_steps=0)
    _, out = oracle.screen_filter(st, irr, pos, nrm, ident, clip, spatial_filter_steps=3)
    floor = (ident[..., 0] == 1) & (irr[..., 3] > 0)
    # Neighbour differences (noise) shrink on the floor; edges are kept.
    def roughness(img):
        d = np.abs(np.diff(img[..., 1], axis=1))
        m = floor[:, 1:] & floor[:, :-1]
        return d[m].mean()
    assert roughness(out) < 0.5 * roughness(raw)
    assert np.all(np.isfinite(out))
    assert np.all(out[pos[..., 3] <= 0] == 0.0)
