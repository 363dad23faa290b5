"""GPU screen reconstruction (lux_screen_filter) against the oracle on the
same analytic G-buffer frames: the temporal history is bit-exact; the
a-trous output (expf weights) agrees within 1e-5 relative."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import synthetic_screen, to_device, from_device, empty_device

pytestmark = pytest.mark.gpu

W, H = 160, 96
RTOL, ATOL = 1e-5, 1e-6


@pytest.mark.parametrize("steps", [0, 1, 3, 4])
def test_screen_filter_matches_oracle(steps):
    s = bp.RadianceCascades(probe_spacing=0.25, normal_bias=0.005, history_frames=24).sanitized()
    ctx = bp.LuxContext()
    screen = bp.ScreenFilter(ctx, W, H)
    out = empty_device(H * W * 16)
    history = None
    prev_clip = None
    eyes = [(0.0, 1.2, 2.5), (0.03, 1.21, 2.48), (0.06, 1.2, 2.45), (0.06, 1.2, 2.45)]
    for frame, eye in enumerate(eyes):
        irr, pos, nrm, ident, clip = synthetic_screen(W, H, eye, (0.0, 0.3, 0.0), seed=10 + frame)
        prev = clip if prev_clip is None else prev_clip
        kw = dict(scene_changed=frame == 2, dirty=[-0.2, 0.0, -0.2, 0.2, 0.5, 0.2] if frame == 3 else None)
        d = [to_device(a) for a in (irr, pos, nrm, ident)]
        screen.filter(s, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), prev, out.data_ptr(),
                      spatial_filter_steps=steps, **kw)
        gh_irr, gh_meta = screen.read_history()
        history, oout = oracle.screen_filter(s.to_c(), irr, pos, nrm, ident, prev, history=history,
                                             spatial_filter_steps=steps, **kw)
        np.testing.assert_array_equal(gh_irr.view(np.uint32), history[..., 0:4].view(np.uint32), err_msg=f"frame {frame}")
        np.testing.assert_array_equal(gh_meta.view(np.uint32), history[..., 4:8].view(np.uint32), err_msg=f"frame {frame}")
        ctx.synchronize()
        gout = from_device(out, np.float32, (H, W, 4))
        if steps == 0:
            np.testing.assert_array_equal(gout.view(np.uint32), oout.view(np.uint32))
        else:
            np.testing.assert_allclose(gout, oout, rtol=RTOL, atol=ATOL, err_msg=f"frame {frame}")
        prev_clip = clip
    assert (gh_meta[..., 0] > 1.0).mean() > 0.3  # history accumulated over the frames
