"""Learned radiance cache (lux_cache_*): the tcgen05 BF16 MLP against a
plain PyTorch FP32 reference of the same network, the backward pass through
one Adam step, and online training on a smooth radiance field."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from tests.helpers import empty_device, from_device, to_device

pytestmark = pytest.mark.gpu

# BF16 weights and BF16 activations between layers, FP32 accumulation.
RTOL, ATOL = 2e-2, 2e-3


def bf16_round(a):
    import torch
    return torch.as_tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float32)


def torch_mlp(x_bits, layers):
    """FP32 reference: inputs and weights rounded to BF16, hidden
    activations rounded to BF16 between layers (what the kernel stores)."""
    import torch
    x = torch.from_numpy(x_bits.astype(np.uint32) << 16).view(torch.float32)
    h = x
    for k, w in enumerate(layers):
        z = h @ bf16_round(w).T
        h = bf16_round(torch.relu(z)) if k < 4 else z
    return h


def random_samples(n, seed, lo=-2.0, hi=2.0):
    rng = np.random.default_rng(seed)
    s = np.zeros(n, dtype=bp.CACHE_SAMPLE_DTYPE)
    s["position"] = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    s["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    s["normal"] = np.array([0.0, 1.0, 0.0])
    s["albedo"] = rng.uniform(0.2, 0.8, size=(n, 3))
    s["weight"] = 1.0
    return s


def field(s):
    """A smooth radiance field of position and direction."""
    p, d = s["position"].astype(np.float64), s["direction"].astype(np.float64)
    r = 0.6 + 0.4 * np.sin(1.3 * p[:, 0] + 0.7 * d[:, 1])
    g = 0.5 + 0.3 * np.cos(0.9 * p[:, 2] - 0.5 * d[:, 0])
    b = 0.4 + 0.2 * p[:, 1] * d[:, 2]
    out = np.zeros((len(s), 4), np.float32)
    out[:, 0], out[:, 1], out[:, 2] = r, g, b
    return out


def make_cache(ctx, **kw):
    cache = bp.LearnedCache(ctx, **kw)
    cache.set_bounds((-2.0, -2.0, -2.0), (2.0, 2.0, 2.0))
    return cache


@pytest.mark.parametrize("n", [128, 1000, 20000])
def test_forward_matches_torch_fp32(n):
    ctx = bp.LuxContext()
    cache = make_cache(ctx)
    s = random_samples(n, 1)
    d_s = to_device(s)
    d_x = empty_device(n * 128)
    cache.encode(d_s.data_ptr(), n, d_x.data_ptr())
    ctx.synchronize()
    x_bits = from_device(d_x, np.uint16, (n, 64))
    d_y = empty_device(n * 16)
    cache.forward(d_x.data_ptr(), n, d_y.data_ptr())
    ctx.synchronize()
    got = from_device(d_y, np.float32, (n, 4))
    ref = torch_mlp(x_bits, cache.weights()).numpy()
    assert cache.stats().error_flags == 0
    scale = np.abs(ref[:, :3]).max()
    np.testing.assert_allclose(got[:, :3], ref[:, :3], rtol=RTOL, atol=ATOL * max(scale, 1.0))
    assert np.all(got[:, 3] == 1.0)
    # The encoding: direction SH at 32..47 (degree 0 constant, degree 1 =
    # 0.4886 (-y, z, -x)), normal at 48..50, constant 1 at 54, zeros after.
    x = (x_bits.astype(np.uint32) << 16).view(np.float32)
    d = s["direction"]
    np.testing.assert_allclose(x[:, 32], 0.28209479, rtol=1e-2)
    np.testing.assert_allclose(x[:, 33:36], 0.48860251 * np.stack([-d[:, 1], d[:, 2], -d[:, 0]], 1), atol=1e-2)
    np.testing.assert_allclose(x[:, 48:51], s["normal"], atol=1e-2)
    assert np.all(x[:, 54] == 1.0) and np.all(x[:, 55:] == 0.0)


def test_one_step_gradient_signs_match_torch():
    """After one Adam step every weight moves by -lr * sign(gradient) (bias
    correction makes the first step m / sqrt(v) = sign g); the signs must
    match torch autograd of the same loss on the same BF16 inputs."""
    import torch
    ctx = bp.LuxContext()
    n = 4096
    cache = make_cache(ctx, batch=n, learning_rate=1e-3)
    s = random_samples(n, 2)
    t = field(s)
    d_s, d_t = to_device(s), to_device(t)
    d_x = empty_device(n * 128)
    cache.encode(d_s.data_ptr(), n, d_x.data_ptr())
    ctx.synchronize()
    x_bits = from_device(d_x, np.uint16, (n, 64))
    before = cache.weights()
    cache.train(d_s.data_ptr(), d_t.data_ptr(), n)
    after = cache.weights()
    assert cache.stats().error_flags == 0
    # torch reference gradient.
    x = torch.from_numpy(x_bits.astype(np.uint32) << 16).view(torch.float32)
    ws = [bf16_round(w).clone().requires_grad_(True) for w in before]
    h = x
    for k, w in enumerate(ws):
        z = h @ w.T
        h = torch.relu(z) if k < 4 else z
    y = h[:, :3]
    tt = torch.from_numpy(t[:, :3])
    loss = (((y - tt) ** 2) / (y.detach() ** 2 + 0.01)).sum() / (3 * n)
    loss.backward()
    for k in range(5):
        g = ws[k].grad.numpy()
        step = after[k] - before[k]
        big = np.abs(g) > 0.05 * np.abs(g).max()
        agree = np.mean(np.sign(step[big]) == -np.sign(g[big]))
        assert agree > 0.97, (k, agree)
        moved = np.abs(step[big])
        np.testing.assert_allclose(moved, 1e-3, rtol=0.05)


def test_training_reduces_error():
    ctx = bp.LuxContext()
    cache = make_cache(ctx, batch=16384)
    s = random_samples(65536, 3)
    t = field(s)
    d_s, d_t = to_device(s), to_device(t)
    q = random_samples(8192, 4)
    tq = field(q)
    d_q = to_device(q)
    d_out = empty_device(len(q) * 16)

    def error():
        cache.query(d_q.data_ptr(), len(q), d_out.data_ptr())
        ctx.synchronize()
        out = from_device(d_out, np.float32, (len(q), 4))
        return float(np.sqrt(np.mean((out[:, :3] - tq[:, :3]) ** 2)) / np.mean(tq[:, :3]))

    start = error()
    for _ in range(160):
        cache.train(d_s.data_ptr(), d_t.data_ptr(), len(s))
    end = error()
    st = cache.stats()
    assert st.error_flags == 0 and st.steps == 640
    # In-sample fit (queries are training samples): each training position
    # carries one direction, so this checks the optimiser rather than
    # generalisation between scattered samples.
    fit = s[:8192].copy()
    tf = t[:8192]
    d_f = to_device(fit)
    cache.query(d_f.data_ptr(), len(fit), d_out.data_ptr())
    ctx.synchronize()
    out = from_device(d_out, np.float32, (len(fit), 4))
    in_sample = float(np.sqrt(np.mean((out[:, :3] - tf[:, :3]) ** 2)) / np.mean(tf[:, :3]))
    print("relative RMSE before / after training:", start, end, "in-sample", in_sample, "loss", st.last_loss)
    assert in_sample < 0.1 and end < 0.5 * start and st.last_loss < 0.05
