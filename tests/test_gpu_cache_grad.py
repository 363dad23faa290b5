"""Learned radiance cache: gradient values and Adam steps.

The weight and hash-table gradients of one pass (lux_cache_gradients, no
step) against PyTorch autograd of the same loss on the same BF16 encodings,
within BF16 tolerance; then two training steps against torch.optim.Adam (the
weights) and torch.optim.SparseAdam (the hash table, whose entries a step
does not reach keep value and moments) given the same gradients."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from tests.helpers import empty_device, from_device, to_device
from tests.test_gpu_cache import bf16_round, field, make_cache, random_samples

pytestmark = pytest.mark.gpu

GRAD_TOL = 3e-2  # relative L2 error: BF16 operands and BF16 layer gradients, FP32 accumulation


def corners(cache, s):
    """Hash-grid corner indices [n, levels, 8] and trilinear weights (the
    encoding's level_corners / grid_index)."""
    d = cache.desc
    levels, table = int(d.levels), 1 << int(d.log2_table)
    lo, hi = np.full(3, -2.0, np.float32), np.full(3, 2.0, np.float32)
    inv = (np.float32(1.0) / (hi - lo)).astype(np.float32)
    u = np.clip((s["position"].astype(np.float32) - lo) * inv, 0.0, 1.0).astype(np.float32)
    idx = np.zeros((len(s), levels, 8), np.int64)
    wts = np.zeros((len(s), levels, 8), np.float32)
    for level in range(levels):
        res = np.float32(np.floor(float(d.base_resolution) * float(d.growth) ** level))
        p = (u * res).astype(np.float32)
        fl = np.clip(np.floor(p), 0.0, res - 1.0).astype(np.float32)
        f = np.clip(p - fl, 0.0, 1.0).astype(np.float32)
        i0 = fl.astype(np.uint64)
        stride = np.uint64(int(res) + 1)
        for k in range(8):
            c = i0 + np.array([k & 1, (k >> 1) & 1, k >> 2], np.uint64)
            if int(stride) ** 3 <= table:
                g = c[:, 0] + stride * (c[:, 1] + stride * c[:, 2])
            else:
                m = np.uint64(0xFFFFFFFF)
                g = ((c[:, 0] ^ ((c[:, 1] * np.uint64(2654435761)) & m) ^ ((c[:, 2] * np.uint64(805459861)) & m))
                     & np.uint64(table - 1))
            idx[:, level, k] = level * table + g.astype(np.int64)
            a = [f[:, a_] if (k >> a_) & 1 else np.float32(1.0) - f[:, a_] for a_ in range(3)]
            wts[:, level, k] = (a[0] * a[1]) * a[2]
    return idx, wts


def torch_gradients(x_bits, layers, targets, n):
    """Autograd of the relative L2 loss (denominator held constant) with the
    BF16-rounded weights and encodings the kernels use."""
    import torch
    x = torch.from_numpy(x_bits.astype(np.uint32) << 16).view(torch.float32).clone().requires_grad_(True)
    ws = [bf16_round(w).clone().requires_grad_(True) for w in layers]
    h = x
    for k, w in enumerate(ws):
        z = h @ w.T
        h = bf16_round(torch.relu(z)).detach() + torch.relu(z) - torch.relu(z).detach() if k < 4 else z
    y = h[:, :3]
    tt = torch.from_numpy(targets[:, :3])
    loss = (((y - tt) ** 2) / (y.detach() ** 2 + 0.01)).sum() / (3 * n)
    loss.backward()
    return [w.grad.numpy() for w in ws], x.grad.numpy()


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_gradients_match_torch_autograd():
    # 160 tiles of 128 samples over at most 148 CTAs: some CTAs sum two tiles
    # in their tensor-memory weight gradients.
    n = 160 * 128
    ctx = bp.LuxContext()
    cache = make_cache(ctx, batch=n, log2_table=14)
    s = random_samples(n, 5)
    t = field(s)
    d_s, d_t = to_device(s), to_device(t)
    d_x = empty_device(n * 128)
    cache.encode(d_s.data_ptr(), n, d_x.data_ptr())
    ctx.synchronize()
    x_bits = from_device(d_x, np.uint16, (n, 64))
    layers = cache.weights()
    gw, gt = cache.gradients(d_s.data_ptr(), d_t.data_ptr(), n)
    assert cache.stats().error_flags == 0
    ref_w, ref_x = torch_gradients(x_bits, layers, t, n)
    for k in range(5):
        assert rel(gw[k], ref_w[k]) < GRAD_TOL, (k, rel(gw[k], ref_w[k]))
    # Hash table: the input-feature gradients scattered through the corners.
    idx, wts = corners(cache, s)
    levels = int(cache.desc.levels)
    ref_t = np.zeros(gt.size, np.float64)
    g_feat = ref_x[:, :2 * levels].reshape(n, levels, 2)
    for c in range(2):
        contrib = (wts * g_feat[:, :, c:c + 1]).reshape(-1)
        np.add.at(ref_t, idx.reshape(-1) * 2 + c, contrib)
    assert rel(gt.reshape(-1), ref_t) < GRAD_TOL, rel(gt.reshape(-1), ref_t)
    # A second call starts from cleared gradients.
    gw2, gt2 = cache.gradients(d_s.data_ptr(), d_t.data_ptr(), n)
    for k in range(5):
        assert rel(gw2[k], gw[k]) < 1e-3


def test_two_adam_steps_match_torch_optimisers():
    import torch
    n = 4096
    ctx = bp.LuxContext()
    cache = make_cache(ctx, batch=n, log2_table=14, learning_rate=1e-3)
    w0 = [w.copy() for w in cache.weights()]
    t0 = cache.table().copy()
    pw = [torch.nn.Parameter(torch.from_numpy(w.copy())) for w in w0]
    pt = torch.nn.Parameter(torch.from_numpy(t0.reshape(-1).copy()))
    adam = torch.optim.Adam(pw, lr=1e-3, betas=(0.9, 0.99), eps=1e-10)
    sparse = torch.optim.SparseAdam([pt], lr=1e-3, betas=(0.9, 0.99), eps=1e-10)
    smallest = np.full(t0.size, np.inf)  # smallest non-zero |table gradient| over the steps
    for step in range(2):
        s = random_samples(n, 10 + step)
        t = field(s)
        d_s, d_t = to_device(s), to_device(t)
        gw, gt = cache.gradients(d_s.data_ptr(), d_t.data_ptr(), n)
        cache.train(d_s.data_ptr(), d_t.data_ptr(), n)
        for p, g in zip(pw, gw):
            p.grad = torch.from_numpy(g.copy())
        adam.step()
        g = np.abs(gt.reshape(-1))
        smallest = np.where(g > 0, np.minimum(smallest, g), smallest)
        pt.grad = torch.from_numpy(gt.reshape(-1).copy()).to_sparse()
        sparse.step()
    assert cache.stats().error_flags == 0 and cache.stats().steps == 2
    got_w, got_t = cache.weights(), cache.table().reshape(-1)
    for k in range(5):
        dg, dr = got_w[k] - w0[k], pw[k].detach().numpy() - w0[k]
        assert np.abs(dr).max() > 1e-4
        np.testing.assert_allclose(dg, dr, rtol=1e-3, atol=1e-7, err_msg=f"layer {k}")
    dg, dr = got_t - t0.reshape(-1), pt.detach().numpy() - t0.reshape(-1)
    assert np.count_nonzero(dr) > 1000
    # SparseAdam adds eps to sqrt(v) before the sqrt(1 - beta2^t) correction,
    # the kernel after it: a relative difference of about eps / (0.14 |g|), so
    # entries whose every gradient is above 1e-4 compare to 1e-3.
    big = np.isfinite(smallest) & (smallest > 1e-4)
    assert big.sum() > 1000
    np.testing.assert_allclose(dg[big], dr[big], rtol=1e-3, atol=1e-7)
    moved = dr != 0
    assert np.mean(np.sign(dg[moved]) == np.sign(dr[moved])) > 0.999
    assert np.all(dg[~moved] == 0)  # entries no step reached are unchanged
