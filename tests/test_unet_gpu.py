"""The U-Net's forward and backward kernels against torch autograd on the CPU.

The reference network is built in torch (float64 on the CPU) from the library's own parameters,
rounding to BF16 exactly where the device stores BF16 (the weights, the packed input, every
convolution's ReLU output, every pooled tensor). The device also keeps its gradients in BF16
between layers, which the reference does not, so gradients are compared per layer by direction
(cosine) and size (relative norm), with the tolerances written below.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.nn.functional as Fn  # noqa: E402

from deeptime_gpu import unet as U  # noqa: E402

pytestmark = pytest.mark.gpu

LEVELS, BASE, IN_PAD = 4, 32, 32


def layer_table():
    """(cin, cout) of the convolutions in the library's parameter order, then the head."""
    convs = []
    for l in range(LEVELS):
        c = BASE << l
        convs.append((IN_PAD if l == 0 else BASE << (l - 1), c))
        convs.append((c, c))
    for l in range(LEVELS - 2, -1, -1):
        c = BASE << l
        convs.append(((BASE << (l + 1)) + c, c))
        convs.append((c, c))
    return convs


def unpack(params):
    out, off = [], 0
    for cin, cout in layer_table():
        w = params[off:off + 9 * cin * cout].reshape(9, cin, cout)
        off += 9 * cin * cout
        b = params[off:off + cout]
        off += cout
        out.append((w, b))
    hw = params[off:off + BASE]
    hb = params[off + BASE:off + BASE + 1]
    return out, hw, hb


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float64)


def conv(x, w, b):
    # x [N][C][H][W]; w [9][cin][cout] -> OIHW; periodic in x, zero in y
    wt = w.permute(2, 1, 0).reshape(w.shape[2], w.shape[1], 3, 3)
    xp = Fn.pad(x, (1, 1, 0, 0), mode="circular")
    return Fn.conv2d(xp, wt, b, padding=(1, 0))


def reference(params_t, x, t):
    convs, hw, hb = params_t
    convs = [(bf16(w), b) for w, b in convs]
    n, h, w_, _ = x.shape
    inp = torch.zeros((n, IN_PAD, h, w_), dtype=torch.float64)
    inp[:, 0:2] = bf16(x.permute(0, 3, 1, 2))
    skips, cur = [], inp
    for l in range(LEVELS):
        a = bf16(torch.relu(conv(cur, *convs[2 * l])))
        o = bf16(torch.relu(conv(a, *convs[2 * l + 1])))
        if l + 1 < LEVELS:
            skips.append(o)
            cur = bf16(Fn.avg_pool2d(o, 2))
        else:
            cur = o
    for l in range(LEVELS - 2, -1, -1):
        up = Fn.interpolate(cur, scale_factor=2, mode="nearest")
        u = torch.cat([up, skips[l]], dim=1)
        di = 2 * LEVELS + 2 * (LEVELS - 2 - l)
        da = bf16(torch.relu(conv(u, *convs[di])))
        cur = bf16(torch.relu(conv(da, *convs[di + 1])))
    pred = torch.einsum("nchw,c->nhw", cur, hw) + hb[0]
    return torch.mean((pred - t) ** 2)


def test_loss_and_gradients_match_torch_autograd():
    rng = np.random.default_rng(0)
    B, H, W = 2, 16, 512
    model = U.UNet(seed=2024)
    p = model.params()
    assert p.size == model.n_params
    # perturb the biases so every ReLU path is exercised
    x = rng.standard_normal((B, H, W, 2)).astype(np.float32)
    t = rng.standard_normal((B, H, W)).astype(np.float32) * 0.1
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    loss = model.loss_and_grad_dev(xd.data_ptr(), td.data_ptr(), B, H, W)
    g = model.gradients()

    convs, hw, hb = unpack(p.astype(np.float64))
    params_t = ([(torch.tensor(w, requires_grad=True), torch.tensor(b, requires_grad=True)) for w, b in convs],
                torch.tensor(hw, requires_grad=True), torch.tensor(hb, requires_grad=True))
    ref = reference(params_t, torch.from_numpy(x).double(), torch.from_numpy(t).double())
    ref.backward()
    assert abs(loss - ref.item()) <= 2e-3 * abs(ref.item()), (loss, ref.item())

    gc, ghw, ghb = unpack(g.astype(np.float64))
    stats = []
    for k, ((gw, gb), (tw, tb)) in enumerate(zip(gc, params_t[0])):
        rw = tw.grad.numpy()
        if k == 0:  # the padding channels of the input are zero: only channels 0, 1 carry gradient
            gw, rw = gw[:, :2], rw[:, :2]
        cos = float((gw * rw).sum() / (np.linalg.norm(gw) * np.linalg.norm(rw) + 1e-300))
        rel = float(np.linalg.norm(gw - rw) / (np.linalg.norm(rw) + 1e-300))
        rb = tb.grad.numpy()
        relb = float(np.linalg.norm(gb - rb) / (np.linalg.norm(rb) + 1e-12))
        stats.append((k, round(cos, 5), round(rel, 4), round(relb, 4)))
    print(stats)
    # BF16 gradients between layers on the device, exact ones in the reference
    for k, cos, rel, relb in stats:
        assert cos > 0.995 and rel < 0.08 and relb < 0.08, stats
    assert np.linalg.norm(ghw - params_t[1].grad.numpy()) <= 0.02 * np.linalg.norm(params_t[1].grad.numpy())
    assert abs(ghb[0] - params_t[2].grad.numpy()[0]) <= 0.02 * abs(params_t[2].grad.numpy()[0]) + 1e-6


def test_training_reduces_the_loss_and_weights_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    B, H, W = 4, 16, 512
    model = U.UNet(seed=7)
    x = torch.from_numpy(rng.standard_normal((B, H, W, 2)).astype(np.float32)).cuda()
    # a target the network can represent (a function of the input; periodic convolutions cannot
    # learn a target that depends on position alone)
    t = (0.5 * x[..., 0] + 0.25 * x[..., 1]).contiguous()
    first = model.train_step_dev(x.data_ptr(), t.data_ptr(), B, H, W, 1e-3)
    for _ in range(60):
        last = model.train_step_dev(x.data_ptr(), t.data_ptr(), B, H, W, 1e-3)
    assert last < 0.5 * first, (first, last)
    path = str(tmp_path / "w.bin")
    model.save(path)
    other = U.UNet(seed=99)
    other.load(path)
    y1 = torch.empty((1, H, W), device="cuda")
    y2 = torch.empty((1, H, W), device="cuda")
    model.predict_dev(x[0].data_ptr(), y1.data_ptr(), 1, H, W)
    other.predict_dev(x[0].data_ptr(), y2.data_ptr(), 1, H, W)
    assert torch.equal(y1, y2)


def test_the_tensor_memory_path_reproduces_the_default_one(monkeypatch):
    # the tcgen05 convolutions (DT_UNET_TC=1, read when a model is made) against the default
    # mma.sync ones on the same weights: both sum exact BF16 products in FP32 in the same K order
    rng = np.random.default_rng(3)
    B, H, W = 2, 16, 512
    x = torch.from_numpy(rng.standard_normal((B, H, W, 2)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((B, H, W)).astype(np.float32) * 0.1).cuda()
    monkeypatch.setenv("DT_UNET_TC", "1")
    tc = U.UNet(seed=11)
    monkeypatch.setenv("DT_UNET_TC", "0")
    ref = U.UNet(seed=11)
    y1 = torch.empty((B, H, W), device="cuda")
    y2 = torch.empty((B, H, W), device="cuda")
    tc.predict_dev(x.data_ptr(), y1.data_ptr(), B, H, W)
    ref.predict_dev(x.data_ptr(), y2.data_ptr(), B, H, W)
    assert torch.allclose(y1, y2, rtol=1e-3, atol=1e-3 * float(y2.abs().max())), float((y1 - y2).abs().max())
    l1 = tc.loss_and_grad_dev(x.data_ptr(), t.data_ptr(), B, H, W)
    g1 = tc.gradients()
    l2 = ref.loss_and_grad_dev(x.data_ptr(), t.data_ptr(), B, H, W)
    g2 = ref.gradients()
    assert abs(l1 - l2) <= 1e-3 * abs(l2)
    assert np.linalg.norm(g1 - g2) <= 1e-3 * np.linalg.norm(g2)
