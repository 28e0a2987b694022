"""GPU tests of the denoiser's hand-written kernels through the C ABI, each
against a plain PyTorch fp32 reference of the same operation (torch is the
checker only):

- the tensor-core 3x3 convolution (forward, input gradient, ReLU mask, the
  upsample-and-add decoder input) against F.conv2d / conv2d_input on the same
  bf16-rounded operands: max-abs <= 1e-4 relative to the output's scale;
- its weight gradient against conv2d_weight: <= 1e-3 relative;
- the whole network forward against a torch model that rounds its
  activations to bf16 where the kernels store bf16: <= 1e-2 relative;
- the parameter gradients of the whole network against torch autograd through
  the same bf16 forward (error channel detached from the trunk, as in the
  kernels): each layer's relative L2 error <= 3e-2 (the kernels also store the
  gradients of the activations in bf16);
- the L1 + SSIM + error-head loss and its gradient: value within 1e-4, the
  bf16 gradient within 1e-2 relative;
- Adam against torch.optim.Adam: 1e-6 relative;
- a few hundred training steps on a fixed batch lower the loss.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gamesplat_b200 import _lib as L
from gamesplat_b200 import denoiser as DN

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
F = torch.nn.functional


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _bf(t):
    return t.bfloat16().float()


def _conv_ref(x_nhwc, w, b=None):
    """3x3 same convolution in fp32; x NHWC float, w [3,3,cin,cout]."""
    y = F.conv2d(x_nhwc.permute(0, 3, 1, 2), w.permute(3, 2, 0, 1), b, padding=1)
    return y.permute(0, 2, 3, 1)


def _up2(t_nhwc, h=None, w=None):
    """Nearest 2x upsample to h x w; an odd size's last row / column repeats
    the last half-resolution one."""
    up = t_nhwc.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)
    h = h or up.shape[1]
    w = w or up.shape[2]
    if h > up.shape[1]:
        up = torch.cat([up, up[:, -1:]], dim=1)
    if w > up.shape[2]:
        up = torch.cat([up, up[:, :, -1:]], dim=2)
    return up


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
@pytest.mark.parametrize("relu,masked", [(0, 0), (1, 1)])
def test_conv_forward_matches_torch(cin, cout, relu, masked):
    g = torch.Generator(device="cuda").manual_seed(cin * 7 + cout + relu)
    n, h, w = 2, 6, 200   # a full and a partial 128-pixel strip
    x = torch.randn(n, h, w, cin, device="cuda", generator=g).bfloat16()
    wt = (torch.randn(3, 3, cin, cout, device="cuda", generator=g) * 0.2).float()
    b = torch.randn(cout, device="cuda", generator=g).float()
    mask = torch.randn(n, h, w, cout, device="cuda", generator=g).bfloat16() if masked else None
    out = torch.zeros(n, h, w, cout, device="cuda")
    out16 = torch.zeros(n, h, w, cout, device="cuda", dtype=torch.bfloat16)
    scratch = torch.empty(L.lib().gs_conv3x3_scratch_bytes(cin, cout), dtype=torch.uint8, device="cuda")
    err = torch.zeros(4, dtype=torch.int32, device="cuda")
    st = L.lib().gs_conv3x3_bf16(_p(x), None, n, h, w, cin, cout, _p(wt), _p(b), relu, 0, _p(mask), _p(out16),
                                 _p(out), _p(scratch), _p(err), None)
    L.check(st, "gs_conv3x3_bf16")
    torch.cuda.synchronize()
    ref = _conv_ref(x.float(), _bf(wt), b)
    if relu:
        ref = ref.clamp_min(0)
    if masked:
        ref = torch.where(mask.float() > 0, ref, torch.zeros_like(ref))
    scale = float(ref.abs().max())
    assert int(err[0]) == 0
    assert float((out - ref).abs().max()) <= 1e-4 * scale + 1e-6
    assert float((out16.float() - ref).abs().max()) <= 8e-3 * scale


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32)])
def test_conv_input_gradient_matches_torch(cin, cout):
    """transposed = 1: the input gradient of a (cin -> cout) layer."""
    g = torch.Generator(device="cuda").manual_seed(11 + cin)
    n, h, w = 2, 5, 150
    dy = torch.randn(n, h, w, cout, device="cuda", generator=g).bfloat16()
    wt = (torch.randn(3, 3, cin, cout, device="cuda", generator=g) * 0.2).float()
    out = torch.zeros(n, h, w, cin, device="cuda")
    scratch = torch.empty(L.lib().gs_conv3x3_scratch_bytes(cin, cout), dtype=torch.uint8, device="cuda")
    err = torch.zeros(4, dtype=torch.int32, device="cuda")
    L.check(L.lib().gs_conv3x3_bf16(_p(dy), None, n, h, w, cin, cout, _p(wt), None, 0, 1, None, None, _p(out),
                                    _p(scratch), _p(err), None), "gs_conv3x3_bf16")
    torch.cuda.synchronize()
    ref = torch.nn.grad.conv2d_input((n, cin, h, w), _bf(wt).permute(3, 2, 0, 1), dy.float().permute(0, 3, 1, 2),
                                     padding=1).permute(0, 2, 3, 1)
    assert float((out - ref).abs().max()) <= 1e-4 * float(ref.abs().max()) + 1e-6


@pytest.mark.parametrize("n,h,w", [(1, 8, 260), (2, 9, 301)])
def test_conv_upsample_add_input_matches_torch(n, h, w):
    """x_half: the decoder input up2(x_half) + x, rounded to bf16 as the kernel stores it."""
    g = torch.Generator(device="cuda").manual_seed(5 + w)
    x = torch.randn(n, h, w, 32, device="cuda", generator=g).bfloat16()
    xh = torch.randn(n, h // 2, w // 2, 32, device="cuda", generator=g).bfloat16()
    wt = (torch.randn(3, 3, 32, 32, device="cuda", generator=g) * 0.2).float()
    out = torch.zeros(n, h, w, 32, device="cuda")
    scratch = torch.empty(L.lib().gs_conv3x3_scratch_bytes(32, 32), dtype=torch.uint8, device="cuda")
    err = torch.zeros(4, dtype=torch.int32, device="cuda")
    L.check(L.lib().gs_conv3x3_bf16(_p(x), _p(xh), n, h, w, 32, 32, _p(wt), None, 0, 0, None, None, _p(out),
                                    _p(scratch), _p(err), None), "gs_conv3x3_bf16")
    torch.cuda.synchronize()
    ref = _conv_ref(_bf(x.float() + _up2(xh.float(), h, w)), _bf(wt))
    assert float((out - ref).abs().max()) <= 1e-4 * float(ref.abs().max()) + 1e-6


@pytest.mark.parametrize("cin,cout,half", [(16, 32, False), (32, 32, False), (32, 16, False), (32, 32, True)])
def test_conv_weight_gradient_matches_torch(cin, cout, half):
    g = torch.Generator(device="cuda").manual_seed(cin + 3 * cout + int(half))
    n, h, w = 2, 6, 136   # two full 64-pixel blocks and a partial one per row
    x = torch.randn(n, h, w, cin, device="cuda", generator=g).bfloat16()
    xh = torch.randn(n, h // 2, w // 2, cin, device="cuda", generator=g).bfloat16() if half else None
    dy = torch.randn(n, h, w, cout, device="cuda", generator=g).bfloat16()
    dw = torch.zeros(3, 3, cin, cout, device="cuda")
    db = torch.zeros(cout, device="cuda")
    err = torch.zeros(4, dtype=torch.int32, device="cuda")
    L.check(L.lib().gs_conv3x3_wgrad_bf16(_p(x), _p(xh), n, h, w, cin, cout, _p(dy), _p(dw), _p(db), _p(err), None),
            "gs_conv3x3_wgrad_bf16")
    torch.cuda.synchronize()
    xin = _bf(x.float() + _up2(xh.float())) if half else x.float()
    ref = torch.nn.grad.conv2d_weight(xin.permute(0, 3, 1, 2), (cout, cin, 3, 3), dy.float().permute(0, 3, 1, 2),
                                      padding=1).permute(2, 3, 1, 0)
    assert int(err[0]) == 0
    assert float((dw - ref).abs().max()) <= 1e-3 * float(ref.abs().max())
    dbr = dy.float().sum(dim=(0, 1, 2))
    assert float((db - dbr).abs().max()) <= 1e-3 * float(dbr.abs().max())


def _torch_net(x, flat, emulate_bf16=True):
    """The denoiser in torch fp32 (NHWC in, NHWC out); activations rounded to
    bf16 where the kernels store bf16."""
    r = _bf if emulate_bf16 else (lambda t: t)
    layers = [(torch.as_tensor(w, device="cuda"), torch.as_tensor(b, device="cuda"))
              for w, b in DN.split_params(flat)]
    e1 = r(_conv_ref(x, *layers[0]).clamp_min(0))
    p1 = r(F.avg_pool2d(e1.permute(0, 3, 1, 2), 2).permute(0, 2, 3, 1))
    e2 = r(_conv_ref(p1, *layers[1]).clamp_min(0))
    e3 = r(_conv_ref(e2, *layers[2]).clamp_min(0))
    u = r(_up2(e3) + e1)
    d4 = r(_conv_ref(u, *layers[3]).clamp_min(0))
    return _conv_ref(d4, *layers[4])


def _features(n, h, w, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.zeros(n, h, w, 16, device="cuda")
    x[..., :8] = torch.rand(n, h, w, 8, device="cuda", generator=g)
    return x.bfloat16()


def _random_params(seed):
    rng = np.random.default_rng(seed)
    flat = []
    for cin, cout in DN.LAYERS:
        flat.append(rng.normal(0, np.sqrt(2.0 / (9 * cin)), 9 * cin * cout))
        flat.append(rng.normal(0, 0.05, cout))
    return np.concatenate(flat).astype(np.float32)


def test_network_forward_and_backward_match_torch():
    n, h, w = 2, 20, 136
    x = _features(n, h, w, 1)
    flat = _random_params(2)
    # the kernels compute with bf16 weights (and fp32 biases): give torch the same values
    flat_bf = flat.copy()
    o = 0
    for cin, cout in DN.LAYERS:
        k = 9 * cin * cout
        flat_bf[o:o + k] = torch.from_numpy(flat[o:o + k]).bfloat16().float().numpy()
        o += k + cout
    out = torch.zeros(n, h, w, 16, device="cuda")
    with DN.Denoiser(0) as d:
        d.set_params(flat)
        d.forward(x.data_ptr(), n, h, w, out.data_ptr())
        torch.cuda.synchronize()
        ref = _torch_net(x.float(), flat_bf)
        assert float((out - ref).abs().max()) <= 1e-2 * float(ref.abs().max())
        g = torch.Generator(device="cuda").manual_seed(3)
        dout = torch.randn(n, h, w, 16, device="cuda", generator=g).bfloat16()
        d.backward(x.data_ptr(), dout.data_ptr(), n, h, w)
        grads = d.grads()
        d.status()
    params = [(torch.tensor(wv, device="cuda", requires_grad=True), torch.tensor(bv, device="cuda",
                                                                                requires_grad=True))
              for wv, bv in DN.split_params(flat_bf)]
    layers = params

    def net(xx):
        # the kernels' forward: activations stored in bf16 (so the ReLU masks are the kernels'
        # masks; with an fp32 forward ~0.2 % of them flip, which moves a random-sign gradient
        # sum by ~sqrt(0.2 %) = 5 %), and the error channel 4 trained by the last layer only
        e1 = _bf(_conv_ref(xx, *layers[0]).clamp_min(0))
        p1 = _bf(F.avg_pool2d(e1.permute(0, 3, 1, 2), 2).permute(0, 2, 3, 1))
        e2 = _bf(_conv_ref(p1, *layers[1]).clamp_min(0))
        e3 = _bf(_conv_ref(e2, *layers[2]).clamp_min(0))
        d4 = _bf(_conv_ref(_bf(_up2(e3) + e1), *layers[3]).clamp_min(0))
        o = _conv_ref(d4, *layers[4])
        o_err = _conv_ref(d4.detach(), *layers[4])
        return torch.cat([o[..., :4], o_err[..., 4:5], o[..., 5:]], dim=-1)

    (net(x.float()) * dout.float()).sum().backward()
    got = DN.split_params(grads)
    errs = []
    for (gw, gb), (pw, pb) in zip(got, params):
        rw = pw.grad.cpu().numpy()
        rb = pb.grad.cpu().numpy()
        errs.append((float(np.linalg.norm(gw - rw) / np.linalg.norm(rw)),
                     float(np.linalg.norm(gb - rb) / max(np.linalg.norm(rb), 1e-12))))
    assert all(ew <= 3e-2 and eb <= 3e-2 for ew, eb in errs), errs


def _torch_loss(out, x, target, ssim_w, err_w):
    pred = torch.cat([x[..., 5:8].float() + out[..., 0:3], x[..., 3:4].float() + out[..., 3:4]], dim=-1)
    d = pred - target
    l1 = d.abs().mean()
    e = (d.detach() ** 2).mean(dim=-1)
    le = ((out[..., 4] - 1000.0 * e) ** 2).mean()
    k = torch.exp(-torch.arange(-5, 6, device="cuda", dtype=torch.float32) ** 2 / (2 * 1.5 ** 2))
    k = k / k.sum()

    def blur(t):   # NHWC, per channel, zero padding
        c = t.shape[-1]
        tt = t.permute(0, 3, 1, 2)
        tt = F.conv2d(tt, k.view(1, 1, 1, 11).repeat(c, 1, 1, 1), padding=(0, 5), groups=c)
        tt = F.conv2d(tt, k.view(1, 1, 11, 1).repeat(c, 1, 1, 1), padding=(5, 0), groups=c)
        return tt.permute(0, 2, 3, 1)

    p, t = pred[..., :3], target[..., :3]
    mx, my = blur(p), blur(t)
    sxx, syy, sxy = blur(p * p) - mx * mx, blur(t * t) - my * my, blur(p * t) - mx * my
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    s = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
    ssim = s[:, 5:-5, 5:-5, :].mean()
    return l1 + ssim_w * (1 - ssim) + err_w * le, l1, ssim, le


def test_loss_and_gradient_match_torch():
    n, h, w = 2, 24, 40
    g = torch.Generator(device="cuda").manual_seed(9)
    x = _features(n, h, w, 4)
    out = (torch.randn(n, h, w, 16, device="cuda", generator=g) * 0.1).float()
    target = torch.rand(n, h, w, 4, device="cuda", generator=g).float()
    dout = torch.zeros(n, h, w, 16, device="cuda", dtype=torch.bfloat16)
    with DN.Denoiser(0) as d:
        parts = d.loss(x.data_ptr(), out.data_ptr(), target.data_ptr(), n, h, w, dout.data_ptr(), 0.2, 0.01)
    o = out.clone().requires_grad_(True)
    total, l1, ssim, le = _torch_loss(o, x, target, 0.2, 0.01)
    total.backward()
    assert abs(parts[0] - float(l1)) <= 1e-5
    assert abs(parts[1] - float(ssim)) <= 1e-4
    assert abs(parts[2] - float(le)) <= 1e-4 * max(1.0, float(le))
    assert abs(parts[3] - float(total)) <= 1e-4 * max(1.0, float(total))
    ref = o.grad[..., :5]
    got = dout.float()[..., :5]
    assert float((got - ref).abs().max()) <= 1e-2 * float(ref.abs().max())
    assert float(dout.float()[..., 5:].abs().max()) == 0.0


def test_adam_matches_torch():
    n, h, w = 1, 16, 64
    x = _features(n, h, w, 6)
    flat = _random_params(7)
    g = torch.Generator(device="cuda").manual_seed(8)
    dout = torch.randn(n, h, w, 16, device="cuda", generator=g).bfloat16()
    with DN.Denoiser(0) as d:
        d.set_params(flat)
        p = torch.tensor(flat, device="cuda", requires_grad=True)
        opt = torch.optim.Adam([p], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
        for _ in range(3):
            d.forward(x.data_ptr(), n, h, w, 0)
            d.backward(x.data_ptr(), dout.data_ptr(), n, h, w)
            gr = d.grads()
            d.adam(1e-3)
            p.grad = torch.tensor(gr, device="cuda")
            opt.step()
            got = d.params()
            ref = p.detach().cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-6 * max(1.0, np.abs(ref).max())
            d.set_params(ref)   # continue from the same parameters (resets the moments on both sides)
            opt = torch.optim.Adam([p], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)


def test_training_lowers_the_loss():
    n, h, w = 4, 32, 64
    x = _features(n, h, w, 10)
    # target: a smooth function of the noisy inputs the network can learn
    xf = x.float()
    target = torch.stack([0.5 * xf[..., 0] + 0.5 * xf[..., 5], 0.5 * xf[..., 1] + 0.5 * xf[..., 6],
                          0.5 * xf[..., 2] + 0.5 * xf[..., 7], xf[..., 3]], dim=-1).contiguous()
    with DN.Denoiser(0) as d:
        d.init_params(3)
        first = d.train_step(x.data_ptr(), target.data_ptr(), n, h, w, 2e-3)[3]
        for _ in range(300):
            d.train_step(x.data_ptr(), target.data_ptr(), n, h, w, 2e-3, want_loss=False)
        last = d.train_step(x.data_ptr(), target.data_ptr(), n, h, w, 2e-3)[3]
    assert np.isfinite(first) and np.isfinite(last)
    assert last < 0.5 * first, (first, last)
