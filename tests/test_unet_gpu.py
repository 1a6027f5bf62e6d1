"""Tensor-core 3x3 convolution and the full denoiser on the GPU, checked
against PyTorch FP32 references (oracle/unet_ref.py):

* one layer: the kernel's BF16 output vs conv2d in FP32 on the same BF16-
  rounded inputs/weights, rounded to BF16 -- differences come only from FP32
  summation order, so >= 99.9% of values must agree within 1 BF16 ulp;
* the whole UNet: vs the same network with BF16 rounding at the kernels'
  rounding points (tight), and vs the plain FP32 network (the precision cost
  of BF16, reported and bounded)."""
import ctypes as C

import numpy as np
import pytest

import lumina
from lumina import _ffi

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
F = torch.nn.functional

import unet_ref  # noqa: E402


def q(t):
    return t.to(torch.bfloat16).to(torch.float32)


def blocked(x, cpad):
    n, c, h, w = x.shape
    out = torch.zeros(n * cpad * h * w, dtype=torch.bfloat16, device="cuda")
    _ffi.check(_ffi.lib().lg_to_blocked_bf16(C.c_void_p(x.data_ptr()), n, c, h, w, C.c_void_p(out.data_ptr()),
                                            cpad, None))
    return out


def unblock(buf, n, c, h, w):
    out = torch.empty((n, c, h, w), dtype=torch.float32, device="cuda")
    _ffi.check(_ffi.lib().lg_from_blocked_bf16(C.c_void_p(buf.data_ptr()), n, c, h, w, C.c_void_p(out.data_ptr()),
                                              None))
    torch.cuda.synchronize()
    return out


def close_frac(got, ref):
    ulp = 2.0 ** -7  # BF16 has 8 significant bits
    ok = (got - ref).abs() <= ulp * ref.abs() + 1e-6
    return float(ok.float().mean())


@pytest.mark.parametrize("cin_real,cin,cout,n,h,w", [
    (3, 16, 32, 1, 16, 40),
    (32, 32, 32, 2, 10, 130),
    (32, 32, 64, 1, 8, 24),
    (64, 64, 128, 1, 6, 200),
    (128, 128, 256, 1, 4, 16),
    (384, 384, 128, 1, 4, 24),
    (192, 192, 64, 2, 8, 8),
    (96, 96, 32, 1, 9, 33),
])
def test_conv_layer_matches_torch(cin_real, cin, cout, n, h, w):
    g = torch.Generator(device="cpu").manual_seed(cin * 7 + cout)
    x = torch.rand((n, cin_real, h, w), generator=g).cuda()
    wt = (torch.randn((cout, cin_real, 3, 3), generator=g) * (2.0 / (cin_real * 9)) ** 0.5).cuda()
    b = (torch.rand((cout,), generator=g) * 0.1 - 0.05).cuda()
    xin = blocked(x, cin)
    out_c, coff = cout + 32, 16  # write into a wider buffer at an offset (concat by addressing)
    out = torch.zeros(n * out_c * h * w, dtype=torch.bfloat16, device="cuda")
    pool = (h % 2 == 0) and (w % 2 == 0)
    out2 = torch.zeros(n * cout * (h // 2) * (w // 2), dtype=torch.bfloat16, device="cuda") if pool else None
    _ffi.check(_ffi.lib().lg_conv3x3_device(
        C.c_void_p(xin.data_ptr()), n, cin, h, w, C.c_void_p(wt.data_ptr()), cin_real, C.c_void_p(b.data_ptr()), cout,
        0.1, 0, C.c_void_p(out.data_ptr()), out_c, coff, C.c_void_p(out2.data_ptr()) if pool else None, cout, 0, None))
    got = unblock(out, n, out_c, h, w)[:, coff:coff + cout]
    ref = q(F.leaky_relu(F.conv2d(q(x), q(wt), b, padding=1), 0.1))
    assert close_frac(got, ref) >= 0.999
    assert float((got - ref).abs().max()) < 0.05
    # The error of the BF16 result against the FP64 host conv of the unrounded operands (the precision
    # statement): BF16 inputs, weights and output each carry up to 2^-9 relative rounding.
    ref64 = F.leaky_relu(F.conv2d(x.cpu().double(), wt.cpu().double(), b.cpu().double(), padding=1), 0.1)
    err = (got.cpu().double() - ref64).abs()
    rel_mean = float(err.mean() / ref64.abs().mean())
    rel_max = float(err.max() / ref64.abs().max())
    print(f"conv {cin_real}->{cout} at {n}x{h}x{w} vs FP64: mean |err| / mean |y| = {rel_mean:.2e}, "
          f"max |err| / max |y| = {rel_max:.2e}")
    assert rel_mean < 2.0 ** -7 and rel_max < 2.0 ** -5
    untouched = unblock(out, n, out_c, h, w)[:, :coff]
    assert float(untouched.abs().max()) == 0.0
    if pool:
        gp = unblock(out2, n, cout, h // 2, w // 2)
        assert close_frac(gp, F.max_pool2d(ref, 2)) >= 0.999


def test_conv_upsample_epilogue():
    n, cin, cout, h, w = 1, 64, 64, 6, 20
    g = torch.Generator(device="cpu").manual_seed(5)
    x = torch.rand((n, cin, h, w), generator=g).cuda()
    wt = (torch.randn((cout, cin, 3, 3), generator=g) * 0.05).cuda()
    b = torch.zeros(cout).cuda()
    xin = blocked(x, cin)
    out_c = 192
    out = torch.zeros(n * out_c * 2 * h * 2 * w, dtype=torch.bfloat16, device="cuda")
    _ffi.check(_ffi.lib().lg_conv3x3_device(
        C.c_void_p(xin.data_ptr()), n, cin, h, w, C.c_void_p(wt.data_ptr()), cin, C.c_void_p(b.data_ptr()), cout, 0.1,
        1, C.c_void_p(out.data_ptr()), out_c, 64, None, 0, 0, None))
    got = unblock(out, n, out_c, 2 * h, 2 * w)[:, 64:128]
    ref = F.interpolate(q(F.leaky_relu(F.conv2d(q(x), q(wt), b, padding=1), 0.1)), scale_factor=2, mode="nearest")
    assert close_frac(got, ref) >= 0.999


# Decoder blocks whose first conv folds its upsampled input in inference (default tiles: all three).
FOLD_ALL = ("u3", "u2", "u1")


def _folded_blocks(tiles):
    """The blocks lg_unet folds for a tile list (kernel choices 6 and 7 with the compiled shapes)."""
    def folds(t):
        return (t[3] == 7 and tuple(t[:3]) == (32, 32, 2)) or (t[3] == 6 and tuple(t[:3]) in ((64, 32, 2), (32, 32, 3)))
    return tuple(b for b, i in (("u3", 8), ("u2", 10), ("u1", 12)) if folds(tiles[i]))


@pytest.mark.parametrize("fold", [True, False])
@pytest.mark.parametrize("n,h,w,in_ch", [(2, 32, 48, 3), (1, 64, 136, 3), (2, 32, 48, 12)])
def test_unet_forward_matches_torch(n, h, w, in_ch, fold):
    """Inference forward against the BF16-emulated restatement (same roundings, FP32 sums), with the
    folded-upsampling form of u3a/u2a/u1a (default) and without; and against the plain network in FP32 and
    in FP64 (the host oracle of the precision statement)."""
    flat = unet_ref.make_params(77, unet_ref.UNetRef(in_ch=in_ch))
    net = lumina.UNet(in_ch=in_ch)
    net.set_params(flat)
    net.set_fold_upsampling(fold)
    assert np.array_equal(net.get_params(), flat)
    x = np.random.default_rng(3).uniform(0, 1, (n, in_ch, h, w)).astype(np.float32)
    y = net.forward(x)
    assert y.shape == (n, 3, h, w)
    m = unet_ref.load_flat(unet_ref.UNetRef(in_ch=in_ch).eval(), flat)
    fb = FOLD_ALL if fold else ()
    with torch.no_grad():
        ref_q = unet_ref.forward_bf16(m, torch.from_numpy(x), fold=fb).numpy()
        ref_q64 = unet_ref.forward_bf16(m, torch.from_numpy(x), torch.float64, fold=fb).numpy()
        ref_f = m(torch.from_numpy(x)).numpy()
        ref_64 = m.double()(torch.from_numpy(x).double()).numpy()  # FP64 host network, unrounded weights
    err_q = np.abs(y - ref_q)
    err_f = np.abs(y - ref_f)
    err_64 = np.abs(y - ref_64)
    # Noise floor: the same BF16-rounded network summed in FP32 vs FP64 already
    # differs this much (a different summation order flips BF16 roundings).
    floor = np.abs(ref_q - ref_q64)
    print(f"UNet {n}x{h}x{w} fold={fold}: vs BF16-emulated max {err_q.max():.2e} mean {err_q.mean():.2e} "
          f"(floor max {floor.max():.2e} mean {floor.mean():.2e}); vs FP32 max {err_f.max():.2e} "
          f"mean {err_f.mean():.2e}; vs FP64 max {err_64.max():.2e} mean {err_64.mean():.2e}")
    assert err_64.mean() < 5e-3 and err_64.max() < 0.1
    assert err_q.mean() <= 2.0 * floor.mean() + 1e-4
    assert err_q.max() <= 2.0 * floor.max() + 2e-3
    assert err_f.mean() < 5e-3 and err_f.max() < 0.1


def test_unet_rejects_bad_size():
    net = lumina.UNet()
    with pytest.raises(lumina.LuminaError):
        net.forward(np.zeros((1, 3, 12, 16), np.float32))


def _batch(n, h, w, seed, in_ch=3):
    rng = np.random.default_rng(seed)
    clean = rng.uniform(0.1, 0.9, (n, 3, h, w)).astype(np.float32)
    noisy = np.clip(clean + rng.normal(0, 0.1, clean.shape), 0, 1).astype(np.float32)
    if in_ch > 3:  # auxiliary planes (G-buffer stand-ins) after the colour
        aux = rng.uniform(0, 1, (n, in_ch - 3, h, w)).astype(np.float32)
        noisy = np.concatenate([noisy, aux], axis=1)
    return noisy, clean


@pytest.mark.parametrize("in_ch", [3, 12])
def test_unet_gradients_match_torch_autograd(in_ch):
    """Gradients of the mean L1 loss from the project's backward kernels vs
    torch autograd through the FP32 network, per parameter tensor."""
    flat = unet_ref.make_params(21, unet_ref.UNetRef(in_ch=in_ch))
    net = lumina.UNet(in_ch=in_ch)
    net.set_params(flat)
    n, h, w = 2, 32, 48
    noisy, clean = _batch(n, h, w, 4, in_ch)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
    m = unet_ref.load_flat(unet_ref.UNetRef(in_ch=in_ch), flat)
    out = m(torch.from_numpy(noisy))
    ref_loss = F.l1_loss(out, torch.from_numpy(clean))
    ref_loss.backward()
    assert abs(loss - float(ref_loss.detach())) < 2e-3 * max(1.0, float(ref_loss.detach()))
    off = 0
    worst = []
    for k, p in m.named_parameters():
        gn = g[off:off + p.numel()]
        off += p.numel()
        gr = p.grad.numpy().ravel()
        cos = float(np.dot(gn, gr) / (np.linalg.norm(gn) * np.linalg.norm(gr) + 1e-30))
        rel = float(np.linalg.norm(gn - gr) / (np.linalg.norm(gr) + 1e-30))
        worst.append((cos, rel, k))
    worst.sort()
    print("worst parameter tensors (cosine, relative L2 error):", worst[:4])
    assert all(c > 0.98 and r < 0.25 for c, r, _ in worst), worst[:4]


def _grad_errors(flat, g, model, noisy, clean, dtype):
    """Per-tensor (cosine, relative L2) of the kernels' gradients g against
    autograd through unet_ref.forward_bf16 in `dtype`."""
    m = unet_ref.load_flat(model, flat).to(dtype)
    out = unet_ref.forward_bf16(m, torch.from_numpy(noisy), dtype=dtype)
    F.l1_loss(out, torch.from_numpy(clean).to(dtype)).backward()
    off, res = 0, {}
    for k, p in m.named_parameters():
        gn = g[off:off + p.numel()].astype(np.float64)
        off += p.numel()
        gr = p.grad.double().numpy().ravel()
        cos = float(np.dot(gn, gr) / (np.linalg.norm(gn) * np.linalg.norm(gr) + 1e-30))
        rel = float(np.linalg.norm(gn - gr) / (np.linalg.norm(gr) + 1e-30))
        res[k] = (cos, rel)
    return res


@pytest.mark.parametrize("in_ch", [3, 12])
def test_unet_gradients_match_bf16_emulated_autograd(in_ch):
    """Gradients vs autograd through the BF16-emulated restatement, which
    rounds activations and weights where the kernels do, and (through the
    casts' backward) the activation gradients where the kernels store them.
    The emulation in FP32 against the same emulation in FP64 gives the noise
    floor of that rounding (a value near a BF16 rounding boundary can go
    either way); per tensor the kernels' relative L2 error against the FP64
    emulation must stay within 3x that floor + 1%, and the cosine above
    0.998."""
    model = lambda: unet_ref.UNetRef(in_ch=in_ch)
    flat = unet_ref.make_params(21, model())
    net = lumina.UNet(in_ch=in_ch)
    net.set_params(flat)
    n, h, w = 2, 32, 48
    noisy, clean = _batch(n, h, w, 4, in_ch)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    _, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
    ours = _grad_errors(flat, g, model(), noisy, clean, torch.float64)
    g32 = np.concatenate([p.ravel() for p in _autograd_bf16(flat, model(), noisy, clean, torch.float32)])
    floor = _grad_errors(flat, g32, model(), noisy, clean, torch.float64)
    worst = sorted(((ours[k][1] - 3 * floor[k][1], ours[k], floor[k], k) for k in ours), reverse=True)
    print("worst tensors (excess, (cos, rel) ours vs emulation, (cos, rel) FP32 vs FP64 emulation):", worst[:4])
    for _, (cos, rel), (_, frel), k in worst:
        assert cos > 0.998 and rel <= 3 * frel + 0.01, (k, cos, rel, frel)


def _autograd_bf16(flat, model, noisy, clean, dtype):
    m = unet_ref.load_flat(model, flat).to(dtype)
    out = unet_ref.forward_bf16(m, torch.from_numpy(noisy), dtype=dtype)
    F.l1_loss(out, torch.from_numpy(clean).to(dtype)).backward()
    return [p.grad.double().numpy().ravel() for p in m.parameters()]


def test_unet_adam_step_and_training_reduces_loss():
    flat = unet_ref.make_params(22)
    net = lumina.UNet()
    net.set_params(flat)
    n, h, w = 4, 32, 32
    noisy, clean = _batch(n, h, w, 5)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    lr = 1e-3
    # Two Adam steps on the kernels' own gradients vs torch.optim.Adam on the same gradients.
    p_t = torch.nn.Parameter(torch.from_numpy(flat.copy()))
    opt = torch.optim.Adam([p_t], lr=lr)
    for _ in range(2):
        l0, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
        net.adam_apply(lr)
        p_t.grad = torch.from_numpy(g)
        opt.step()
        assert np.allclose(net.get_params(), p_t.detach().numpy(), rtol=1e-5, atol=1e-6)
    losses = [l0] + [net.train_step(dx.data_ptr(), dt.data_ptr(), n, h, w, lr) for _ in range(30)]
    print("training losses:", [round(x, 4) for x in losses[::5]])
    assert losses[-1] < 0.7 * losses[0]


def test_denoise_rgb8_gbuffer_variant():
    """12-channel network through denoise_rgb8: colour + albedo + normal + position u8 planes."""
    flat = unet_ref.make_params(31, unet_ref.UNetRef(in_ch=12))
    net = lumina.UNet(in_ch=12)
    net.set_params(flat)
    rng = np.random.default_rng(2)
    imgs = [rng.integers(0, 256, (20, 27, 3), dtype=np.uint8) for _ in range(4)]
    got = net.denoise_rgb8(*imgs)
    x = np.concatenate([i.astype(np.float32) / 255.0 for i in imgs], axis=2).transpose(2, 0, 1)[None]
    x = F.pad(torch.from_numpy(x), (0, 5, 0, 4), mode="replicate")
    m = unet_ref.load_flat(unet_ref.UNetRef(in_ch=12).eval(), flat)
    with torch.no_grad():
        y = unet_ref.forward_bf16(m, x, fold=FOLD_ALL)[0, :, :20, :27].numpy().transpose(1, 2, 0)
    ref = (np.clip(y, 0, 1) * 255.0 + 0.5).astype(np.uint8)
    diff = np.abs(got.astype(int) - ref.astype(int))
    assert diff.max() <= 6 and np.mean(diff <= 1) > 0.95
    with pytest.raises(AssertionError):
        net.denoise_rgb8(imgs[0])


def _hdr_batch(n, h, w, seed, in_ch=3):
    """Linear radiance with a long tail (as path-traced frames have) and a cleaner target."""
    rng = np.random.default_rng(seed)
    clean = rng.exponential(0.6, (n, 3, h, w)).astype(np.float32)
    noisy = (clean * rng.gamma(4.0, 0.25, clean.shape)).astype(np.float32)
    return noisy, clean


@pytest.mark.parametrize("n,h,w", [(2, 32, 48), (1, 24, 136)])
def test_unet_hdr_variant_forward_matches_torch(n, h, w):
    """ReLU + bilinear upsampling + log1p/expm1 HDR I/O vs the torch restatement
    with BF16 rounding at the kernels' rounding points, compared in log space."""
    m = unet_ref.UNetRef(variant="hdr").eval()
    flat = unet_ref.make_params(78, m)
    unet_ref.load_flat(m, flat)
    net = lumina.UNet(variant="hdr")
    net.set_params(flat)
    x, _ = _hdr_batch(n, h, w, 6)
    y = net.forward(x)
    with torch.no_grad():
        ref_q = unet_ref.forward_bf16(m, torch.from_numpy(x)).numpy()
        ref_q64 = unet_ref.forward_bf16(m, torch.from_numpy(x), torch.float64).numpy()
        ref_f = m(torch.from_numpy(x)).numpy()
    L = np.log1p
    err_q, floor = np.abs(L(y) - L(ref_q)), np.abs(L(ref_q) - L(ref_q64))
    err_f = np.abs(L(y) - L(ref_f))
    print(f"HDR UNet {n}x{h}x{w} (log space): vs BF16-emulated max {err_q.max():.2e} mean {err_q.mean():.2e} "
          f"(floor max {floor.max():.2e} mean {floor.mean():.2e}); vs FP32 max {err_f.max():.2e} mean {err_f.mean():.2e}")
    assert (y >= 0).all()
    assert err_q.mean() <= 2.0 * floor.mean() + 1e-4
    assert err_q.max() <= 2.0 * floor.max() + 2e-3
    assert err_f.mean() < 5e-3 and err_f.max() < 0.1


def test_unet_hdr_variant_gradients_match_torch_autograd():
    m = unet_ref.UNetRef(variant="hdr")
    flat = unet_ref.make_params(23, m)
    unet_ref.load_flat(m, flat)
    net = lumina.UNet(variant="hdr")
    net.set_params(flat)
    n, h, w = 2, 32, 48
    noisy, clean = _hdr_batch(n, h, w, 7)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
    ref_loss = unet_ref.hdr_loss(m, torch.from_numpy(noisy), torch.from_numpy(clean))
    ref_loss.backward()
    assert abs(loss - float(ref_loss.detach())) < 2e-3 * max(1.0, float(ref_loss.detach()))
    off, worst = 0, []
    for k, p in m.named_parameters():
        gn = g[off:off + p.numel()]
        off += p.numel()
        gr = p.grad.numpy().ravel()
        cos = float(np.dot(gn, gr) / (np.linalg.norm(gn) * np.linalg.norm(gr) + 1e-30))
        rel = float(np.linalg.norm(gn - gr) / (np.linalg.norm(gr) + 1e-30))
        worst.append((cos, rel, k))
    worst.sort()
    print("HDR variant, worst parameter tensors (cosine, relative L2 error):", worst[:4])
    assert all(c > 0.98 and r < 0.25 for c, r, _ in worst), worst[:4]
    # and a few steps of training lower the loss
    losses = [loss] + [net.train_step(dx.data_ptr(), dt.data_ptr(), n, h, w, 1e-3) for _ in range(20)]
    assert losses[-1] < 0.8 * losses[0], losses[::5]


def _hdr_grads_bf16(flat, noisy, clean, dtype):
    """Autograd of the HDR loss (L1 in log1p space) through the BF16-emulated
    restatement in `dtype`, flat in parameter order."""
    m = unet_ref.load_flat(unet_ref.UNetRef(variant="hdr"), flat).to(dtype)
    y = unet_ref.forward_bf16(m, torch.from_numpy(noisy), dtype=dtype, log_out=True)
    F.l1_loss(y, torch.log1p(torch.from_numpy(clean).to(dtype))).backward()
    return np.concatenate([p.grad.double().numpy().ravel() for p in m.parameters()]), \
        [(k, p.numel()) for k, p in m.named_parameters()]


def test_unet_hdr_gradients_match_bf16_emulated_autograd():
    """HDR variant: the kernels' gradients vs autograd through the BF16-emulated
    restatement in FP64, per tensor within 3x the FP32-vs-FP64 emulation
    floor + 1% relative L2, cosine above 0.998 (the bar of the reference
    variant's test above)."""
    flat = unet_ref.make_params(24, unet_ref.UNetRef(variant="hdr"))
    net = lumina.UNet(variant="hdr")
    net.set_params(flat)
    n, h, w = 2, 32, 48
    noisy, clean = _hdr_batch(n, h, w, 8)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    _, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
    g64, names = _hdr_grads_bf16(flat, noisy, clean, torch.float64)
    g32, _ = _hdr_grads_bf16(flat, noisy, clean, torch.float32)

    def err(a, b):
        return (float(np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)),
                float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)))

    off, worst = 0, []
    for k, cnt in names:
        sl = slice(off, off + cnt)
        off += cnt
        (cos, rel), (_, frel) = err(g[sl].astype(np.float64), g64[sl]), err(g32[sl], g64[sl])
        worst.append((rel - 3 * frel, cos, rel, frel, k))
    worst.sort(reverse=True)
    print("HDR worst tensors (excess, cos, rel, FP32 floor rel):", worst[:4])
    for _, cos, rel, frel, k in worst:
        assert cos > 0.998 and rel <= 3 * frel + 0.01, (k, cos, rel, frel)


def test_autotune_keeps_results():
    """lg_unet_autotune picks per-layer tile shapes by timing; the network's
    output and gradients must stay within the same bars against torch."""
    flat = unet_ref.make_params(79)
    net = lumina.UNet()
    net.set_params(flat)
    n, h, w = 2, 32, 144
    x = np.random.default_rng(8).uniform(0, 1, (n, 3, h, w)).astype(np.float32)
    y0 = net.forward(x)
    tiles = net.autotune(n, h, w, backward=True)
    print("autotuned tiles (bn, kc, stages):", tiles)
    assert len(tiles) == 30 and all(t[0] in (32, 64, 128) and t[1] in (16, 32) and 0 <= t[3] <= 7 for t in tiles)
    y1 = net.forward(x)
    assert np.array_equal(net.get_params(), flat)
    m = unet_ref.load_flat(unet_ref.UNetRef().eval(), flat)
    for y, fb in ((y0, FOLD_ALL), (y1, _folded_blocks(tiles))):
        with torch.no_grad():
            ref_q = unet_ref.forward_bf16(m, torch.from_numpy(x), fold=fb).numpy()
            ref_q64 = unet_ref.forward_bf16(m, torch.from_numpy(x), torch.float64, fold=fb).numpy()
        floor = np.abs(ref_q - ref_q64)
        err = np.abs(y - ref_q)
        assert err.mean() <= 2.0 * floor.mean() + 1e-4 and err.max() <= 2.0 * floor.max() + 2e-3
    noisy, clean = _batch(n, h, w, 4)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
    mm = unet_ref.load_flat(unet_ref.UNetRef(), flat)
    unet_ref.F.l1_loss(mm(torch.from_numpy(noisy)), torch.from_numpy(clean)).backward()
    ref_g = np.concatenate([p.grad.numpy().ravel() for _, p in mm.named_parameters()])
    cos = float(np.dot(g, ref_g) / (np.linalg.norm(g) * np.linalg.norm(ref_g)))
    assert cos > 0.99


def test_persistent_conv_kernel_is_bit_identical():
    """Every conv on the persistent warp-specialised kernel (same tile shapes,
    same MMAs in the same order) gives bit-identical outputs, loss and
    gradients to the one-tile-per-CTA kernel."""
    flat = unet_ref.make_params(80)
    n, h, w = 2, 40, 264  # partial tiles at the right and bottom edges, several tiles per CTA
    x = np.random.default_rng(9).uniform(0, 1, (n, 3, h, w)).astype(np.float32)
    noisy, clean = _batch(n, h, w, 12)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    outs = []
    for persist in (0, 1):
        net = lumina.UNet()
        net.set_params(flat)
        net.set_tiles([(0, 0, 0, persist)] * 30)
        y = net.forward(x)
        loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
        outs.append((y, loss, g))
        net.close()
    (y0, l0, g0), (y1, l1, g1) = outs
    assert np.array_equal(y0, y1)
    assert abs(l0 - l1) <= 1e-6 * max(1.0, abs(l0))
    assert np.array_equal(g0, g1)  # the weight-gradient partials are summed in a fixed order


# Forward convs in order (d1a .. u1b) with the resident-weights kernel where
# the layer has one output block and its weights fit beside the ring.
RESIDENT_TILES = [(32, 16, 10, 2), (32, 32, 6, 2), (64, 32, 4, 2), (64, 32, 4, 2)] + [(0, 0, 0, 1)] * 7 + \
                 [(64, 32, 4, 2), (32, 32, 5, 2), (32, 32, 6, 2)]
# The same layers on 4-row tiles (kernel choice 3).
ROWS4_TILES = [(32, 16, 8, 3), (32, 32, 4, 3), (64, 32, 3, 3), (64, 32, 3, 3)] + [(0, 0, 0, 1)] * 7 + \
              [(64, 32, 3, 3), (32, 32, 3, 3), (32, 32, 4, 3)]


# Row taps packed into N (kernel choices 4: resident weights, 4-row tiles; 5:
# resident, 8-row tiles; 6 and 7: streamed weights, 4- and 8-row tiles) on
# every conv with 32 or 64 output channels, forward (d1a .. u1b) and
# input-gradient (in the library's order of the 16 backward convs).
DYP4_TILES = [(32, 16, 7, 4), (32, 32, 3, 4), (64, 32, 3, 4), (64, 32, 2, 4)] + [(0, 0, 0, 1)] * 6 + \
             [(64, 32, 2, 6), (64, 32, 2, 4), (32, 32, 3, 4), (32, 32, 3, 4)]
DYP4_BWD = [(32, 32, 3, 4), (64, 32, 3, 4), (32, 32, 3, 4), (64, 32, 2, 4), (0, 0, 0, 1), (64, 32, 2, 4)] + \
           [(0, 0, 0, 1)] * 7 + [(64, 32, 2, 4), (32, 32, 3, 4), (32, 32, 3, 4)]
DYP8_TILES = [(32, 16, 4, 5), (32, 32, 2, 5), (64, 32, 2, 6), (64, 32, 2, 6)] + [(0, 0, 0, 1)] * 6 + \
             [(64, 32, 2, 6), (64, 32, 2, 6), (32, 32, 2, 7), (32, 32, 2, 5)]
DYP8_BWD = [(32, 32, 2, 5), (64, 32, 2, 6), (32, 32, 2, 5), (64, 32, 2, 6), (0, 0, 0, 1), (64, 32, 2, 6)] + \
           [(0, 0, 0, 1)] * 7 + [(64, 32, 2, 6), (32, 32, 2, 7), (32, 32, 2, 5)]

def test_resident_weight_conv_kernel_is_bit_identical():
    """The persistent kernel with the weights resident in shared memory (one
    copy per CTA instead of one per ring stage), with 2-, 4- and 8-row tiles,
    and with the three row taps of a column tap packed into one MMA's N, runs
    the same products in the same order for every output row: outputs, loss
    and gradients are bit-identical to the plain persistent kernel's, at
    batch 1 and 2, with partial tiles at the right edge."""
    flat = unet_ref.make_params(81)
    for n, h, w in ((1, 40, 264), (2, 64, 136), (1, 72, 136)):
        x = np.random.default_rng(10).uniform(0, 1, (n, 3, h, w)).astype(np.float32)
        noisy, clean = _batch(n, h, w, 13)
        dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
        outs = []
        for tiles in ([(0, 0, 0, 1)] * 30, RESIDENT_TILES + [(0, 0, 0, 1)] * 16, ROWS4_TILES + [(0, 0, 0, 1)] * 16,
                      DYP4_TILES + DYP4_BWD, DYP8_TILES + DYP8_BWD):
            net = lumina.UNet()
            net.set_params(flat)
            net.set_tiles(tiles)
            net.set_fold_upsampling(False)  # the folded form rounds its summed weights: compared elsewhere
            y = net.forward(x)
            loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
            outs.append((y, loss, g))
            net.close()
        for o in outs[1:]:
            assert np.array_equal(outs[0][0], o[0])
            assert outs[0][1] == o[1]
            assert np.array_equal(outs[0][2], o[2])



# Both folded-upsampling shapes per decoder level: u3a (64, 32, 2, 6); u2a and u1a (32, 32, 3, 6) here,
# (64, 32, 2, 6) and (32, 32, 2, 7) in the default tiles.
FOLD_B_TILES = [(32, 16, 4, 5), (32, 32, 3, 4), (64, 32, 2, 4), (64, 32, 2, 4)] + [(64, 32, 2, 6)] * 6 + \
               [(32, 32, 3, 6), (64, 32, 2, 4), (32, 32, 3, 6), (32, 32, 3, 4)]


@pytest.mark.parametrize("n,h,w", [(1, 40, 264), (2, 64, 136), (1, 72, 136)])
def test_folded_upsampling_matches_restatement(n, h, w):
    """u3a/u2a/u1a in their folded-upsampling form (x-only upsampled lower level, row taps summed per
    output-row parity): each folded kernel shape against the BF16-emulated restatement of that form, at
    sizes with partial row tiles at the bottom, widths whose deeper levels are not multiples of 8 (the
    pixel-by-pixel input view), and batch 2; and close to the unfolded pass."""
    flat = unet_ref.make_params(83)
    m = unet_ref.load_flat(unet_ref.UNetRef().eval(), flat)
    x = np.random.default_rng(12).uniform(0, 1, (n, 3, h, w)).astype(np.float32)
    with torch.no_grad():
        ref_q = unet_ref.forward_bf16(m, torch.from_numpy(x), fold=FOLD_ALL).numpy()
        ref_q64 = unet_ref.forward_bf16(m, torch.from_numpy(x), torch.float64, fold=FOLD_ALL).numpy()
    floor = np.abs(ref_q - ref_q64)
    for tiles in (None, FOLD_B_TILES + [(0, 0, 0, 1)] * 16):
        net = lumina.UNet()
        net.set_params(flat)
        if tiles is not None:
            net.set_tiles(tiles)
            assert _folded_blocks(tiles) == FOLD_ALL
        y = net.forward(x)
        err = np.abs(y - ref_q)
        print(f"folded {n}x{h}x{w}: max {err.max():.2e} mean {err.mean():.2e} "
              f"(floor max {floor.max():.2e} mean {floor.mean():.2e})")
        assert err.mean() <= 2.0 * floor.mean() + 1e-4
        assert err.max() <= 2.0 * floor.max() + 2e-3
        net.set_fold_upsampling(False)
        y_plain = net.forward(x)
        assert np.abs(y - y_plain).max() < 0.05 and np.abs(y - y_plain).mean() < 2e-3
        net.close()

def test_async_train_step_matches_sync():
    """lg_unet_train_step_async queues the same step on the caller's stream
    without waiting: after lg_unet_sync the parameters are bit-identical to
    those of the synchronous steps, and the device loss sum is the sum of n x
    the losses those steps returned."""
    flat = unet_ref.make_params(83)
    n, h, w = 3, 32, 48
    batches = [_batch(n, h, w, 20 + k) for k in range(3)]
    dev = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in batches]
    net = lumina.UNet()
    net.set_params(flat)
    losses = [net.train_step(dx.data_ptr(), dt.data_ptr(), n, h, w, 1e-3) for dx, dt in dev]
    p_sync = net.get_params()
    net.close()
    net = lumina.UNet()
    net.set_params(flat)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        loss_sum = torch.zeros(1, device="cuda")
        for dx, dt in dev:
            net.train_step_async(dx.data_ptr(), dt.data_ptr(), n, h, w, 1e-3, loss_sum.data_ptr(), s.cuda_stream)
        total = float(loss_sum.item())
    net.sync()
    p_async = net.get_params()
    net.close()
    assert np.array_equal(p_sync, p_async)
    assert abs(total - n * sum(losses)) <= 1e-5 * abs(total)


def test_training_is_bit_reproducible():
    """Weight and bias gradients are reduced from per-CTA partials in a fixed
    order (no floating-point atomics), so the same batch gives the same
    gradient bits and two training runs from the same parameters end with the
    same parameters."""
    flat = unet_ref.make_params(82)
    n, h, w = 4, 32, 48
    noisy, clean = _batch(n, h, w, 14)
    dx, dt = torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda()
    runs = []
    for _ in range(2):
        net = lumina.UNet()
        net.set_params(flat)
        _, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), n, h, w)
        for _ in range(5):
            net.train_step(dx.data_ptr(), dt.data_ptr(), n, h, w, 1e-3)
        runs.append((g, net.get_params()))
        net.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
