"""tcgen05 bf16 convolutions and the learned-filter kernels against the float64
CNN oracle (small images) and torch fp32 ``conv2d`` (a 256 x 256 image).

Tolerances: inputs and weights are bf16 and products accumulate in fp32, so a
layer whose output is stored as bf16 (ReLU / mask epilogues) is compared at
1e-2 of the output's largest magnitude (bf16 keeps 8 significant bits);
outputs kept in fp32 (the filter, weight gradients) at 1e-4 relative; the
whole training gradient, whose forward activations are rounded to bf16 at every
layer, at 5e-2 relative L2 per layer.
"""

import ctypes

import numpy as np
import pytest

from oracle import cnn_oracle as co

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200 import _native  # noqa: E402
from thick_ptycho_b200.learned import (LearnedPreconditioner, kernel_layout, pack_padded,  # noqa: E402
                                       transposed_layout, unpack_padded)

LIB = _native.load()


def P(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def S():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def bf(x):
    return torch.as_tensor(x).to(torch.bfloat16).double().numpy()


def act_buffer(nf, nb, batch, ch):
    return torch.zeros(int(LIB.tp_cnn_act_bytes(nf, nb, batch, ch)), dtype=torch.uint8, device="cuda")


def run_conv(x, wl, bias, epi, cin, aux=None):
    B, _, nb, nf = x.shape
    xin = pack_padded(torch.from_numpy(x)).cuda()
    auxb = None if aux is None else pack_padded(torch.from_numpy(aux)).cuda()
    b = None if bias is None else torch.from_numpy(bias.astype(np.float32)).cuda()
    if epi == _native.CONV_FILTER:
        out = torch.empty((13, B * nb * nf), dtype=torch.complex64, device="cuda")
    else:
        out = act_buffer(nf, nb, B, 32)
    rc = LIB.tp_conv3x3_bf16(nf, nb, B, cin, epi, P(xin), P(wl.cuda()), P(b), P(auxb), P(out), 1.0, S())
    _native.check(rc, "tp_conv3x3_bf16")
    LIB.tp_device_status(S(), ctypes.byref(ctypes.c_int32()))
    if epi == _native.CONV_FILTER:
        return out.cpu().numpy()
    return unpack_padded(out, 32, B, nf, nb).cpu().numpy().astype(np.float64)


def close(got, ref, tol):
    return np.abs(got - ref).max() <= tol * max(np.abs(ref).max(), 1e-30)


@pytest.mark.parametrize("cin,nf,nb,batch", [(16, 21, 13, 2), (32, 21, 13, 2), (32, 40, 3, 5), (16, 1, 1, 1)])
def test_conv_relu_against_oracle(cin, nf, nb, batch):
    rng = np.random.default_rng(cin * 7 + nf)
    x = rng.standard_normal((batch, cin, nb, nf))
    w = rng.standard_normal((32, cin, 3, 3)) * 0.3
    bias = rng.standard_normal(32) * 0.5
    got = run_conv(x, kernel_layout(torch.from_numpy(w)), bias, _native.CONV_RELU, cin)
    ref = np.maximum(co.conv3x3(bf(x), bf(w), bias.astype(np.float32).astype(np.float64)), 0)
    assert close(got, ref, 1e-2)


def test_conv_mask_epilogue_is_relu_backward():
    rng = np.random.default_rng(11)
    nf, nb, batch = 17, 11, 2
    dy = rng.standard_normal((batch, 32, nb, nf))
    aux = rng.standard_normal((batch, 32, nb, nf))
    w = rng.standard_normal((32, 32, 3, 3)) * 0.2
    got = run_conv(dy, transposed_layout(torch.from_numpy(w)), None, _native.CONV_MASK, 32, aux=aux)
    ref = co.conv3x3_dgrad(bf(dy), bf(w)) * (bf(aux) > 0)
    assert close(got, ref, 1e-2)


def test_conv_filter_epilogue_fp32():
    rng = np.random.default_rng(12)
    nf, nb, batch = 19, 9, 2
    x = np.maximum(rng.standard_normal((batch, 32, nb, nf)), 0)
    w = rng.standard_normal((32, 32, 3, 3)) * 0.2
    bias = rng.standard_normal(32) * 0.1
    F = run_conv(x, kernel_layout(torch.from_numpy(w)), bias, _native.CONV_FILTER, 32)
    o = co.conv3x3(bf(x), bf(w), bias.astype(np.float32).astype(np.float64))
    ref = co.filter_from_output(o).reshape(batch, 13, nb * nf).transpose(1, 0, 2).reshape(13, -1)
    assert close(F, ref, 1e-4)


def test_conv_full_image_against_torch_fp32():
    """A 256 x 256 image (129 CTAs) against torch's fp32 conv2d of the same bf16 values."""
    g = torch.Generator(device="cuda").manual_seed(0)
    nf = nb = 256
    x = torch.randn((1, 32, nb, nf), device="cuda", generator=g).to(torch.bfloat16).float()
    w = (torch.randn((32, 32, 3, 3), device="cuda", generator=g) * 0.1).to(torch.bfloat16).float()
    b = torch.randn(32, device="cuda", generator=g) * 0.1
    xin = pack_padded(x)
    out = act_buffer(nf, nb, 1, 32)
    _native.check(LIB.tp_conv3x3_bf16(nf, nb, 1, 32, _native.CONV_RELU, P(xin), P(kernel_layout(w)), P(b), None,
                                      P(out), 1.0, S()), "tp_conv3x3_bf16")
    got = unpack_padded(out, 32, 1, nf, nb)
    ref = torch.relu(torch.nn.functional.conv2d(x, w, b, padding=1))
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < 1e-2, err


def test_wgrad_against_oracle():
    rng = np.random.default_rng(13)
    for cin, nf, nb, batch in [(16, 23, 9, 2), (32, 15, 14, 3)]:
        x = rng.standard_normal((batch, cin, nb, nf))
        dy = rng.standard_normal((batch, 32, nb, nf))
        dw = torch.zeros((9, cin, 32), dtype=torch.float32, device="cuda")
        db = torch.zeros(32, dtype=torch.float32, device="cuda")
        xb, dyb = pack_padded(torch.from_numpy(x)).cuda(), pack_padded(torch.from_numpy(dy)).cuda()
        _native.check(LIB.tp_conv3x3_wgrad(nf, nb, batch, cin, P(xb), P(dyb), P(dw), P(db), S()), "tp_conv3x3_wgrad")
        got = dw.view(3, 3, cin, 32).permute(3, 2, 0, 1).cpu().numpy()
        ref = co.conv3x3_wgrad(bf(x), bf(dy))
        assert np.linalg.norm(got - ref) <= 1e-4 * np.linalg.norm(ref)
        assert np.allclose(db.cpu().numpy(), bf(dy).sum(axis=(0, 2, 3)), rtol=1e-4, atol=1e-3)


def test_filter_apply_and_gradient_against_oracle():
    rng = np.random.default_rng(14)
    nf, nb, nimg, per = 11, 8, 2, 3
    N = nf * nb
    F = (rng.standard_normal((nimg, 13, nb, nf)) + 1j * rng.standard_normal((nimg, 13, nb, nf))) * 0.1
    z = rng.standard_normal((nimg * per, nb, nf)) + 1j * rng.standard_normal((nimg * per, nb, nf))
    e = rng.standard_normal((nimg * per, nb, nf)) + 1j * rng.standard_normal((nimg * per, nb, nf))
    Fd = torch.from_numpy(F.transpose(1, 0, 2, 3).reshape(13, nimg * N).astype(np.complex64)).cuda()
    zd = torch.from_numpy(z.reshape(-1, N).astype(np.complex64)).cuda()
    y = torch.empty_like(zd)
    _native.check(LIB.tp_cnn_filter_apply(nf, nb, nimg * per, per, 0, P(Fd), P(zd), P(y), S()), "apply")
    ref = co.filter_apply(F, z, per)
    assert np.linalg.norm(y.cpu().numpy().reshape(ref.shape) - ref) <= 1e-5 * np.linalg.norm(ref)
    ed = torch.from_numpy(e.reshape(-1, N).astype(np.complex64)).cuda()
    dy = act_buffer(nf, nb, nimg, 32)
    _native.check(LIB.tp_cnn_filter_grad(nf, nb, nimg, per, P(zd), P(ed), 1.0, P(dy), S()), "grad")
    got = unpack_padded(dy, 32, nimg, nf, nb).cpu().numpy()
    ref = np.zeros((nimg, 32, nb, nf))
    for v in range(nimg * per):
        for t, (ddy, ddx) in enumerate(co.TAPS):
            g = 2 * np.conj(co.shift(z[v], ddy, ddx)) * e[v]
            ref[v // per, 2 * t] += g.real
            ref[v // per, 2 * t + 1] += g.imag
    assert close(got, ref, 1e-2)


def test_training_gradients_against_oracle():
    """Loss and all weight/bias gradients of the four-layer network + filter."""
    rng = np.random.default_rng(15)
    nf, nb, nimg, per = 12, 10, 2, 2
    N = nf * nb
    m = LearnedPreconditioner(nf, nb, kappa=2.0, seed=3, out_scale=0.7)
    with torch.no_grad():
        m.w[3].mul_(30.0)
        for b in m.b:
            b.copy_(torch.randn(32, generator=torch.Generator().manual_seed(4)).cuda() * 0.05)
    m._sync_kernel_weights()
    d = (rng.standard_normal((nimg, N)) + 1j * rng.standard_normal((nimg, N))) * 0.5
    z = rng.standard_normal((nimg * per, N)) + 1j * rng.standard_normal((nimg * per, N))
    t = rng.standard_normal((nimg * per, N)) + 1j * rng.standard_normal((nimg * per, N))
    sc = rng.uniform(0.5, 1.5, nimg * per)
    c64 = lambda a: torch.from_numpy(a.astype(np.complex64)).cuda()  # noqa: E731
    loss, gw, gb = m.loss_and_grads(c64(d), c64(z), c64(t), torch.from_numpy(sc.astype(np.float32)).cuda(), per)
    W = [bf(w.cpu()) for w in m.w]
    Bv = [b.cpu().double().numpy() for b in m.b]
    d64 = d.astype(np.complex64).astype(complex).reshape(nimg, nb, nf)
    ref_loss, rw, rb, _, _ = co.loss_and_grads(W, Bv, d64, m.kappa, z.astype(np.complex64).astype(complex).reshape(-1, nb, nf),
                                               t.astype(np.complex64).astype(complex).reshape(-1, nb, nf), sc, per,
                                               out_scale=m.out_scale)
    assert abs(float(loss) - ref_loss) <= 1e-2 * ref_loss
    for i in range(4):
        g = gw[i].cpu().double().numpy()
        assert np.linalg.norm(g - rw[i]) <= 5e-2 * np.linalg.norm(rw[i]), (i, np.linalg.norm(g - rw[i]) / np.linalg.norm(rw[i]))
        gbi = gb[i].cpu().double().numpy()
        assert np.linalg.norm(gbi - rb[i]) <= 5e-2 * np.linalg.norm(rb[i]) + 1e-6, i
