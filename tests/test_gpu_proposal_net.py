"""The motion-proposal network's tensor-core kernels against references (GPU).

* The TMA-fed tcgen05 GEMM against a float32 torch product of the same bf16 operands, for
  each operand width (64- and 32-element k-blocks), epilogue (f32, bf16 + bias + ReLU, split
  reduction with atomics) and tile width the network uses, with ragged row counts.
* The implicit-GEMM convolution, the network input (correlation volume and predictor values),
  the forward pass, the gradients of every parameter and AdamW against the float64 CPU oracle
  (oracle/proposal_oracle.py), which rounds to bf16 where the device stores bf16.
* A short training run on a fixed batch lowers the loss.
"""
import numpy as np
import pytest

from oracle import proposal_oracle as PO

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _bf(x):
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda().to(torch.bfloat16)


def _gemm(A, B, M, N, K, bk=64, mode=0, relu=0, bias=None, ksplit=1, ntile=None, out_bf16=False):
    from riv2_b200 import proposal as P
    net = P.ProposalNet.__new__(P.ProposalNet)
    net.torch, net.dev = torch, torch.device("cuda", 0)
    net.err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D = torch.zeros((M, N), dtype=torch.bfloat16 if out_bf16 else torch.float32, device="cuda")
    net.gemm(A, A.shape[1], B, B.shape[1], D, N, M, N, K, bk=bk, mode=mode, relu=relu, bias=bias, ksplit=ksplit,
             ntile=ntile)
    torch.cuda.synchronize()
    assert int(net.err.item()) == 0
    return D.float()


@pytest.mark.parametrize("M,N,K,bk,ntile", [(300, 32, 320, 64, None), (1000, 128, 320, 64, None),
                                            (257, 320, 32, 32, 160), (128, 16, 128, 64, None),
                                            (4096, 128, 128, 64, None), (77, 256, 192, 64, None)])
def test_gemm_matches_float32_product(M, N, K, bk, ntile):
    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    ref = A.float() @ B.float().T
    D = _gemm(A, B, M, N, K, bk=bk, ntile=ntile)
    err = (D - ref).abs().max().item()
    assert err <= 1e-3 * max(1.0, ref.abs().max().item()), err


def test_gemm_bf16_epilogue_with_bias_and_relu():
    M, N, K = 500, 128, 320
    g = torch.Generator(device="cpu").manual_seed(1)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    ref = torch.relu(A.float() @ B.float().T + bias).to(torch.bfloat16).float()
    D = _gemm(A, B, M, N, K, mode=2, relu=1, bias=bias, out_bf16=True)
    # one bf16 rounding step of difference at most
    assert ((D - ref).abs() <= ref.abs() * 2 ** -7 + 1e-6).all()


@pytest.mark.parametrize("ksplit", [1, 7, 40])
def test_gemm_split_reduction_accumulates(ksplit):
    M, N, K = 32, 320, 64 * 100 + 17  # long reduction, ragged last k-block
    g = torch.Generator(device="cpu").manual_seed(ksplit)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    pad = (-K) % 8  # row pitch a multiple of 8 elements
    Ap = torch.zeros(M, K + pad, dtype=torch.bfloat16)
    Bp = torch.zeros(N, K + pad, dtype=torch.bfloat16)
    Ap[:, :K], Bp[:, :K] = A, B
    ref = (A.float() @ B.float().T).cuda()
    D = _gemm(Ap.cuda(), Bp.cuda(), M, N, K, mode=1, ksplit=ksplit, ntile=64)
    assert (D - ref).abs().max().item() <= 2e-3 * ref.abs().max().item()


def _params(seed=3):
    from riv2_b200 import proposal as P
    p = P.init_params(seed)
    rng = np.random.default_rng(seed)
    offs = P.weight_offsets()
    for name, n in P.BIASES:  # non-zero biases, so that they are exercised
        o = offs[name][0]
        p[o:o + n] = rng.normal(0, 0.05, n).astype(np.float32)
    return p


def _layout():
    from riv2_b200 import proposal as P
    offs = P.weight_offsets()
    lay = {name: (offs[name][0], r, c, fan) for name, r, c, fan in P.WEIGHTS}
    lay.update({name: (offs[name][0], n, 1, n) for name, n in P.BIASES})
    return lay


def _random_inputs(n, seed):
    rng = np.random.default_rng(seed)
    feat = PO.bf16(rng.uniform(-1, 1, (n, 24, 24, 2)))
    feat[..., 1] = (rng.random((n, 24, 24)) < 0.02).astype(np.float64)
    pred16 = np.zeros((n, 16))
    pred16[:, :14] = PO.bf16(rng.integers(-40, 41, (n, 14)) / 64.0)
    return feat, pred16


def _device_inputs(feat, pred16):
    n = feat.shape[0]
    x1 = np.zeros((n, 320), np.float32)
    x1[:, 288:304] = pred16
    return _bf(feat), _bf(x1)


def test_features_match_oracle():
    from riv2_b200 import proposal as P
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=4)
    from oracle import oracle as O
    f0 = O.rgb_to_yuv(clip.frame(0), 352, 288, 352, 288)
    f1 = O.rgb_to_yuv(clip.frame(3), 352, 288, 352, 288)
    rng = np.random.default_rng(0)
    n = 396
    coded = np.zeros((n, 4), np.int8)
    coded[:, 0:2] = rng.integers(-13, 13, (n, 2))
    coded[:, 2:4] = rng.integers(0, 2, (n, 2))
    for prev in (None, coded):
        cur = torch.from_numpy(f1.y.copy()).cuda()
        ref = torch.from_numpy(f0.y.copy()).cuda()
        pc = None if prev is None else torch.from_numpy(prev).cuda()
        feat = torch.empty((n, 24, 24, 2), dtype=torch.bfloat16, device="cuda")
        x1 = torch.empty((n, 320), dtype=torch.bfloat16, device="cuda")
        rc = P.lib().riv_nn_features(cur.data_ptr(), ref.data_ptr(), 352, 288, None if pc is None else pc.data_ptr(),
                                     0, n, feat.data_ptr(), x1.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        wf, wp = PO.features(f1.y, f0.y, prev)
        assert np.array_equal(feat.float().cpu().numpy(), wf)
        assert np.array_equal(x1[:, 288:304].float().cpu().numpy(), wp)
        assert not x1[:, 304:].float().abs().sum().item()


def test_front_equals_features_then_conv1():
    """riv_nn_front (input on chip + conv1 on mma.sync) against riv_nn_features followed by the
    tcgen05 conv1, and against the float64 oracle's conv1: the same bf16 outputs up to one
    rounding step (the two sum the nine taps' f32 products in different orders)."""
    from oracle import oracle as O
    from riv2_b200 import proposal as P
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=9)
    f0 = O.rgb_to_yuv(clip.frame(0), 352, 288, 352, 288)
    f1 = O.rgb_to_yuv(clip.frame(2), 352, 288, 352, 288)
    rng = np.random.default_rng(3)
    n = 396
    coded = np.zeros((n, 4), np.int8)
    coded[:, 0:2] = rng.integers(-13, 13, (n, 2))
    coded[:, 2:4] = rng.integers(0, 2, (n, 2))
    net = P.ProposalNet(_params())
    w1, b1 = net.w("w1"), net.bias("b1")
    cur = torch.from_numpy(f1.y.copy()).cuda()
    ref = torch.from_numpy(f0.y.copy()).cuda()
    for prev, (mb0, cnt) in ((None, (0, n)), (coded, (5, 300))):
        pc = None if prev is None else torch.from_numpy(prev).cuda()
        pcp = None if pc is None else pc.data_ptr()
        feat = torch.empty((cnt, 24, 24, 2), dtype=torch.bfloat16, device="cuda")
        xa = torch.zeros((cnt, 320), dtype=torch.bfloat16, device="cuda")
        xb = torch.zeros((cnt, 320), dtype=torch.bfloat16, device="cuda")
        a_ref = torch.empty((cnt, 144, 32), dtype=torch.bfloat16, device="cuda")
        a_new = torch.full((cnt, 144, 32), 7.0, dtype=torch.bfloat16, device="cuda")
        L = P.lib()
        assert L.riv_nn_features(cur.data_ptr(), ref.data_ptr(), 352, 288, pcp, mb0, cnt, feat.data_ptr(),
                                 xa.data_ptr(), None) == 0
        assert L.riv_nn_conv(1, feat.data_ptr(), 24 * 24 * 2, w1.data_ptr(), b1.data_ptr(), a_ref.data_ptr(),
                             144 * 32, 32, cnt, net.err.data_ptr(), None) == 0
        assert L.riv_nn_front(cur.data_ptr(), ref.data_ptr(), 352, 288, pcp, mb0, cnt, w1.data_ptr(), b1.data_ptr(),
                              a_new.data_ptr(), xb.data_ptr(), None) == 0
        torch.cuda.synchronize()
        net.check()
        assert torch.equal(xa[:, 288:], xb[:, 288:])
        r, q = a_ref.float().cpu().numpy(), a_new.float().cpu().numpy()
        assert np.abs(r - q).max() <= 2 ** -7 * max(1.0, np.abs(r).max())
        assert (r != q).mean() < 0.01  # nearly all equal; the rest one bf16 step apart
        # and the float64 oracle's conv1 on the same input
        Pm = PO.unpack(net.params_numpy(), _layout())
        cols = PO.im2col(feat.float().cpu().numpy().astype(np.float64), 1)
        want = PO.bf16(np.maximum(cols @ Pm["w1"].T + Pm["b1"], 0.0)).reshape(cnt, 144, 32)
        assert np.abs(q - want).max() <= 2 ** -7 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("layer,nmb", [(2, 1), (2, 37), (3, 300), (4, 257), (2, 1000), (3, 4), (4, 8160)])
def test_conv_layers_match_oracle(layer, nmb, monkeypatch):
    """conv2-4 (im2col-TMA operand) against the float64 oracle's convolution of the same bf16
    input, with MB counts whose tiles end mid-MB and a ragged last tile; conv4 writes into
    fc1's input rows (320 columns per MB), leaving the predictor columns alone.  The k-block
    gather kernel (same K order of the f32 accumulation) gives the same bits."""
    from riv2_b200 import proposal as P
    hin, hout = {2: (12, 6), 3: (6, 6), 4: (6, 3)}[layer]
    net = P.ProposalNet(_params())
    rng = np.random.default_rng(100 * layer + nmb)
    x = np.maximum(rng.standard_normal((nmb, hin, hin, 32)), 0.0) * rng.uniform(0.5, 2.0, (nmb, 1, 1, 1))
    xin = _bf(x.reshape(nmb, hin * hin * 32))
    out_mb = 320 if layer == 4 else hout * hout * 32
    L = P.lib()

    def run():
        out = torch.full((nmb, out_mb), 3.0, dtype=torch.bfloat16, device="cuda")
        assert L.riv_nn_conv(layer, xin.data_ptr(), hin * hin * 32, net.w(f"w{layer}").data_ptr(),
                             net.bias(f"b{layer}").data_ptr(), out.data_ptr(), out_mb, 32, nmb, net.err.data_ptr(),
                             None) == 0
        torch.cuda.synchronize()
        net.check()
        return out.float().cpu().numpy()

    got = run()
    Pm = PO.unpack(net.params_numpy(), _layout())
    cols = PO.im2col(xin.float().cpu().numpy().astype(np.float64).reshape(nmb, hin, hin, 32), layer)
    want = PO.bf16(np.maximum(cols @ Pm[f"w{layer}"].T + Pm[f"b{layer}"], 0.0)).reshape(nmb, hout * hout * 32)
    q = got[:, :hout * hout * 32]
    assert np.abs(q - want).max() <= 2 ** -7 * max(1.0, np.abs(want).max())
    assert (q != want).mean() < 0.02
    assert (got[:, hout * hout * 32:] == 3.0).all()
    monkeypatch.setenv("RIV_CONV_GATHER", "1")
    assert np.array_equal(run(), got)


def test_forward_matches_oracle():
    from riv2_b200 import proposal as P
    p = _params()
    n = 300
    feat, pred16 = _random_inputs(n, 1)
    net = P.ProposalNet(p)
    fd, xd = _device_inputs(feat, pred16)
    o = net.forward(fd, xd, n).cpu().numpy()
    net.check()
    Pm = PO.unpack(p, _layout())
    want, acts = PO.forward(Pm, feat, pred16)
    # every conv layer's bf16 output (one rounding step apart at most)
    a4 = xd[:, :288].float().cpu().numpy().reshape(n, 3, 3, 32)
    assert np.abs(a4 - acts[4]).max() <= 2 ** -7 * max(1.0, np.abs(acts[4]).max())
    err = np.abs(o - want).max()
    assert err <= 2e-2 * max(1.0, np.abs(want).max()), err


def test_gradients_match_oracle():
    from riv2_b200 import proposal as P
    p = _params(5)
    n = 256
    feat, pred16 = _random_inputs(n, 2)
    rng = np.random.default_rng(9)
    tmv = rng.integers(-25, 26, (n, 2)).astype(np.int16)
    tskip = (rng.random(n) < 0.3).astype(np.uint8)
    net = P.ProposalNet(p)
    fd, xd = _device_inputs(feat, pred16)
    net.forward(fd, xd, n, save=True)
    net.prepare_backward(fd, xd, n)
    loss = net.backward(fd, xd, n, torch.from_numpy(tmv).cuda(), torch.from_numpy(tskip).cuda())
    net.check()
    g = net.g.cpu().numpy()
    lay = _layout()
    Pm = PO.unpack(p, lay)
    o, acts = PO.forward(Pm, feat, pred16)
    want_loss, dO = PO.head_loss(o, tmv, tskip)
    assert abs(loss.item() / n - want_loss) <= 1e-2 * abs(want_loss)
    G = PO.backward(Pm, acts, dO)
    for name, (off, r, c, fan) in lay.items():
        got = g[off:off + r * c].reshape(r, c) if c > 1 else g[off:off + r]
        if c > 1:
            assert not got[:, fan:].any(), f"{name}: padding columns have gradients"
            got = got[:, :fan]
        ref = G[name]
        rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-12)
        assert rel < 3e-2, (name, rel)


def test_adamw_matches_numpy():
    from riv2_b200 import proposal as P
    p = _params(7)
    net = P.ProposalNet(p)
    rng = np.random.default_rng(1)
    grads = [rng.normal(0, 1e-2, p.size).astype(np.float32) for _ in range(3)]
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    w = p.astype(np.float64).copy()
    lr, b1, b2, eps, wd = 1e-3, 0.9, 0.999, 1e-8, 0.01
    for t, gr in enumerate(grads, 1):
        net.g.copy_(torch.from_numpy(gr))
        net.adamw(lr=lr, b1=b1, b2=b2, eps=eps, wd=wd)
        m = b1 * m + (1 - b1) * gr
        v = b2 * v + (1 - b2) * gr.astype(np.float64) ** 2
        decay = np.zeros_like(w)
        decay[:P.NW] = 1.0
        w = w - lr * wd * w * decay
        w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    got = net.p.cpu().numpy()
    assert np.abs(got - w).max() <= 1e-6
    assert torch.equal(net.wb, net.p[:P.NW].to(torch.bfloat16))


def test_training_lowers_the_loss():
    from riv2_b200 import proposal as P
    n = 1024
    feat, pred16 = _random_inputs(n, 11)
    # targets that depend on the input: the arg-max of channel 0 of the correlation volume
    f0 = feat[..., 0].reshape(n, -1)
    k = f0.argmax(axis=1)
    tmv = np.stack([(k % 24 - 12) * 4, (k // 24 - 12) * 4], axis=1).clip(-25, 25).astype(np.int16)
    tskip = (pred16[:, 0] > 0).astype(np.uint8)
    net = P.ProposalNet(seed=1)
    fd, xd = _device_inputs(feat, pred16)
    tm, ts = torch.from_numpy(tmv).cuda(), torch.from_numpy(tskip).cuda()
    losses = []
    for step in range(60):
        losses.append(net.train_step(fd, xd, tm, ts, lr=2e-3).item() / n)
    net.check()
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.6 * losses[0], losses[::10]
