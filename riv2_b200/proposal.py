"""The motion-proposal network of the learned encode form: parameters, forward, backward and
AdamW, all computed by this library's sm_100a kernels (riv_nn.cu) through its C ABI.

PyTorch only holds device memory and supplies the stream; every arithmetic step of the
forward, the backward and the optimizer is one of the library's kernels:

* the four 3x3 convolutions: implicit-GEMM tcgen05 kernel (`riv_nn_conv`);
* the MLP and every backward product: TMA-fed tcgen05 GEMM (`riv_nn_gemm`);
* im2col^T, col2im with the ReLU derivative, transposes, bias-gradient sums, the head's
  loss and gradient and AdamW: element-wise kernels of the same file.

Shapes (per 16x16 MB): input 24x24x2 (correlation volume + predictor prior map); conv1 3x3/2
2->32 (12x12); conv2 3x3/2 (6x6); conv3 3x3/1 (6x6); conv4 3x3/2 (3x3); fc1 (288 + 16
predictor values + 16 zeros = 320) -> 128; fc2 128 -> 128; fc3 128 -> 16 (four candidate MVs
in half-pel units / 32, then a skip logit).  BF16 weights and activations, FP32 accumulation.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

from ._native import load_cuda

CH, K1, KC, F1, HID, OUT, FEAT = 32, 32, 320, 320, 128, 16, 24
# (name, rows, cols, real fan-in) of each weight, [out][in] with the reduction contiguous
WEIGHTS = (("w1", CH, K1, 18), ("w2", CH, KC, 288), ("w3", CH, KC, 288), ("w4", CH, KC, 288),
           ("f1", HID, F1, 304), ("f2", HID, HID, HID), ("f3", OUT, HID, HID))
BIASES = (("b1", CH), ("b2", CH), ("b3", CH), ("b4", CH), ("bf1", HID), ("bf2", HID), ("bf3", OUT))
NW = sum(r * c for _, r, c, _ in WEIGHTS)
NB = sum(n for _, n in BIASES)
MAGIC = b"RIVPROP1"
# Every symbol include/riv_nn.h declares (checked by the CPU test suite).
EXPORTED_SYMBOLS = ("riv_nn_gemm", "riv_nn_conv", "riv_nn_features", "riv_nn_im2col_t", "riv_nn_col2im",
                    "riv_nn_relu_bwd", "riv_nn_transpose", "riv_nn_colsum", "riv_nn_head_loss", "riv_nn_adamw",
                    "riv_nn_front")


def weight_offsets():
    off, out = 0, {}
    for name, r, c, _ in WEIGHTS:
        out[name] = (off, r, c)
        off += r * c
    for name, n in BIASES:
        out[name] = (off, n, 1)
        off += n
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights over the real fan-in (padding columns zero), zero biases; fc3 small."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NW + NB, np.float32)
    offs = weight_offsets()
    for name, r, c, fan in WEIGHTS:
        o = offs[name][0]
        std = np.sqrt(2.0 / fan) if name != "f3" else 0.02
        w = np.zeros((r, c), np.float32)
        w[:, :fan] = rng.normal(0.0, std, (r, fan))
        p[o:o + r * c] = w.reshape(-1)
    # spread the four candidates' initial outputs a little so they start apart
    o = offs["bf3"][0]
    p[o:o + 8] = np.array([0.0, 0.0, 0.1, 0.0, -0.1, 0.0, 0.0, 0.1], np.float32)
    return p


def save_params(path: str, p: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<II", NW, NB))
        f.write(np.ascontiguousarray(p, np.float32).tobytes())


def load_params(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        head = f.read(16)
        if head[:8] != MAGIC or struct.unpack("<II", head[8:]) != (NW, NB):
            raise ValueError(f"{path}: not a proposal-network parameter file of this layout")
        return np.frombuffer(f.read(), np.float32).copy()


def bf16_weights(p: np.ndarray) -> np.ndarray:
    """The weights as bf16 bit patterns (round to nearest even), in layout order."""
    w = np.ascontiguousarray(p[:NW], np.float32).view(np.uint32).astype(np.uint64)
    w = ((w + 0x7FFF + ((w >> 16) & 1)) >> 16).astype(np.uint16)
    return w


_L = None


def lib():
    global _L
    if _L is None:
        L = load_cuda()
        P, I, LL, F = C.c_void_p, C.c_int, C.c_longlong, C.c_float
        L.riv_nn_gemm.argtypes = [P, I, P, I, P, I, P, I, I, I, I, I, I, I, I, P, P]
        L.riv_nn_conv.argtypes = [I, P, I, P, P, P, I, I, I, P, P]
        L.riv_nn_features.argtypes = [P, P, I, I, P, I, I, P, P, P]
        L.riv_nn_front.argtypes = [P, P, I, I, P, I, I, P, P, P, P, P]
        L.riv_nn_im2col_t.argtypes = [I, P, I, I, P, P]
        L.riv_nn_col2im.argtypes = [I, P, I, P, I, P, P, P]
        L.riv_nn_relu_bwd.argtypes = [P, I, P, I, I, I, I, P, P, P]
        L.riv_nn_transpose.argtypes = [P, I, I, I, P, P]
        L.riv_nn_colsum.argtypes = [P, I, LL, I, P, P]
        L.riv_nn_head_loss.argtypes = [P, P, P, I, P, P, P, P]
        L.riv_nn_adamw.argtypes = [P, P, P, P, P, LL, F, F, F, F, F, I, I, P]
        _L = L
    return _L


def _ck(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed (CUDA error {rc})")


class ProposalNet:
    """Parameters on one GPU (f32 master copy + bf16 weights) and the kernels' buffers."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.p = torch.from_numpy(p.copy()).to(self.dev)
        self.wb = torch.empty(NW, dtype=torch.bfloat16, device=self.dev)
        self.wb.copy_(self.p[:NW].to(torch.bfloat16))
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.step_n = 0
        self.offs = weight_offsets()
        self._bufs = {}

    # ---- helpers
    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def w(self, name):
        o, r, c = self.offs[name]
        return self.wb[o:o + r * c]

    def bias(self, name):
        o, n, _ = self.offs[name]
        return self.p[o:o + n]

    def gw(self, name):
        o, r, c = self.offs[name]
        return self.g[o:o + r * c]

    def buf(self, key, shape, dtype):
        t = self._bufs.get(key)
        if t is None or t.shape != tuple(shape) or t.dtype != dtype:
            t = self.torch.empty(shape, dtype=dtype, device=self.dev)
            self._bufs[key] = t
        return t

    def params_numpy(self) -> np.ndarray:
        return self.p.detach().cpu().numpy()

    def check(self):
        self.torch.cuda.synchronize(self.dev)
        if int(self.err.item()):
            raise RuntimeError("a bounded device wait of the network kernels expired")

    # ---- kernels
    def gemm(self, A, lda, B, ldb, D, ldd, M, N, K, bk=64, mode=0, relu=0, bias=None, ksplit=1, ntile=None):
        ntile = ntile or (N if N <= 256 else 160 if N % 160 == 0 else 64)
        _ck(lib().riv_nn_gemm(A.data_ptr(), lda, B.data_ptr(), ldb, D.data_ptr(), ldd,
                              None if bias is None else bias.data_ptr(), M, N, K, bk, mode, relu, ksplit, ntile,
                              self.err.data_ptr(), self._stream()), "riv_nn_gemm")

    def conv(self, layer, x, in_mb, out, out_mb, out_ld, n):
        name = f"w{layer}"
        _ck(lib().riv_nn_conv(layer, x.data_ptr(), in_mb, self.w(name).data_ptr(), self.bias(f"b{layer}").data_ptr(),
                              out.data_ptr(), out_mb, out_ld, n, self.err.data_ptr(), self._stream()), "riv_nn_conv")

    # ---- forward
    def forward(self, feat, x1, n, save=False):
        """feat: n x 24 x 24 x 2 bf16; x1: n x 320 bf16 whose columns 288.. hold the predictor
        values (columns 0..287 are written here).  Returns n x 16 f32."""
        t = self.torch
        a1 = self.buf("a1", (n, 144, 32), t.bfloat16)
        a2 = self.buf("a2", (n, 36, 32), t.bfloat16)
        a3 = self.buf("a3", (n, 36, 32), t.bfloat16)
        self.conv(1, feat, FEAT * FEAT * 2, a1, 144 * 32, 32, n)
        self.conv(2, a1, 144 * 32, a2, 36 * 32, 32, n)
        self.conv(3, a2, 36 * 32, a3, 36 * 32, 32, n)
        self.conv(4, a3, 36 * 32, x1, F1, 32, n)
        h1 = self.buf("h1", (n, HID), t.bfloat16)
        h2 = self.buf("h2", (n, HID), t.bfloat16)
        o = self.buf("o", (n, OUT), t.float32)
        self.gemm(x1, F1, self.w("f1"), F1, h1, HID, n, HID, F1, mode=2, relu=1, bias=self.bias("bf1"))
        self.gemm(h1, HID, self.w("f2"), HID, h2, HID, n, HID, HID, mode=2, relu=1, bias=self.bias("bf2"))
        self.gemm(h2, HID, self.w("f3"), HID, o, OUT, n, OUT, HID, mode=0, relu=0, bias=self.bias("bf3"))
        return o

    # ---- backward
    def _t(self, key, src, ld, rows, cols):
        out = self.buf(key, (cols, rows), self.torch.bfloat16)
        _ck(lib().riv_nn_transpose(src.data_ptr(), ld, rows, cols, out.data_ptr(), self._stream()), "transpose")
        return out

    def _ksplit(self, tiles, red_blocks):
        return max(1, min(red_blocks, (2 * 148) // max(tiles, 1)))

    def backward(self, feat, x1, n, tmv, tskip):
        """Gradients of the mean loss into self.g (zeroed first); returns the device loss sum."""
        t, L, st = self.torch, lib(), self._stream()
        self.g.zero_()
        loss = self.buf("loss", (1,), t.float32)
        loss.zero_()
        o, h1, h2 = self._bufs["o"], self._bufs["h1"], self._bufs["h2"]

        def gslice(name):
            off, r, c = self.offs[name]
            return self.g[off:off + r * c]

        # head: loss, dO (n x 32, columns 16.. zero) and dO^T (16 x n)
        do = self.buf("do", (n, 32), t.bfloat16)
        dot = self.buf("dot", (OUT, n), t.bfloat16)
        _ck(L.riv_nn_head_loss(o.data_ptr(), tmv.data_ptr(), tskip.data_ptr(), n, do.data_ptr(), dot.data_ptr(),
                               loss.data_ptr(), st), "head loss")
        red = (n + 63) // 64
        # fully connected layers, last to first: dW = dZ^T . X (out x in), dX = dZ . W
        layers = (("f3", "bf3", h2, OUT, HID), ("f2", "bf2", h1, HID, HID), ("f1", "bf1", x1, HID, F1))
        dz, dz_ld = do, 32
        dzt = dot
        for i, (wn, bn, x, nout, nin) in enumerate(layers):
            _ck(L.riv_nn_colsum(dz.data_ptr(), dz_ld, n, nout, gslice(bn).data_ptr(), st), "colsum")
            xt = self._t(f"{wn}_xt", x, nin, n, nin)  # nin x n
            nt = 160 if nin == F1 else nin
            self.gemm(dzt, n, xt, n, gslice(wn), nin, nout, nin, n, mode=1,
                      ksplit=self._ksplit(nin // nt, red), ntile=nt)
            # W^T (nin x nout), with the reduction padded to 32 for the 16-wide fc3
            kw = max(nout, 32)
            wt = self.buf(f"{wn}_t", (nin, kw), t.bfloat16)
            if kw != nout:
                wt.zero_()
                wtt = self._t(f"{wn}_tt", self.w(wn), nin, nout, nin)
                wt[:, :nout].copy_(wtt)
            else:
                _ck(L.riv_nn_transpose(self.w(wn).data_ptr(), nin, nout, nin, wt.data_ptr(), st), "transpose")
            dx = self.buf(f"{wn}_dx", (n, nin), t.float32)
            self.gemm(dz, dz_ld, wt, kw, dx, nin, n, nin, kw, bk=32 if kw == 32 else 64, mode=0, ntile=nt)
            if i == 2:
                break
            act = x  # this layer's input: the ReLU output the gradient passes back through
            nz = self.buf(f"{wn}_dz", (n, nin), t.bfloat16)
            nzt = self.buf(f"{wn}_dzt", (nin, n), t.bfloat16)
            _ck(L.riv_nn_relu_bwd(dx.data_ptr(), nin, act.data_ptr(), nin, n, nin, 1, nz.data_ptr(), nzt.data_ptr(),
                                  st), "relu bwd")
            dz, dz_ld, dzt = nz, nin, nzt
        # conv4's output gradient: columns 0..287 of dX1 as (n * 9) x 32, times relu'(conv4 output)
        dx1 = self._bufs["f1_dx"]
        m = n * 9
        dz = self.buf("dzc4", (m, 32), t.bfloat16)
        dzt = self.buf("dzc4t", (32, m), t.bfloat16)
        _ck(L.riv_nn_relu_bwd(dx1.data_ptr(), F1, x1.data_ptr(), F1, m, 32, 9, dz.data_ptr(), dzt.data_ptr(), st),
            "relu bwd")
        hin = {2: 12, 3: 6, 4: 6}
        prev_act = {2: (self._bufs["a1"], 144 * 32), 3: (self._bufs["a2"], 36 * 32), 4: (self._bufs["a3"], 36 * 32)}
        for layer in (4, 3, 2, 1):
            kp = K1 if layer == 1 else KC
            _ck(L.riv_nn_colsum(dz.data_ptr(), 32, m, 32, gslice(f"b{layer}").data_ptr(), st), "colsum")
            colt = self._bufs[f"colt{layer}"]  # kp x m
            nt = 32 if kp == 32 else 64
            self.gemm(dzt, m, colt, m, gslice(f"w{layer}"), kp, 32, kp, m, mode=1,
                      ksplit=self._ksplit(kp // nt, (m + 63) // 64), ntile=nt)
            if layer == 1:
                break
            wt = self._t(f"wt{layer}", self.w(f"w{layer}"), kp, 32, kp)  # kp x 32
            dcol = self.buf(f"dcol{layer}", (m, kp), t.float32)
            self.gemm(dz, 32, wt, 32, dcol, kp, m, kp, 32, bk=32, mode=0, ntile=160)
            act, act_mb = prev_act[layer]
            mi = n * hin[layer] ** 2
            dz = self.buf(f"dzc{layer - 1}", (mi, 32), t.bfloat16)
            dzt = self.buf(f"dzc{layer - 1}t", (32, mi), t.bfloat16)
            _ck(L.riv_nn_col2im(layer, dcol.data_ptr(), n, act.data_ptr(), act_mb, dz.data_ptr(), dzt.data_ptr(), st),
                "col2im")
            m = mi
        return loss

    def prepare_backward(self, feat, x1, n):
        """im2col^T of every convolution's input (the reduction operands of the weight
        gradients), computed after the forward pass."""
        t, L, st = self.torch, lib(), self._stream()
        srcs = {1: (feat, FEAT * FEAT * 2), 2: (self._bufs["a1"], 144 * 32), 3: (self._bufs["a2"], 36 * 32),
                4: (self._bufs["a3"], 36 * 32)}
        hout = {1: 12, 2: 6, 3: 6, 4: 3}
        for layer, (src, mb) in srcs.items():
            kp = K1 if layer == 1 else KC
            m = n * hout[layer] ** 2
            colt = self.buf(f"colt{layer}", (kp, m), t.bfloat16)
            _ck(L.riv_nn_im2col_t(layer, src.data_ptr(), mb, n, colt.data_ptr(), st), "im2col_t")

    def adamw(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.01):
        L, st = lib(), self._stream()
        self.step_n += 1
        _ck(L.riv_nn_adamw(self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                           self.wb.data_ptr(), NW, lr, b1, b2, eps, wd, self.step_n, 1, st), "adamw")
        off = NW * 4
        _ck(L.riv_nn_adamw(self.p.data_ptr() + off, self.g.data_ptr() + off, self.m.data_ptr() + off,
                           self.v.data_ptr() + off, None, NB, lr, b1, b2, eps, wd, self.step_n, 0, st), "adamw")

    def train_step(self, feat, x1, tmv, tskip, lr=1e-3):
        n = feat.shape[0]
        self.forward(feat, x1, n, save=True)
        self.prepare_backward(feat, x1, n)
        loss = self.backward(feat, x1, n, tmv, tskip)
        self.adamw(lr=lr)
        return loss
