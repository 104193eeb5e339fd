"""U-net of the learned warm start, on the library's own CUDA kernels.

Convolutions are implicit GEMMs: an im2col tile and the weights in BF16 go
through the tensor-core GEMM (tcgen05.mma, FP32 accumulation in tensor memory,
``maf_nn_gemm``); bias, ReLU, pooling, upsampling, the skip concatenations, the
normalising head, every backward pass and Adam are the hand-written kernels of
``nn.cu``.  Master weights are FP32 (Adam updates them); the GEMMs read their
BF16 copies.  PyTorch only holds the device buffers (allocation, views); no
torch operation computes anything here.

Architecture (activations pixel-major, H and W multiples of 16; widths multiples of 8):

    x (cin) -> conv 32 -> conv 32 = e1 ----------------------------+
      pool -> conv 64 -> conv 64 = e2 ----------------+             |
        pool -> conv 128 -> conv 128 = b              |             |
      up(b) | e2 (192) -> conv 64 = u2                 |             |
    up(u2) | e1 (96) -> conv 32 -> conv 3 = d    <-----+-------------+
    y = normalize(m + d)

all 3x3 with zero padding, ReLU after every convolution but the last.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _ck, lib

_P = C.c_void_p  # the signatures are declared with the others in magnumaf/__init__.py


def _r8(c: int) -> int:
    return (c + 7) // 8 * 8


def _p(t) -> int:
    return t.data_ptr()


class _Conv:
    """3x3 convolution cin -> cout at a given level (0: full size, 1: half, 2: quarter)."""

    def __init__(self, cin, cout, level, relu, off):
        self.cin, self.cout, self.level, self.relu = cin, cout, level, relu
        self.cp = _r8(cin)          # padded input channels of the im2col tile
        self.coutp = _r8(cout)      # padded output channels of the data-gradient GEMM
        self.woff = off             # offset of W [cout][9][cin] in the flat parameters
        self.boff = off + cout * 9 * cin
        self.n = cout * 9 * cin + cout


class UNet:
    """UNet(cin, seed): the warm-start network.  Parameters are one flat FP32
    device buffer (per layer W [cout][9][cin], then b [cout]); He-initialised,
    the last layer zero (an untrained net returns the input magnetisation)."""

    def __init__(self, cin: int = 8, seed: int = 0, widths=(32, 64, 128)):
        import torch

        self.torch = torch
        w1, w2, w3 = widths
        spec = [(cin, w1, 0, True), (w1, w1, 0, True), (w1, w2, 1, True), (w2, w2, 1, True), (w2, w3, 2, True),
                (w3, w3, 2, True), (w3 + w2, w2, 1, True), (w2 + w1, w1, 0, True), (w1, 3, 0, False)]
        self.layers = []
        off = 0
        for ci, co, lv, relu in spec:
            layer = _Conv(ci, co, lv, relu, off)
            self.layers.append(layer)
            off += layer.n
        self.cin = cin
        self.widths = (w1, w2, w3)
        self.n_params = off
        rng = np.random.default_rng(seed)
        p = np.zeros(off, dtype=np.float32)
        for layer in self.layers[:-1]:
            fan_in = 9 * layer.cin
            p[layer.woff:layer.boff] = rng.normal(0.0, math.sqrt(2.0 / fan_in), size=layer.boff - layer.woff)
        dev = torch.device("cuda")
        self.params = torch.from_numpy(p).to(dev)
        self.grad = torch.zeros_like(self.params)
        self.m1 = torch.zeros_like(self.params)
        self.m2 = torch.zeros_like(self.params)
        self.step_count = 0
        self._wb = [None] * len(self.layers)
        self._shape = None
        self._dirty = True

    # ------------------------------------------------------------ parameters
    def get_params(self) -> np.ndarray:
        return self.params.cpu().numpy().copy()

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError("expected %d parameters" % self.n_params)
        self.params.copy_(self.torch.from_numpy(p))
        self.m1.zero_()
        self.m2.zero_()
        self.step_count = 0
        self._dirty = True

    def _stream(self):
        return _P(self.torch.cuda.current_stream().cuda_stream)

    def _cast_weights(self):
        """BF16 copies of every layer's weights: Wb [cout][9 cp] and WtB [9 cp][coutp]."""
        torch = self.torch
        st = self._stream()
        for i, L in enumerate(self.layers):
            if self._wb[i] is None:
                self._wb[i] = (torch.empty((L.cout, 9 * L.cp), dtype=torch.bfloat16, device="cuda"),
                               torch.empty((9 * L.cp, L.coutp), dtype=torch.bfloat16, device="cuda"))
            wb, wtb = self._wb[i]
            _ck(lib.maf_nn_wcast(_P(_p(self.params) + 4 * L.woff), L.cout, L.cin, L.cp, L.coutp, _P(_p(wb)),
                                 _P(_p(wtb)), st))
        self._dirty = False

    # ------------------------------------------------------------ buffers
    def _buffers(self, B, H, W):
        if self._shape == (B, H, W):
            return
        if H % 16 or W % 16:
            raise ValueError("H and W must be multiples of 16")
        torch = self.torch
        f32, b16 = torch.float32, torch.bfloat16
        P = [B * H * W, B * (H // 2) * (W // 2), B * (H // 4) * (W // 4)]
        self.P = P
        self.dims = [(H, W), (H // 2, W // 2), (H // 4, W // 4)]
        z = lambda *s, dt=f32: torch.zeros(s, dtype=dt, device="cuda")
        self.inb = [z(P[L.level], L.cp, dt=b16) for L in self.layers]  # BF16 input of each conv
        self.out = [z(P[L.level], L.cout) for L in self.layers]         # FP32 output (after ReLU)
        self.m_in = z(P[0], 3)
        self.pool1 = z(P[1], self.widths[0])
        self.pool2 = z(P[2], self.widths[1])
        kmax = max(9 * L.cp * P[L.level] for L in self.layers)
        self.col = torch.zeros(kmax, dtype=b16, device="cuda")
        self.colT = torch.zeros(kmax, dtype=b16, device="cuda")
        self.gemm = torch.zeros(max(max(P[L.level] * L.coutp, P[L.level] * 9 * L.cp) for L in self.layers),
                                dtype=f32, device="cuda")
        self.y = z(P[0], 3)
        # backward
        self.dA = [z(P[L.level], L.cout) for L in self.layers]
        self.dY = z(max(P[L.level] * L.cout for L in self.layers))
        self.dYb = torch.zeros(max(P[L.level] * L.coutp for L in self.layers), dtype=b16, device="cuda")
        self.dYbT = torch.zeros_like(self.dYb)
        self.dX = z(max(P[L.level] * L.cp for L in self.layers))
        self.gd = z(P[0], 3)
        self.cell_loss = z(P[0])
        self.loss = z(1)
        self.splits = 64
        self.work = z(self.splits * max(L.cout * 9 * L.cp for L in self.layers))
        self.wg = z(max(L.cout * 9 * L.cp for L in self.layers))
        self._shape = (B, H, W)

    # ------------------------------------------------------------ forward
    def _conv_fwd(self, i, B):
        L = self.layers[i]
        P = self.P[L.level]
        h, w = self.dims[L.level]
        st = self._stream()
        wb, _ = self._wb[i]
        _ck(lib.maf_nn_im2col(_P(_p(self.inb[i])), B, h, w, L.cp, _P(_p(self.col)), 0, st))
        _ck(lib.maf_nn_gemm(_P(_p(self.col)), 9 * L.cp, _P(_p(wb)), 9 * L.cp, _P(_p(self.gemm)), L.cout, P, L.cout,
                            9 * L.cp, st))
        nxt = self.inb[i + 1] if i + 1 < len(self.layers) and self.layers[i + 1].cin == L.cout and \
            self.layers[i + 1].level == L.level else None
        _ck(lib.maf_nn_bias_act(_P(_p(self.gemm)), L.cout, _P(_p(self.params) + 4 * L.boff), P, L.cout,
                                int(L.relu), _P(_p(self.out[i])), _P(_p(nxt)) if nxt is not None else None,
                                self.layers[i + 1].cp if nxt is not None else L.coutp, st))

    def _forward(self, x_ptr, B, H, W):
        self._buffers(B, H, W)
        if self._dirty:
            self._cast_weights()
        st = self._stream()
        w1, w2, w3 = self.widths
        (H1, W1), (H2, W2) = self.dims[1], self.dims[2]
        _ck(lib.maf_nn_input(_P(x_ptr), B, self.cin, H, W, self.layers[0].cp, _P(_p(self.inb[0])),
                             _P(_p(self.m_in)), st))
        self._conv_fwd(0, B)
        self._conv_fwd(1, B)                      # e1 = out[1]
        _ck(lib.maf_nn_pool(_P(_p(self.out[1])), B, H, W, w1, _P(_p(self.pool1)), _P(_p(self.inb[2])),
                            self.layers[2].cp, st))
        self._conv_fwd(2, B)
        self._conv_fwd(3, B)                      # e2 = out[3]
        _ck(lib.maf_nn_pool(_P(_p(self.out[3])), B, H1, W1, w2, _P(_p(self.pool2)), _P(_p(self.inb[4])),
                            self.layers[4].cp, st))
        self._conv_fwd(4, B)
        self._conv_fwd(5, B)                      # b = out[5]
        _ck(lib.maf_nn_up_cat(_P(_p(self.out[5])), w3, _P(_p(self.out[3])), w2, B, H1, W1, _P(_p(self.inb[6])),
                              self.layers[6].cp, st))
        self._conv_fwd(6, B)                      # u2 = out[6]
        _ck(lib.maf_nn_up_cat(_P(_p(self.out[6])), w2, _P(_p(self.out[1])), w1, B, H, W, _P(_p(self.inb[7])),
                              self.layers[7].cp, st))
        self._conv_fwd(7, B)
        self._conv_fwd(8, B)                      # d = out[8]

    def forward(self, x_ptr: int, B: int, H: int, W: int, y_ptr: int = None):
        """x [B][cin][H][W] FP32 (device) -> y = normalize(m + d) [B H W][3] FP32 into self.y
        (and into y_ptr, same layout, when given)."""
        self._forward(x_ptr, B, H, W)
        st = self._stream()
        P0 = self.P[0]
        _ck(lib.maf_nn_head(_P(_p(self.m_in)), _P(_p(self.out[8])), 3, None, P0, _P(y_ptr or _p(self.y)), None, None,
                            None, st))
        return self.y

    # ------------------------------------------------------------ backward
    def _conv_bwd(self, i, B, dx=None, dx_channels=0):
        """dA[i] (FP32 [P][cout]) -> parameter gradients of layer i and, when dx is
        given, the gradient of its input into dx (FP32 [P][dx_channels], the first
        dx_channels of the cp im2col channels)."""
        L = self.layers[i]
        P = self.P[L.level]
        h, w = self.dims[L.level]
        st = self._stream()
        _, wtb = self._wb[i]
        _ck(lib.maf_nn_relu_bwd(_P(_p(self.dA[i])), _P(_p(self.out[i])), P, L.cout, int(L.relu), _P(_p(self.dY)),
                                _P(_p(self.dYb)), L.coutp, st))
        _ck(lib.maf_nn_colsum(_P(_p(self.dY)), P, L.cout, _P(_p(self.grad) + 4 * L.boff), st))
        # dW [cout][9 cp] = dY^T . col: both operands with the pixels contiguous
        _ck(lib.maf_nn_transpose(_P(_p(self.dYb)), P, L.coutp, _P(_p(self.dYbT)), st))
        _ck(lib.maf_nn_im2col(_P(_p(self.inb[i])), B, h, w, L.cp, _P(_p(self.colT)), 1, st))
        _ck(lib.maf_nn_gemm_splitk(_P(_p(self.dYbT)), P, _P(_p(self.colT)), P, _P(_p(self.wg)), L.cout, 9 * L.cp, P,
                                   self.splits, _P(_p(self.work)), st))
        _ck(lib.maf_nn_wgrad(_P(_p(self.wg)), L.cout, L.cin, L.cp, _P(_p(self.grad) + 4 * L.woff), st))
        if dx is not None:
            # dcol [P][9 cp] = dY . W, then col2im
            _ck(lib.maf_nn_gemm(_P(_p(self.dYb)), L.coutp, _P(_p(wtb)), L.coutp, _P(_p(self.gemm)), 9 * L.cp, P,
                                9 * L.cp, L.coutp, st))
            _ck(lib.maf_nn_col2im(_P(_p(self.gemm)), B, h, w, L.cp, dx_channels, _P(_p(dx)), 0, st))

    def _backward(self, B):
        st = self._stream()
        w1, w2, w3 = self.widths
        H, W = self.dims[0]
        H1, W1 = self.dims[1]
        self._conv_bwd(8, B, self.dA[7], w1)
        self._conv_bwd(7, B, self.dX, self.layers[7].cp)   # d cat(up(u2), e1) [P0][w2 + w1]
        # e1 = out[1] gets its skip part here and its pooled-path part below
        _ck(lib.maf_nn_up_cat_bwd(_P(_p(self.dX)), self.layers[7].cp, w2, w1, B, H, W, _P(_p(self.dA[6])),
                                  _P(_p(self.dA[1].zero_())), st))
        self._conv_bwd(6, B, self.dX, self.layers[6].cp)   # d cat(up(b), e2) [P1][w3 + w2]
        _ck(lib.maf_nn_up_cat_bwd(_P(_p(self.dX)), self.layers[6].cp, w3, w2, B, H1, W1, _P(_p(self.dA[5])),
                                  _P(_p(self.dA[3].zero_())), st))
        self._conv_bwd(5, B, self.dA[4], w3)
        self._conv_bwd(4, B, self.dX, w2)                   # d pool2 [P2][w2]
        _ck(lib.maf_nn_pool_bwd(_P(_p(self.dX)), B, H1, W1, w2, _P(_p(self.dA[3])), 1, st))
        self._conv_bwd(3, B, self.dA[2], w2)
        self._conv_bwd(2, B, self.dX, w1)                   # d pool1 [P1][w1]
        _ck(lib.maf_nn_pool_bwd(_P(_p(self.dX)), B, H, W, w1, _P(_p(self.dA[1])), 1, st))
        self._conv_bwd(1, B, self.dA[0], w1)
        self._conv_bwd(0, B)

    def loss_grad(self, x_ptr: int, t_ptr: int, B: int, H: int, W: int, want_grad: bool = True) -> float:
        """Loss = mean over pixels of |y - t|^2 (t [B H W][3] FP32, device); with want_grad the
        parameter gradients land in self.grad."""
        self._forward(x_ptr, B, H, W)
        st = self._stream()
        P0 = self.P[0]
        _ck(lib.maf_nn_head(_P(_p(self.m_in)), _P(_p(self.out[8])), 3, _P(t_ptr), P0, _P(_p(self.y)),
                            _P(_p(self.dA[8])), _P(_p(self.cell_loss)), _P(_p(self.loss)), st))
        if want_grad:
            self._backward(B)
        return float(self.loss.item())

    def train_step(self, x_ptr: int, t_ptr: int, B: int, H: int, W: int, lr: float) -> float:
        loss = self.loss_grad(x_ptr, t_ptr, B, H, W, True)
        self.step_count += 1
        _ck(lib.maf_nn_adam(_P(_p(self.params)), _P(_p(self.grad)), _P(_p(self.m1)), _P(_p(self.m2)), self.n_params,
                            float(lr), self.step_count, self._stream()))
        self._dirty = True
        return loss
