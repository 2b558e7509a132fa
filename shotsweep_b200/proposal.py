"""Learned velocity proposal: a ~3M-parameter BF16 encoder-decoder that maps gathers to a velocity model.

Input: a model's five shot gathers (5 x 1000 x 70) in the stored float16 form
sign(g) log1p(|g|), divided by the training set's largest magnitude
(3_train.py:157,198,513); output: a 70 x 70 velocity, tanh-normalised as
(v - 3000) / 1500 (3_train.py:158).  The layout follows the reference's
InversionNet (3_train.py:219-240: an encoder that shrinks the time axis with
strided convolutions to a 1 x 1 code, and a decoder that grows it to 80 x 80,
cropped to 70 x 70) at a width of about 3M parameters, with leaky ReLU(0.2)
activations and no batch normalisation:

    e1 8x1/4   5->32    e2 4x1/2  32->64   e3 4x1/2  64->64   e4 4x1/2  64->128
    e5 3x3/2 128->128   e6 3x3/2 128->256  e7 3x3/2 256->256  e8 4x9 window 256->128
    d1 fc 128 -> 5x5x128, then four x2 upsamplings with 3x3 convolutions
    d2 128->128  d3 128->64  d4 64->64  d5 64->32, crop to 70x70, 3x3 head 32->1, tanh

Every convolution runs as im2col plus the library's tcgen05 GEMM (BF16 operands,
F32 accumulation, bias and leaky ReLU fused into the epilogue); the backward
pass uses the same GEMM for weight and input gradients, a gather-form col2im,
and AdamW with float32 master weights (3_train.py:529: AdamW, weight decay 1e-4).
A training step can be captured as one CUDA graph.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

SLOPE = 0.2
T_IN, X_IN, S_IN = 1000, 70, 5
OUT = 70


@dataclass(frozen=True)
class Layer:
    name: str
    cin: int
    cout: int
    kh: int = 1
    kw: int = 1
    sh: int = 1
    sw: int = 1
    ph: int = 0
    pw: int = 0
    up: int = 1
    kind: str = 'conv'     # 'conv', 'window' (kernel = whole input -> 1x1), 'fc' (1x1 -> out_hw x out_hw)
    out_hw: int = 0


LAYERS = (
    Layer('e1', 5, 32, 8, 1, 4, 1, 2, 0),
    Layer('e2', 32, 64, 4, 1, 2, 1, 1, 0),
    Layer('e3', 64, 64, 4, 1, 2, 1, 1, 0),
    Layer('e4', 64, 128, 4, 1, 2, 1, 1, 0),
    Layer('e5', 128, 128, 3, 3, 2, 2, 1, 1),
    Layer('e6', 128, 256, 3, 3, 2, 2, 1, 1),
    Layer('e7', 256, 256, 3, 3, 2, 2, 1, 1),
    Layer('e8', 256, 128, 4, 9, kind='window'),
    Layer('d1', 128, 128, kind='fc', out_hw=5),
    Layer('d2', 128, 128, 3, 3, 1, 1, 1, 1, 2),
    Layer('d3', 128, 64, 3, 3, 1, 1, 1, 1, 2),
    Layer('d4', 64, 64, 3, 3, 1, 1, 1, 1, 2),
    Layer('d5', 64, 32, 3, 3, 1, 1, 1, 1, 2),
)
HEAD_C, HEAD_OFF = 32, 5


def round8(n):
    return (n + 7) // 8 * 8


def plan_shapes():
    """Per layer: (Hin, Win, Hout, Wout, K, Kc, N)."""
    h, w = T_IN, X_IN
    out = []
    for L in LAYERS:
        if L.kind == 'conv':
            ho = (h * L.up + 2 * L.ph - L.kh) // L.sh + 1
            wo = (w * L.up + 2 * L.pw - L.kw) // L.sw + 1
            K, N = L.kh * L.kw * L.cin, L.cout
        elif L.kind == 'window':
            assert (h, w) == (L.kh, L.kw), (L.name, h, w)
            ho = wo = 1
            K, N = L.kh * L.kw * L.cin, L.cout
        else:
            assert (h, w) == (1, 1)
            ho = wo = L.out_hw
            K, N = L.cin, L.out_hw * L.out_hw * L.cout
        out.append((h, w, ho, wo, K, round8(K), N))
        h, w = ho, wo
    assert (h, w) == (OUT + 2 * HEAD_OFF, OUT + 2 * HEAD_OFF)
    return out


def param_layout():
    """Offsets (floats) of every weight [N][Kc], bias [N], head weight [9][32] and head bias in one flat block."""
    off, lay = 0, {}

    def take(name, n):
        nonlocal off
        lay[name] = (off, n)
        off += (n + 63) // 64 * 64
    for L, (_, _, _, _, K, Kc, N) in zip(LAYERS, plan_shapes()):
        take(L.name + '.w', N * Kc)
        take(L.name + '.b', N)
    take('head.w', 9 * HEAD_C)
    take('head.b', 1)
    return lay, off


def init_params(seed=0):
    """He-uniform weights for leaky ReLU(0.2), zero biases (float32, flat)."""
    lay, total = param_layout()
    rng = np.random.default_rng([seed, 31])
    p = np.zeros(total, np.float32)
    for L, (_, _, _, _, K, Kc, N) in zip(LAYERS, plan_shapes()):
        bound = np.sqrt(6.0 / ((1 + SLOPE ** 2) * K))
        w = rng.uniform(-bound, bound, (N, K)).astype(np.float32)
        o, n = lay[L.name + '.w']
        p[o:o + n].reshape(N, Kc)[:, :K] = w
    o, n = lay['head.w']
    bound = np.sqrt(3.0 / (9 * HEAD_C))
    p[o:o + n] = rng.uniform(-bound, bound, n).astype(np.float32)
    return p


class ProposalNet:
    """The network with its parameters, optimiser state and buffers for batches of `batch` models."""

    def __init__(self, batch, device=None, seed=0, params=None):
        self.dev = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        _lib.require_cuda(self.dev)
        self.L = _lib.load()
        self.B = int(batch)
        self.shapes = plan_shapes()
        self.lay, total = param_layout()
        f32 = dict(dtype=torch.float32, device=self.dev)
        bf = dict(dtype=torch.bfloat16, device=self.dev)
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.params = torch.tensor(p, **f32)
        self.p16 = self.params.to(torch.bfloat16)
        self.grads = torch.zeros(total, **f32)
        self.m = torch.zeros(total, **f32)
        self.v = torch.zeros(total, **f32)
        self.lr = torch.tensor([5e-4], **f32)
        self.step_count = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        B = self.B
        self.x0 = torch.empty(B * T_IN * X_IN * S_IN, **bf)
        self.y = []
        self.cols = []       # each convolution's im2col columns, kept from forward to backward
        max_dcols = 1
        for L, (hi, wi, ho, wo, K, Kc, N) in zip(LAYERS, self.shapes):
            M = B * (ho * wo if L.kind != 'fc' else 1)
            self.y.append(torch.empty(M * N, **bf))
            self.cols.append(torch.empty(M * Kc, **bf) if L.kind == 'conv' else None)
            max_dcols = max(max_dcols, M * K)
        self.dcols = torch.empty(max_dcols, **bf)   # column gradients, BF16 (rounded once, summed in F32 by col2im)
        self.dpre = [torch.empty_like(y) for y in self.y]
        self.pred = torch.empty(B, OUT, OUT, **f32)
        self.target = torch.empty(B, OUT, OUT, **f32)
        self.dpre_head = torch.empty(B, OUT, OUT, **f32)
        self.loss_sum = torch.zeros(1, **f32)
        self.ids = torch.zeros(B, dtype=torch.int32, device=self.dev)
        self.graph = None

    # -- views ------------------------------------------------------------------
    def _view(self, t, name):
        o, n = self.lay[name]
        return t[o:o + n]

    def weight16(self, i):
        return self._view(self.p16, LAYERS[i].name + '.w')

    def n_params(self):
        return sum(self.shapes[i][4] * self.shapes[i][6] + self.shapes[i][6] for i in range(len(LAYERS))) + 9 * HEAD_C + 1

    def _conv(self, i):
        L, (hi, wi, ho, wo, K, Kc, N) = LAYERS[i], self.shapes[i]
        if L.kind == 'conv':
            d = [self.B, hi, wi, L.cin, L.kh, L.kw, L.sh, L.sw, L.ph, L.pw, L.up]
        elif L.kind == 'window':
            d = [self.B, hi, wi, L.cin, L.kh, L.kw, 1, 1, 0, 0, 1]
        else:
            d = [self.B, 1, 1, L.cin, 1, 1, 1, 1, 0, 0, 1]
        return (ctypes.c_int32 * 11)(*d)

    def _head(self):
        hw = self.shapes[-1][2]
        return (ctypes.c_int32 * 6)(self.B, hw, hw, HEAD_C, HEAD_OFF, OUT)

    def _stream(self):
        return _lib.stream_handle(self.dev)

    def _gemm(self, A, lda, Bm, ldb, M, N, K, epi, C, ldc, bias=None, slope=SLOPE, layout=0):
        """C = A B^T through the tensor cores; layout bit 0 / 1: A / B stored K-outer (read M/N-major)."""
        _lib.check(self.L.ss_gemm_bf16_layout(_lib.ptr(A), lda, _lib.ptr(Bm), ldb, M, N, K, layout, epi, _lib.ptr(C),
                                              ldc, _lib.ptr(bias), slope, 0, _lib.ptr(self.err), self._stream()),
                   'ss_gemm_bf16_layout')

    # -- forward / backward -------------------------------------------------------
    def load_batch(self, stored, scale, targets=None):
        """Inputs of samples self.ids from stored float16 gathers [n, 5, 1000, 70] (and targets [n, 70, 70])."""
        _lib.check(self.L.ss_gathers_nhwc_bf16(_lib.ptr(stored), _lib.ptr(self.ids), self.B, S_IN, T_IN, X_IN,
                                               float(scale), _lib.ptr(self.x0), self._stream()), 'ss_gathers_nhwc_bf16')
        if targets is not None:
            _lib.check(self.L.ss_gather_rows_f32(_lib.ptr(targets), _lib.ptr(self.ids), self.B, OUT * OUT,
                                                 _lib.ptr(self.target), self._stream()), 'ss_gather_rows_f32')

    def forward(self):
        x = self.x0
        for i, L in enumerate(LAYERS):
            hi, wi, ho, wo, K, Kc, N = self.shapes[i]
            M = self.B * (ho * wo if L.kind != 'fc' else 1)
            if L.kind == 'conv':
                _lib.check(self.L.ss_im2col_bf16(_lib.ptr(x), self._conv(i), Kc, _lib.ptr(self.cols[i]),
                                                 self._stream()), 'ss_im2col_bf16')
                A, lda = self.cols[i], Kc
            else:
                A, lda = x, K
            self._gemm(A, lda, self.weight16(i), Kc, M, N, K, _lib.EPI_BIAS_LRELU_BF16, self.y[i], N,
                       self._view(self.params, L.name + '.b'))
            x = self.y[i]
        _lib.check(self.L.ss_head_forward(_lib.ptr(x), self._head(), _lib.ptr(self._view(self.params, 'head.w')),
                                          _lib.ptr(self._view(self.params, 'head.b')), _lib.ptr(self.pred),
                                          self._stream()), 'ss_head_forward')
        return self.pred

    def backward(self):
        """Loss of self.pred against self.target, then every gradient into self.grads (zeroed first)."""
        self.grads.zero_()
        self.loss_sum.zero_()
        n = self.B * OUT * OUT
        _lib.check(self.L.ss_l1_tanh_loss(_lib.ptr(self.pred), _lib.ptr(self.target), n, _lib.ptr(self.loss_sum),
                                          _lib.ptr(self.dpre_head), self._stream()), 'ss_l1_tanh_loss')
        _lib.check(self.L.ss_head_backward(_lib.ptr(self.y[-1]), self._head(),
                                           _lib.ptr(self._view(self.params, 'head.w')), _lib.ptr(self.dpre_head),
                                           SLOPE, _lib.ptr(self._view(self.grads, 'head.w')),
                                           _lib.ptr(self._view(self.grads, 'head.b')), _lib.ptr(self.dpre[-1]),
                                           self._stream()), 'ss_head_backward')
        for i in range(len(LAYERS) - 1, -1, -1):
            L = LAYERS[i]
            hi, wi, ho, wo, K, Kc, N = self.shapes[i]
            M = self.B * (ho * wo if L.kind != 'fc' else 1)
            x = self.x0 if i == 0 else self.y[i - 1]
            dp = self.dpre[i]
            # bias gradient: column sums of the pre-activation gradient
            _lib.check(self.L.ss_bias_grad_bf16(_lib.ptr(dp), N, M, N, _lib.ptr(self._view(self.grads, L.name + '.b')),
                                                self._stream()), 'ss_bias_grad_bf16')
            # weight gradient dW[N][K] += dp^T cols: both operands read as stored (pixels outermost)
            src, lds = (self.cols[i], Kc) if L.kind == 'conv' else (x, K)   # forward columns, or the input itself
            self._gemm(dp, N, src, lds, N, K, M, _lib.EPI_F32_ADD, self._view(self.grads, L.name + '.w'), Kc,
                       layout=3)
            if i == 0:
                break
            # column gradients dcols[M][K] = dp W (weights read as stored, [N][Kc]), rounded to BF16 (slope 1, no
            # bias: a plain BF16 store), then gathered onto the input
            self._gemm(dp, N, self.weight16(i), Kc, M, K, N, _lib.EPI_BIAS_LRELU_BF16, self.dcols, K, slope=1.0,
                       layout=2)
            Lp = LAYERS[i - 1]
            _lib.check(self.L.ss_col2im16_lrelu_bf16(_lib.ptr(self.dcols), self._conv(i), K, _lib.ptr(x), SLOPE,
                                                     _lib.ptr(self.dpre[i - 1]), Lp.cout, self._stream()),
                       'ss_col2im16_lrelu_bf16')

    def optimizer_step(self, weight_decay=1e-4):
        _lib.check(self.L.ss_adamw(_lib.ptr(self.params), _lib.ptr(self.grads), _lib.ptr(self.m), _lib.ptr(self.v),
                                   self.params.numel(), _lib.ptr(self.lr), 0.9, 0.999, 1e-8, weight_decay,
                                   _lib.ptr(self.step_count), _lib.ptr(self.p16), self._stream()), 'ss_adamw')

    def train_step(self, stored, scale, targets):
        self.load_batch(stored, scale, targets)
        self.forward()
        self.backward()
        self.optimizer_step()

    def check(self):
        if int(self.err.item()) != 0:
            raise RuntimeError(f'tensor-core GEMM pipeline wait ran out (code {int(self.err.item())})')
