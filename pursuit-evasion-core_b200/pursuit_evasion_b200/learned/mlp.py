"""Learned value surrogate: an MLP trained and queried with libpe_b200 kernels.

Architecture (BF16 weights and activations, FP32 accumulation):
    features (padded to 128) -> 4 x [Linear 256 + SiLU] -> Linear 1
The features of a relative 5D state [x, y, psi, vP, vE] are
[x/e, y/e, cos psi, sin psi, vP~, vE~] (speeds mapped to [-1, 1]); of an 8D
state, the same per car.  Every forward, backward and Adam kernel is
hand-written (csrc/mlp.cu, csrc/mlp_tc.cu, C ABI pe_mlp_*): the layer and
activation-gradient GEMMs run on the tensor cores with tcgen05.mma and the
accumulator in tensor memory, the split-K weight-gradient GEMM on mma.sync,
which reads the row-major activations as they are (the tcgen05 split-K
product, pe_mlp_gemm_tc_splitk, is faster alone but needs both operands
transposed first, and the transposes cost more than it saves).
PyTorch only provides device memory, the stream, random numbers for
minibatches and, in the tests, the FP64 autograd that checks the gradients.  The reference's precedent is a
SiLU MLP trained with Adam on MSE against DP labels
(local_game/learning.py:32-38, training.py:185-186, :352).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from .. import _native

FEATURES = 128  # padded input width (GEMM tiles are 128 wide)
HIDDEN = 256
LAYERS = 4


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class ValueMLP:
    """Parameters and buffers of the surrogate on one CUDA device."""

    def __init__(self, in_features, *, hidden=HIDDEN, layers=LAYERS, seed=0,
                 device=0, max_batch=8192):
        import torch

        self.torch = torch
        self.lib = _native.library()
        self.dev = torch.device("cuda", device)
        self.in_features = int(in_features)
        self.hidden = int(hidden)
        self.layers = int(layers)
        if hidden % 128 or in_features > FEATURES:
            raise ValueError("hidden must be a multiple of 128, in_features <= 128")
        gen = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        dims = [FEATURES] + [hidden] * layers
        for l in range(layers):
            fan_in = in_features if l == 0 else hidden
            bound = 1.0 / math.sqrt(fan_in)
            w = (torch.rand(hidden, dims[l], generator=gen) * 2 - 1) * bound
            if l == 0:
                w[:, in_features:] = 0
            self.w.append(w.to(self.dev))
            self.b.append(((torch.rand(hidden, generator=gen) * 2 - 1) * bound).to(self.dev))
        self.w_out = ((torch.rand(hidden, generator=gen) * 2 - 1) / math.sqrt(hidden)).to(self.dev)
        self.b_out = torch.zeros(1, device=self.dev)
        self.w16 = [w.to(torch.bfloat16).contiguous() for w in self.w]
        # transposed bf16 copies [in][out]: the K-major operand of the
        # activation-gradient GEMM on the tensor cores
        self.w16t = [torch.empty(w.shape[1], w.shape[0], dtype=torch.bfloat16, device=self.dev)
                     for w in self.w]
        self.params = self.w + self.b + [self.w_out, self.b_out]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.grads = [torch.zeros_like(p) for p in self.params]
        self.corr = torch.ones(2, device=self.dev)
        self.loss = torch.zeros(1, device=self.dev)
        self._alloc(max_batch)
        self._transpose_weights()

    def _alloc(self, batch):
        torch = self.torch
        self.batch = batch
        self.feat = torch.zeros(batch, FEATURES, dtype=torch.bfloat16, device=self.dev)
        self.z = [torch.empty(batch, self.hidden, device=self.dev) for _ in range(self.layers)]
        self.h = [torch.empty(batch, self.hidden, dtype=torch.bfloat16, device=self.dev)
                  for _ in range(self.layers)]
        self.dz = [torch.empty(batch, self.hidden, dtype=torch.bfloat16, device=self.dev)
                   for _ in range(self.layers)]
        self.y = torch.empty(batch, device=self.dev)
        self.dy = torch.empty(batch, device=self.dev)
        self.target = torch.empty(batch, device=self.dev)

    def set_batch(self, batch):
        """Reallocate the activation buffers for `batch` rows (for instance
        large inference chunks after training); weights are kept."""
        self._alloc(int(batch))

    # ----------------------------------------------------------- kernels
    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _gemm(self, A, B, M, N, K, lda, ldb, a_mmajor, b_nmajor, epi, *, splits=1,
              C32=None, C16=None, ldc=0, bias=None, zpre=None):
        opt = lambda t: None if t is None else _ptr(t)
        rc = self.lib.pe_mlp_gemm(_ptr(A), _ptr(B), M, N, K, lda, ldb, int(a_mmajor),
                                  int(b_nmajor), epi, splits, opt(C32), opt(C16), ldc,
                                  opt(bias), opt(zpre), self._stream())
        _native.check(rc)

    def _gemm_tc(self, A, B, M, N, K, epi, *, C32=None, C16=None, bias=None, zpre=None):
        """C = A B^T on the tensor cores (tcgen05); A [M][K], B [N][K]."""
        opt = lambda t: None if t is None else _ptr(t)
        _native.check(self.lib.pe_mlp_gemm_tc(_ptr(A), _ptr(B), M, N, K, A.shape[1],
                                              B.shape[1], epi, opt(C32), opt(C16), N,
                                              opt(bias), opt(zpre), self._stream()))

    def _transpose_weights(self):
        for w, wt in zip(self.w16, self.w16t):
            _native.check(self.lib.pe_mlp_transpose(_ptr(w), _ptr(wt), w.shape[0], w.shape[1],
                                                    self._stream()))

    def forward(self, rows, *, target=False, inference=False):
        """Forward over self.feat[:rows]; with target=True also the MSE loss
        (accumulated into self.loss) and dy.  inference=True skips storing
        the FP32 pre-activations, which only backward() reads."""
        x = self.feat
        for l in range(self.layers):
            K = FEATURES if l == 0 else self.hidden
            self._gemm_tc(x, self.w16[l], rows, self.hidden, K, 1,
                          C32=None if inference else self.z[l], C16=self.h[l],
                          bias=self.b[l])
            x = self.h[l]
        _native.check(self.lib.pe_mlp_head_forward(
            _ptr(self.h[-1]), _ptr(self.w_out), _ptr(self.b_out),
            _ptr(self.target) if target else None, _ptr(self.y),
            _ptr(self.dy) if target else None, _ptr(self.loss) if target else None,
            rows, self.hidden, self._stream()))
        return self.y[:rows]

    def backward(self, rows):
        """Gradients of the MSE of the last forward(target=True) into self.grads."""
        for g in self.grads:
            g.zero_()
        L = self.layers
        gw, gb = self.grads[:L], self.grads[L:2 * L]
        gw_out, gb_out = self.grads[2 * L], self.grads[2 * L + 1]
        _native.check(self.lib.pe_mlp_head_backward(
            _ptr(self.h[-1]), _ptr(self.z[-1]), _ptr(self.w_out), _ptr(self.dy),
            _ptr(gw_out), _ptr(gb_out), _ptr(self.dz[-1]), rows, self.hidden,
            self._stream()))
        splits = max(1, min(64, rows // 256))
        while rows % (32 * splits):
            splits -= 1
        for l in reversed(range(L)):
            prev = self.feat if l == 0 else self.h[l - 1]
            K_in = FEATURES if l == 0 else self.hidden
            # dW_l[n][k] = sum_b dz_l[b][n] prev[b][k]
            self._gemm(self.dz[l], prev, self.hidden, K_in, rows, self.hidden, K_in,
                       True, True, 2, splits=splits, C32=gw[l], ldc=K_in)
            _native.check(self.lib.pe_mlp_colsum(_ptr(self.dz[l]), _ptr(gb[l]), rows,
                                                 self.hidden, self._stream()))
            if l > 0:
                # dz_{l-1} = (dz_l W_l) * silu'(z_{l-1})
                self._gemm_tc(self.dz[l], self.w16t[l], rows, self.hidden, self.hidden, 3,
                              C16=self.dz[l - 1], zpre=self.z[l - 1])

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        """One Adam update; the bias corrections are read from self.corr on
        the device (set them with set_step before the call or graph replay)."""
        for i, (p, g, m, v) in enumerate(zip(self.params, self.grads, self.m, self.v)):
            w16 = _ptr(self.w16[i]) if i < self.layers else None
            _native.check(self.lib.pe_mlp_adam(_ptr(p), w16, _ptr(g), _ptr(m), _ptr(v),
                                               p.numel(), lr, beta1, beta2, eps,
                                               _ptr(self.corr), 1.0, self._stream()))
        self._transpose_weights()

    def set_step(self, step, beta1=0.9, beta2=0.999):
        self.corr.copy_(self.torch.tensor([1 - beta1 ** step, 1 - beta2 ** step],
                                          dtype=self.torch.float32))
