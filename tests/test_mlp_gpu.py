"""Hand-written BF16 tensor-core MLP kernels (pe_mlp_*): GEMM layouts and
epilogues against PyTorch fp32 matmuls of the same bf16 operands, and the
forward/backward gradients against PyTorch CPU FP64 autograd on the same
weights and inputs."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def gemm_case(a_mmajor, b_nmajor, epi, M=256, N=256, K=256, splits=1, seed=0):
    from pursuit_evasion_b200.learned.mlp import ValueMLP

    g = torch.Generator().manual_seed(seed)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(K, N, generator=g).to(torch.bfloat16)
    bias = torch.randn(N, generator=g)
    zpre = torch.randn(M, N, generator=g)
    ref = A.float() @ B.float()
    dev = torch.device("cuda", 0)
    A_st = (A.t() if a_mmajor else A).contiguous().to(dev)   # [K][M] or [M][K]
    B_st = (B if b_nmajor else B.t()).contiguous().to(dev)   # [K][N] or [N][K]
    lda = M if a_mmajor else K
    ldb = N if b_nmajor else K
    C32 = torch.zeros(M, N, device=dev)
    C16 = torch.zeros(M, N, dtype=torch.bfloat16, device=dev)
    net = ValueMLP.__new__(ValueMLP)
    from pursuit_evasion_b200 import _native
    net.torch, net.lib, net.dev = torch, _native.library(), dev
    net._gemm(A_st, B_st, M, N, K, lda, ldb, a_mmajor, b_nmajor, epi, splits=splits,
              C32=C32 if epi in (0, 1, 2) else None,
              C16=C16 if epi in (1, 3) else None, ldc=N,
              bias=bias.to(dev) if epi == 1 else None,
              zpre=zpre.to(dev) if epi == 3 else None)
    torch.cuda.synchronize()
    return ref, bias, zpre, C32.cpu(), C16.float().cpu()


@pytest.mark.parametrize("a_mmajor", [False, True])
@pytest.mark.parametrize("b_nmajor", [False, True])
def test_gemm_layouts_store_fp32(a_mmajor, b_nmajor):
    ref, _, _, C32, _ = gemm_case(a_mmajor, b_nmajor, 0)
    torch.testing.assert_close(C32, ref, rtol=1e-4, atol=1e-3)


def test_gemm_split_k_accumulates():
    ref, _, _, C32, _ = gemm_case(True, True, 2, M=256, N=128, K=2048, splits=8)
    torch.testing.assert_close(C32, ref, rtol=1e-4, atol=2e-3)


def test_gemm_bias_silu_and_dsilu_epilogues():
    ref, bias, _, C32, C16 = gemm_case(False, False, 1)
    z = ref + bias
    torch.testing.assert_close(C32, z, rtol=1e-4, atol=1e-3)
    torch.testing.assert_close(C16, torch.nn.functional.silu(z), rtol=1e-2, atol=2e-2)
    ref, _, zpre, _, C16 = gemm_case(False, True, 3)
    s = torch.sigmoid(zpre)
    torch.testing.assert_close(C16, ref * s * (1 + zpre * (1 - s)), rtol=1e-2, atol=5e-2)


# bf16 keeps 8 significant bits: one unit in the last place is 2^-7 of the
# value at most.
BF16_ULP = 2.0 ** -7


def test_gradients_match_fp64_autograd():
    """Forward and backward against FP64 autograd on the same bf16 weights
    and inputs, with bf16 rounding at the points where the kernels store
    bf16 (each layer's activation, each activation gradient).  What is left
    is FP32-vs-FP64 accumulation and the rare value that rounds to the other
    side of a bf16 boundary, so every gradient tensor must agree within half
    a bf16 unit in the last place, in norm."""
    from pursuit_evasion_b200.learned.mlp import FEATURES, ValueMLP

    rows = 512
    net = ValueMLP(6, seed=3, max_batch=rows)
    g = torch.Generator().manual_seed(1)
    feat = torch.zeros(rows, FEATURES)
    feat[:, :6] = torch.rand(rows, 6, generator=g) * 2 - 1
    target = torch.sin(3 * feat[:, 0]) * feat[:, 1] + 0.5 * feat[:, 4]
    net.feat.copy_(feat.to(torch.bfloat16))
    net.target[:rows].copy_(target)
    net.loss.zero_()
    net.forward(rows, target=True)
    net.backward(rows)
    torch.cuda.synchronize()

    def bf16(t):
        return t.to(torch.bfloat16).double()

    x = net.feat.double().cpu()
    ws = [w.double().cpu().requires_grad_() for w in net.w16]  # the bf16 weights used
    bs = [b.double().cpu().requires_grad_() for b in net.b]
    wo = net.w_out.double().cpu().requires_grad_()
    bo = net.b_out.double().cpu().requires_grad_()

    class RoundGrad(torch.autograd.Function):
        """Identity forward; the incoming gradient rounded to bf16 backward
        (the activation-gradient stores)."""
        @staticmethod
        def forward(ctx, t):
            return t.clone()

        @staticmethod
        def backward(ctx, grad):
            return bf16(grad)

    h = x
    for w, b in zip(ws, bs):
        z = RoundGrad.apply(h @ w.t() + b)  # dz of this layer is stored in bf16
        h = torch.nn.functional.silu(z)
        h = h + (bf16(h) - h).detach()     # the activation is stored in bf16
    y = h @ wo + bo
    loss = ((y - target.double()) ** 2).mean()
    loss.backward()
    assert float(net.loss.cpu()) == pytest.approx(float(loss), rel=1e-5)
    refs = [w.grad for w in ws] + [b.grad for b in bs] + [wo.grad, bo.grad]
    names = ([f"w{l}" for l in range(len(ws))] + [f"b{l}" for l in range(len(bs))]
             + ["w_out", "b_out"])
    for name, ours, ref in zip(names, net.grads, refs):
        ours = ours.double().cpu().reshape(ref.shape)
        rel = float((ours - ref).norm() / max(ref.norm(), 1e-12))
        assert rel < 0.5 * BF16_ULP, (name, rel)


def test_training_reduces_loss():
    from pursuit_evasion_b200.learned.mlp import FEATURES, ValueMLP

    rows = 1024
    net = ValueMLP(6, seed=0, max_batch=rows)
    g = torch.Generator().manual_seed(2)
    feat = torch.zeros(rows, FEATURES)
    feat[:, :6] = torch.rand(rows, 6, generator=g) * 2 - 1
    target = feat[:, 0] ** 2 + 0.5 * torch.cos(2 * feat[:, 1]) - 0.3 * feat[:, 5]
    net.feat.copy_(feat.to(torch.bfloat16))
    net.target.copy_(target)
    losses = []
    for step in range(1, 301):
        net.loss.zero_()
        net.forward(rows, target=True)
        net.backward(rows)
        net.set_step(step)
        net.adam(lr=1e-3)
        losses.append(float(net.loss.cpu()))
    assert losses[-1] < 0.05 * losses[0]


def gemm_tc_case(epi, M=256, N=256, K=256, seed=0):
    import ctypes

    from pursuit_evasion_b200 import _native

    g = torch.Generator().manual_seed(seed)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)  # [N][K]: a Linear weight
    bias = torch.randn(N, generator=g)
    zpre = torch.randn(M, N, generator=g)
    ref = A.float() @ B.float().t()
    dev = torch.device("cuda", 0)
    Ad, Bd = A.to(dev), B.to(dev)
    C32 = torch.zeros(M, N, device=dev)
    C16 = torch.zeros(M, N, dtype=torch.bfloat16, device=dev)
    biasd, zd = bias.to(dev), zpre.to(dev)
    lib = _native.library()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _native.check(lib.pe_mlp_gemm_tc(p(Ad), p(Bd), M, N, K, K, K, epi,
                                     p(C32) if epi in (0, 1) else None,
                                     p(C16) if epi in (1, 3) else None, N,
                                     p(biasd) if epi == 1 else None,
                                     p(zd) if epi == 3 else None,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    timeouts = ctypes.c_int32()
    _native.check(lib.pe_mlp_gemm_tc_timeouts(ctypes.byref(timeouts)))
    assert timeouts.value == 0
    return ref, bias, zpre, C32.cpu(), C16.float().cpu()


# the last shape takes the 128 x 256 tiles (enough rows for two CTAs per SM)
@pytest.mark.parametrize("M, N, K", [(128, 128, 64), (256, 256, 256), (1024, 256, 128),
                                     (38016, 256, 128)])
def test_tensor_core_gemm_matches_fp32_reference(M, N, K):
    ref, _, _, C32, _ = gemm_tc_case(0, M=M, N=N, K=K)
    torch.testing.assert_close(C32, ref, rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("M", [256, 38016])
def test_tensor_core_gemm_epilogues(M):
    ref, bias, _, C32, C16 = gemm_tc_case(1, M=M)
    z = ref + bias
    torch.testing.assert_close(C32, z, rtol=1e-4, atol=1e-3)
    torch.testing.assert_close(C16, torch.nn.functional.silu(z), rtol=1e-2, atol=2e-2)
    ref, _, zpre, _, C16 = gemm_tc_case(3, M=M)
    s = torch.sigmoid(zpre)
    torch.testing.assert_close(C16, ref * s * (1 + zpre * (1 - s)), rtol=1e-2, atol=5e-2)


# (M, N, K, splits): one k-step per CTA, several, and the surrogate's
# weight-gradient shape (256 x 256 over a batch of 8192 rows)
@pytest.mark.parametrize("M, N, K, splits", [(128, 128, 256, 4), (256, 128, 1024, 4),
                                             (256, 256, 8192, 32), (384, 256, 512, 1)])
def test_tensor_core_split_k_accumulates(M, N, K, splits):
    """pe_mlp_gemm_tc_splitk adds A B^T to what C32 holds, over `splits` K
    ranges with vector atomics; against the FP32 product of the same bf16
    operands."""
    import ctypes

    from pursuit_evasion_b200 import _native

    g = torch.Generator().manual_seed(M + K + splits)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    C0 = torch.randn(M, N, generator=g)
    ref = C0 + A.float() @ B.float().t()
    dev = torch.device("cuda", 0)
    Ad, Bd, C = A.to(dev), B.to(dev), C0.to(dev)
    lib = _native.library()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _native.check(lib.pe_mlp_gemm_tc_splitk(
        p(Ad), p(Bd), M, N, K, K, K, splits, p(C), N,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    timeouts = ctypes.c_int32()
    _native.check(lib.pe_mlp_gemm_tc_timeouts(ctypes.byref(timeouts)))
    assert timeouts.value == 0
    torch.testing.assert_close(C.cpu(), ref, rtol=1e-4, atol=1e-3 * (K / 256) ** 0.5)
