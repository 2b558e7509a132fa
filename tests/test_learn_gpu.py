"""Tensor-core kernels of the learned proposal against PyTorch float32 references of the same ops.

GEMM: inputs are BF16, so the reference multiplies the same BF16 values in float32; the
tolerance (relative to the largest reference value) is 1e-5, float32 accumulation over K <= 2304.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GEMM_TOL = 1e-5


def gemm(A, B, epi, bias=None, slope=0.2, out=None, splits=0):
    from shotsweep_b200 import _lib
    M, K = A.shape
    N = B.shape[0]
    if out is None:
        dt = torch.bfloat16 if epi == _lib.EPI_BIAS_LRELU_BF16 else torch.float32
        out = torch.zeros(M, N, dtype=dt, device=A.device)
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    L = _lib.load()
    _lib.check(L.ss_gemm_bf16(_lib.ptr(A), A.stride(0), _lib.ptr(B), B.stride(0), M, N, K, epi, _lib.ptr(out),
                              out.stride(0), _lib.ptr(bias), slope, splits, _lib.ptr(err),
                              _lib.stream_handle(A.device)), 'ss_gemm_bf16')
    torch.cuda.synchronize()
    assert err.item() == 0
    return out


@pytest.mark.parametrize('M,N,K', [(200, 40, 40), (1000, 256, 1152), (300, 96, 520), (129, 300, 64),
                                   (8192, 256, 2304), (64, 32, 9216), (333, 37, 32), (40000, 576, 32),
                                   (517, 130, 96)])
def test_gemm_f32_matches_float32_matmul(M, N, K):
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device='cuda', generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    got = gemm(A, B, _lib.EPI_F32)
    assert (got - ref).abs().max().item() <= GEMM_TOL * ref.abs().max().item() * 10 + 1e-6 * K ** 0.5
    bias = torch.randn(N, device='cuda', generator=g)
    got = gemm(A, B, _lib.EPI_BIAS_F32, bias=bias)
    assert torch.allclose(got, ref + bias, rtol=0, atol=GEMM_TOL * ref.abs().max().item() * 10 + 1e-6 * K ** 0.5)


@pytest.mark.parametrize('M,N,K,layout,epi', [(32, 576, 4000, 3, 'add'), (64, 40, 1000, 3, 'add'),
                                                (256, 128, 777, 3, 'add'), (136, 64, 96, 3, 'f32'),
                                                (1000, 576, 32, 2, 'bf16'), (300, 136, 200, 2, 'f32'),
                                                (4096, 1152, 128, 2, 'bf16')])
def test_gemm_operand_layouts(M, N, K, layout, epi):
    """Operands stored K-outer and read in place through M/N-major descriptors (the weight-gradient and
    input-gradient GEMMs of the proposal network) give the K-major product: the same BF16 values multiplied in
    float32, split-K accumulation and the BF16 epilogue included."""
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(M + 3 * N + 7 * K + layout)
    A = torch.randn(M, K, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device='cuda', generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    As = A.T.contiguous() if layout & 1 else A
    Bs = B.T.contiguous() if layout & 2 else B
    code = {'add': _lib.EPI_F32_ADD, 'f32': _lib.EPI_F32, 'bf16': _lib.EPI_BIAS_LRELU_BF16}[epi]
    start = torch.randn(M, N, device='cuda', generator=g) if epi == 'add' else None
    out = start.clone() if epi == 'add' else torch.zeros(M, N, device='cuda', dtype=torch.bfloat16 if epi == 'bf16'
                                                         else torch.float32)
    err = torch.zeros(1, dtype=torch.int32, device='cuda')
    L = _lib.load()
    _lib.check(L.ss_gemm_bf16_layout(_lib.ptr(As), As.stride(0), _lib.ptr(Bs), Bs.stride(0), M, N, K, layout, code,
                                     _lib.ptr(out), out.stride(0), None, 1.0, 0, _lib.ptr(err),
                                     _lib.stream_handle(A.device)), 'ss_gemm_bf16_layout')
    torch.cuda.synchronize()
    assert err.item() == 0
    if epi == 'add':
        ref = ref + start
    scale = ref.abs().max().item()
    if epi == 'bf16':   # one BF16 rounding of the float32 product
        assert ((out.float() - ref).abs() <= 2 ** -8 * ref.abs() + 1e-5 * scale).all()
    else:
        assert (out - ref).abs().max().item() <= 1e-5 * scale * 10 + 1e-6 * K ** 0.5


def test_gemm_split_k_accumulates():
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(11)
    A = torch.randn(64, 50000, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(48, 50000, device='cuda', generator=g).to(torch.bfloat16)
    ref = A.double() @ B.double().T
    start = torch.randn(64, 48, device='cuda', generator=g)
    got = gemm(A, B, _lib.EPI_F32_ADD, out=start.clone())
    err = (got.double() - (ref + start.double())).abs().max().item()
    assert err <= 1e-4 * ref.abs().max().item()


@pytest.mark.parametrize('N', [64, 37])
def test_gemm_bias_leaky_relu_bf16(N):
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(5)
    A = torch.randn(517, 72, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(N, 72, device='cuda', generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device='cuda', generator=g)
    x = A.float() @ B.float().T + bias
    ref = torch.where(x > 0, x, 0.2 * x)
    got = gemm(A, B, _lib.EPI_BIAS_LRELU_BF16, bias=bias).float()
    assert ((got - ref).abs() <= 2 ** -8 * ref.abs() + 1e-5).all()     # one BF16 rounding


def small_batch(B, seed=0):
    """Stored float16 gathers of B synthetic models (simulated) and their normalised targets."""
    from shotsweep_b200 import engine, gpu, synth, train_inputs as TI
    models = np.stack([synth.model(synth.FAMILIES[i % 4], [seed, i]) for i in range(B)])
    eng = gpu.Sim(device='cuda').engine
    g = eng.forward(torch.tensor(models, device='cuda'), engine.scaled_wavelet(gpu.RICKER, eng.device))
    stored = TI.stored_gathers(g)
    scale = float(stored.float().abs().max().item())
    y = TI.targets(torch.tensor(models, device='cuda'))
    return stored, scale, y, models


def test_network_layers_match_cpu_oracle():
    """Every layer, forward and backward, against the float32 CPU restatement, each from the GPU's own inputs
    (so that BF16 rounding differences do not compound): layer outputs and the pre-activation gradients handed
    down within 5e-4 (rel. L2; only BF16 rounding flips), weight and bias gradients within 1e-4, the head and the
    loss gradient within 1e-5.  End to end from the same weights (a sanity bound, not the parity check) the
    prediction agrees within 5e-2 and every gradient within 0.15: a randomly initialised 14-layer network
    roughly doubles a relative difference per layer, forward and again backward."""
    from oracle import proposal_oracle as PO
    from shotsweep_b200 import proposal as P
    B = 2
    stored, scale, y, _ = small_batch(B)
    net = P.ProposalNet(B, seed=3)
    net.ids.copy_(torch.arange(B, dtype=torch.int32))
    net.load_batch(stored, scale, y)
    net.forward()
    net.backward()
    torch.cuda.synchronize()
    net.check()
    params = net.params.cpu().numpy()
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-30))
    xs = [net.x0.view(B, P.T_IN, P.X_IN, P.S_IN).float().cpu().numpy()]
    for i, (L, sh) in enumerate(zip(P.LAYERS, net.shapes)):
        out = PO.layer_forward(params, i, xs[-1]).numpy()
        got = net.y[i].float().cpu().numpy().reshape(out.shape)
        assert rel(got, out) <= 5e-4, (L.name, rel(got, out))
        xs.append(got)
    pred = PO.head_forward(params, xs[-1])
    assert rel(net.pred.cpu().numpy(), pred) <= 1e-5
    dph = PO.l1_tanh_grad(net.pred.cpu().numpy(), net.target.cpu().numpy())
    assert rel(net.dpre_head.cpu().numpy(), dph) <= 1e-5
    g = net.grads.cpu().numpy()
    dw, db, below = PO.head_backward(params, xs[-1], net.dpre_head.cpu().numpy())
    o, n = net.lay['head.w']
    assert rel(g[o:o + n], dw) <= 1e-5
    # the bias gradient is a sum of 9800 terms with cancellation: bounded against the sum of their magnitudes
    assert abs(g[net.lay['head.b'][0]] - db) <= 1e-5 * np.abs(net.dpre_head.cpu().numpy()).sum()
    assert rel(net.dpre[-1].float().cpu().numpy().reshape(below.shape), below) <= 5e-4
    for i in range(len(P.LAYERS) - 1, -1, -1):
        L, (hi, wi, ho, wo, K, Kc, N) = P.LAYERS[i], net.shapes[i]
        dpre = net.dpre[i].float().cpu().numpy()
        dW, db, below = PO.layer_backward(params, i, xs[i], dpre)
        o, n = net.lay[L.name + '.w']
        gw = g[o:o + n].reshape(N, Kc)[:, :K]
        ob, nb = net.lay[L.name + '.b']
        assert rel(gw, dW) <= 1e-4, (L.name, 'w', rel(gw, dW))
        assert rel(g[ob:ob + nb], db) <= 1e-4, (L.name, 'b', rel(g[ob:ob + nb], db))
        if below is not None:
            got = net.dpre[i - 1].float().cpu().numpy().reshape(below.shape)
            assert rel(got, below) <= 5e-4, (L.name, 'dpre', rel(got, below))
    pred_e2e, loss, grad = PO.loss_and_grads(params, xs[0], net.target.cpu().numpy())
    assert rel(net.pred.cpu().numpy(), pred_e2e) <= 5e-2
    assert abs(net.loss_sum.item() / (B * 70 * 70) - loss) <= 5e-2 * loss
    for name, (o, n) in net.lay.items():
        assert rel(g[o:o + n], grad[o:o + n]) <= 0.15, name


def test_adamw_step_and_training_reduces_loss():
    from oracle import proposal_oracle as PO
    from shotsweep_b200 import proposal as P
    B = 4
    stored, scale, y, _ = small_batch(B, seed=1)
    net = P.ProposalNet(B, seed=4)
    net.ids.copy_(torch.arange(B, dtype=torch.int32))
    p0 = net.params.cpu().numpy()
    net.train_step(stored, scale, y)
    torch.cuda.synchronize()
    g = net.grads.cpu().numpy()
    ref, _, _ = PO.adamw_step(p0, g, np.zeros_like(p0), np.zeros_like(p0), 1, 5e-4)
    assert np.abs(net.params.cpu().numpy() - ref).max() <= 1e-6
    assert torch.equal(net.p16, net.params.to(torch.bfloat16))
    losses = []
    for _ in range(30):
        net.train_step(stored, scale, y)
        losses.append(net.loss_sum.item() / (B * 70 * 70))
    net.check()
    assert losses[-1] < 0.5 * losses[0]


# (B, Hin, Win, Cin, KH, KW, sh, sw, ph, pw, up): the network's three layer families, a 1x1 layer, a geometry
# that takes the run-time-geometry kernels (KW = 2, upsampling by 3) and one whose Cin / 8 is not a power of two
CONV_CASES = [(2, 50, 14, 32, 4, 1, 2, 1, 1, 0, 1), (2, 31, 13, 64, 3, 3, 2, 2, 1, 1, 1),
              (2, 10, 9, 16, 3, 3, 1, 1, 1, 1, 2), (3, 1, 1, 128, 1, 1, 1, 1, 0, 0, 1),
              (2, 7, 6, 8, 2, 3, 1, 2, 0, 1, 3), (2, 9, 11, 24, 3, 3, 1, 1, 1, 1, 1)]


def _unfold_cols(x, conv):
    """Columns [pixels][(kh, kw, c)] of NHWC x (float), through torch's unfold on the upsampled map."""
    import torch.nn.functional as F
    B, H, W, C, KH, KW, sh, sw, ph, pw, up = conv
    xin = x.permute(0, 3, 1, 2)
    if up > 1:
        xin = F.interpolate(xin, scale_factor=up, mode='nearest')
    u = F.unfold(xin, (KH, KW), padding=(ph, pw), stride=(sh, sw))
    return u.view(B, C, KH * KW, -1).permute(0, 3, 2, 1).reshape(-1, KH * KW * C)


@pytest.mark.parametrize('conv', CONV_CASES)
def test_im2col_matches_unfold(conv):
    """ss_im2col_bf16 copies: bit-exact against torch's unfold in the kernel's (kh, kw, c) column order."""
    import ctypes
    from shotsweep_b200 import _lib
    B, H, W, C = conv[:4]
    g = torch.Generator(device='cuda').manual_seed(sum(conv))
    x = torch.randn(B, H, W, C, device='cuda', generator=g).to(torch.bfloat16)
    ref = _unfold_cols(x.float(), conv)
    cols = torch.full_like(ref, float('nan'), dtype=torch.bfloat16)
    L = _lib.load()
    _lib.check(L.ss_im2col_bf16(_lib.ptr(x), (ctypes.c_int32 * 11)(*conv), ref.shape[1], _lib.ptr(cols),
                                _lib.stream_handle(x.device)), 'ss_im2col_bf16')
    torch.cuda.synchronize()
    assert torch.equal(cols.float(), ref)


@pytest.mark.parametrize('conv', [c for c in CONV_CASES if c[3] % 8 == 0 and (c[3] // 8) & (c[3] // 8 - 1) == 0])
def test_col2im16_matches_fold(conv):
    """ss_col2im16_lrelu_bf16: BF16 column gradients summed back onto the input in float32 (torch's fold, then the
    upsampling's adjoint), times the leaky-ReLU derivative of y, one BF16 rounding: within one BF16 unit."""
    import ctypes
    from shotsweep_b200 import _lib
    B, H, W, C = conv[:4]
    g = torch.Generator(device='cuda').manual_seed(7 + sum(conv))
    x = torch.randn(B, H, W, C, device='cuda', generator=g).to(torch.bfloat16)
    xr = x.float().requires_grad_(True)
    cols = _unfold_cols(xr, conv)
    dcols = torch.randn(cols.shape, device='cuda', generator=g).to(torch.bfloat16)
    cols.backward(dcols.float())
    ref = torch.where(x.float() > 0, xr.grad, 0.2 * xr.grad)
    out = torch.full_like(x, float('nan'))
    L = _lib.load()
    _lib.check(L.ss_col2im16_lrelu_bf16(_lib.ptr(dcols), (ctypes.c_int32 * 11)(*conv), cols.shape[1], _lib.ptr(x),
                                        0.2, _lib.ptr(out), C, _lib.stream_handle(x.device)), 'ss_col2im16_lrelu_bf16')
    torch.cuda.synchronize()
    assert ((out.float() - ref).abs() <= 2 ** -8 * ref.abs() + 1e-6).all()


@pytest.mark.parametrize('S,T,X,B', [(5, 37, 70, 6), (9, 11, 13, 3)])
def test_gathers_nhwc_matches_restatement(S, T, X, B):
    """ss_gathers_nhwc_bf16: rows `ids` of stored float16 gathers [n][S][T][X], divided by the scale (correctly
    rounded, as torch divides) and rounded to BF16, as NHWC [B][T][X][S]: bit-exact (S = 5 takes the pixel-per-thread
    kernel with shared-memory staged stores, S = 9 the element-per-thread one)."""
    from shotsweep_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(S * T + X)
    n = B + 4
    stored = (torch.randn(n, S, T, X, device='cuda', generator=g) * 300).to(torch.float16)
    ids = torch.randperm(n, device='cuda', generator=g)[:B].to(torch.int32)
    scale = 123.456
    ref = (stored[ids.long()].float() / scale).permute(0, 2, 3, 1).to(torch.bfloat16)
    out = torch.full((B, T, X, S), float('nan'), device='cuda', dtype=torch.bfloat16)
    L = _lib.load()
    _lib.check(L.ss_gathers_nhwc_bf16(_lib.ptr(stored), _lib.ptr(ids), B, S, T, X, scale, _lib.ptr(out),
                                      _lib.stream_handle(out.device)), 'ss_gathers_nhwc_bf16')
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
