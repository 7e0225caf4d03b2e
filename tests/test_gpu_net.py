"""The learned warm start's tensor-core path on the B200: the tcgen05 GEMM (TMA-fed BF16 operands, FP32 accumulation in
TMEM) against a plain PyTorch FP32 matmul of the same BF16 inputs, on aligned, ragged and split-K shapes; the network's
forward pass and its gradients against the float64 CPU oracle (oracle/net_oracle.py, itself pinned by finite
differences) on the same BF16-rounded weights and inputs; and a short training run that lowers the loss.

Tolerances: the GEMM accumulates exactly-representable BF16 products in FP32, so it agrees with the FP32 matmul to
round-off of the summation order (1e-4 relative to the row scale). The network rounds every activation and every
layer's output gradient to BF16 (8 significant bits), so its outputs agree with the float64 oracle to 3e-2 in the
relative L2 norm; its gradients agree with the oracle that emulates the same roundings to 1e-3 at the output layer,
growing smoothly with depth to 1e-1 at the first layer (the rounding noise compounds through ten layers; 1.5e-1 against
the exact oracle), every layer's gradient direction to a cosine of 0.995."""
import ctypes as C

import numpy as np
import pytest

import net_oracle as no

pytestmark = pytest.mark.gpu


def _gemm(a, b, splits=1):
    import torch
    from bowshock_b200 import _ffi
    m, k = a.shape
    n = b.shape[0]
    d = torch.zeros((m, n), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _ffi.load().bowshock_gemm_bf16(C.c_void_p(a.data_ptr()), a.stride(0), C.c_void_p(b.data_ptr()), b.stride(0),
                                       C.c_void_p(d.data_ptr()), d.stride(0), m, n, k, splits,
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream), C.c_void_p(err.data_ptr()))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "a bounded wait of the GEMM gave up"
    return d


@pytest.mark.parametrize("m,n,k,splits", [(128, 64, 64, 1), (256, 128, 512, 1), (300, 200, 136, 1), (64, 16, 16, 1),
                                          (1000, 256, 1024, 1), (512, 576, 4096, 8), (16, 576, 2048, 5), (131072, 64, 576, 1)])
def test_gemm_matches_torch_fp32(m, n, k, splits):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((n, k), generator=g, device="cuda").to(torch.bfloat16)
    d = _gemm(a, b, splits)
    ref = a.float() @ b.float().T
    scale = ref.abs().amax(dim=1, keepdim=True) + 1e-6
    err = ((d - ref).abs() / scale).max().item()
    assert err < 1e-4, f"{m}x{n}x{k} splits {splits}: max rel err {err:.2e}"


@pytest.mark.parametrize("m,n,k", [(131072, 64, 576), (1000, 256, 1024), (300, 200, 136), (64, 16, 16), (4096, 4096, 256)])
def test_persistent_gemm_equals_per_tile_gemm(m, n, k):
    """The persistent GEMM (CTAs looping over tiles, two TMEM accumulators, epilogue overlapped with the next tile's
    MMAs) gives the per-tile kernel's output bit for bit: the same MMAs in the same K order for every tile."""
    import torch
    from bowshock_b200 import _ffi
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((n, k), generator=g, device="cuda").to(torch.bfloat16)
    lib = _ffi.load()
    was = lib.bowshock_gemm_set_persistent(1)
    try:
        d1 = _gemm(a, b)
        lib.bowshock_gemm_set_persistent(0)
        d0 = _gemm(a, b)
    finally:
        lib.bowshock_gemm_set_persistent(was)
    assert torch.equal(d1, d0)
    ref = a.float() @ b.float().T
    assert ((d1 - ref).abs() / (ref.abs().amax(dim=1, keepdim=True) + 1e-6)).max().item() < 1e-4


def _net_and_oracle(batch=8, seed=5):
    from bowshock_b200.net import Net
    L, n = no.layers()
    net = Net(max_batch=64)
    assert net.nparams == n
    lay = net.layout()
    assert [(l["fc"], l["cin"], l["cout"], l["H"], l["W"], l["up"], l["act"], l["woff"], l["boff"]) for l in L] == lay
    rng = np.random.default_rng(seed)
    p = no.init_params(seed, L, n)
    for l in L:
        p[l["boff"]:l["boff"] + l["cout"]] = (0.05 * rng.standard_normal(l["cout"])).astype(np.float32)
    x = no.bf16_round(rng.standard_normal((batch, no.NET_IN)).astype(np.float32))
    net.set_params(p)
    # the GPU multiplies BF16 copies of the weights (biases stay FP32): the oracle gets the same rounded weights
    pr = p.copy()
    for l in L:
        w = slice(l["woff"], l["woff"] + l["cout"] * l["kin"])
        pr[w] = no.bf16_round(p[w])
    return net, L, n, pr, x, rng


def test_net_forward_matches_oracle():
    net, L, n, pr, x, _ = _net_and_oracle()
    y = net.forward(x)
    ref, _ = no.forward(pr, x, L)
    ref = ref[..., :no.NET_OUT]
    rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert rel < 3e-2, f"forward rel L2 err {rel:.3e}"


def test_net_gradients_match_oracle():
    """Against the oracle with the tensor-core path's BF16 roundings emulated (activations and each layer's output
    gradient stored as BF16): every layer's weight and bias gradients to 3e-2 in the relative L2 norm (the remaining
    difference is FP32 against float64 accumulation, which moves a few BF16 roundings); against the exact float64
    oracle, the rounding compounds through the ten layers below the output, to 1.5e-1 at the first layer."""  # noqa
    net, L, n, pr, x, rng = _net_and_oracle()
    t = rng.standard_normal((x.shape[0], no.NET_CELLS, no.NET_OUT)).astype(np.float32) * 0.5
    mask = (rng.random(no.NET_CELLS) > 0.15).astype(np.uint8)
    net.set_mask(mask)
    loss, g = net.gradients(x, t)
    lemu, gemu = no.loss_and_grad(pr, x, t, mask, L, bf16=True)
    lref, gref = no.loss_and_grad(pr, x, t, mask, L)
    assert abs(loss - lemu) / lemu < 1e-2 and abs(loss - lref) / lref < 1e-2, f"loss {loss} vs {lemu} / {lref}"
    worst = []
    for k, l in enumerate(L):
        for name, sl in (("W", slice(l["woff"], l["woff"] + l["cout"] * l["kin"])), ("b", slice(l["boff"], l["boff"] + l["cout"]))):
            rel_e = np.linalg.norm(g[sl] - gemu[sl]) / (np.linalg.norm(gemu[sl]) + 1e-30)
            rel_x = np.linalg.norm(g[sl] - gref[sl]) / (np.linalg.norm(gref[sl]) + 1e-30)
            worst.append((k, name, rel_e, rel_x))
    print("per-layer gradient rel L2 err (emulated BF16, exact):", [(k, nm, f"{a:.2e}", f"{b:.2e}") for k, nm, a, b in worst])
    for k, name, rel_e, rel_x in worst:
        # the error grows smoothly from the output layer (1e-4) to the first (about 6e-2): BF16 rounding noise
        # propagated backwards through the layers, no step anywhere
        assert rel_e < 1e-1, f"layer {k} {name}: gradient rel L2 err {rel_e:.3e} against the BF16-emulating oracle"
        assert rel_x < 1.5e-1, f"layer {k} {name}: gradient rel L2 err {rel_x:.3e} against the exact oracle"
    assert worst[-2][2] < 1e-3 and worst[-4][2] < 2e-2  # the output layer and the one below it
    for k, l in enumerate(L):  # every layer's gradient points the same way
        sl = slice(l["woff"], l["woff"] + l["cout"] * l["kin"])
        cos = float(np.dot(g[sl], gemu[sl]) / (np.linalg.norm(g[sl]) * np.linalg.norm(gemu[sl]) + 1e-30))
        assert cos > 0.995, f"layer {k}: gradient direction cosine {cos:.4f}"


def test_net_training_lowers_the_loss():
    from bowshock_b200.net import Net
    L, n = no.layers()
    net = Net(max_batch=64)
    net.set_params(no.init_params(1, L, n))
    rng = np.random.default_rng(2)
    N = 256
    x = rng.uniform(-1, 1, (N, no.NET_IN)).astype(np.float32)
    jj, ii = np.meshgrid(np.linspace(0, 1, 32), np.linspace(0, 1, 64), indexing="ij")
    base = np.stack([np.sin(np.pi * ii), np.cos(2 * np.pi * jj), ii * jj, ii - jj, np.sin(3 * jj), np.cos(ii)], -1).reshape(-1, 6)
    t = (x[:, :6, None].transpose(0, 2, 1) * base[None]).astype(np.float32)  # smooth fields scaled by the inputs
    net.set_dataset(x, t)
    loss = net.train(300, 64, 1e-3, seed=0)
    assert np.all(np.isfinite(loss))
    assert loss[-20:].mean() < 0.2 * loss[:5].mean(), f"loss {loss[:5].mean():.3e} -> {loss[-20:].mean():.3e}"
    assert net.last_train_ms() > 0


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("batch,h,w,c,up,n", [(2, 4, 8, 128, 0, 128), (3, 8, 16, 128, 1, 64), (2, 16, 32, 64, 1, 64),
                                              (1, 32, 64, 64, 0, 16), (5, 7, 9, 64, 0, 200), (4, 32, 64, 64, 0, 64),
                                              (3, 4, 8, 64, 0, 64), (2, 8, 16, 64, 0, 256)])
def test_implicit_conv_matches_torch_fp32(batch, h, w, c, up, n, mode):
    """The implicit-GEMM convolution (no im2col matrix; mode 1: A gathered by cp.async into the swizzled tile, mode 2: A
    as 4D TMA boxes of the activations shifted by the tap) against torch's FP32 convolution of the same BF16 input
    (nearest 2x upsampled when up = 1) and weights, zero padding 1. Mode 2 takes no upsampling and needs 128-pixel
    tiles of whole rows or images (odd-batch and ragged-image shapes included where they fit)."""
    import torch
    from bowshock_b200 import _ffi
    H, W = h << up, w << up
    fits = (128 % W == 0) and ((H * W) % 128 == 0 or 128 % (H * W) == 0)
    if mode == 2 and (up or not fits):
        pytest.skip("the TMA form takes no upsampling and needs whole-row tiles")
    g = torch.Generator(device="cuda").manual_seed(batch * 31 + h * 7 + c + n + up)
    x = torch.randn((batch, h, w, c), generator=g, device="cuda").to(torch.bfloat16)
    wt = torch.randn((n, 3, 3, c), generator=g, device="cuda").to(torch.bfloat16)
    d = torch.zeros((batch * H * W, n), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _ffi.load().bowshock_conv3x3_bf16(C.c_void_p(x.data_ptr()), batch, h, w, c, up, C.c_void_p(wt.data_ptr()), n,
                                          C.c_void_p(d.data_ptr()), mode, C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                          C.c_void_p(err.data_ptr()))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "a bounded wait of the convolution gave up"
    xi = x.float().permute(0, 3, 1, 2)
    if up:
        xi = torch.nn.functional.interpolate(xi, scale_factor=2, mode="nearest")
    ref = torch.nn.functional.conv2d(xi, wt.float().permute(0, 3, 1, 2), padding=1).permute(0, 2, 3, 1).reshape(-1, n)
    scale = ref.abs().amax(dim=1, keepdim=True) + 1e-6
    e = ((d - ref).abs() / scale).max().item()
    assert e < 1e-4, f"conv {batch}x{h}x{w}x{c} up {up} -> {n} mode {mode}: max rel err {e:.2e}"


def test_implicit_conv_network_equals_im2col():
    """The network's forward outputs are the same, bit for bit, with its convolutions as TMA-fed implicit GEMMs, as
    gathered implicit GEMMs and through im2col matrices (all three feed the tensor cores the same K blocks in the same
    order); the loss and the weight gradients to the order of their FP32 atomic sums (the loss reduction and the split-K
    weight-gradient GEMMs add their partial sums in whatever order the blocks finish, in every form)."""
    from bowshock_b200.net import Net
    net, L, n, pr, x, rng = _net_and_oracle()
    t = rng.standard_normal((x.shape[0], no.NET_CELLS, no.NET_OUT)).astype(np.float32) * 0.5
    outs = []
    for mode in (Net.CONV_TMA, Net.CONV_GATHER, Net.CONV_IM2COL):
        net.set_conv_mode(mode)
        y = net.forward(x)
        loss, g = net.gradients(x, t)
        outs.append((y, loss, g))
    y0, l0, g0 = outs[-1]
    for y1, l1, g1 in outs[:-1]:
        assert np.array_equal(y1, y0)
        assert abs(l1 - l0) <= 1e-5 * abs(l0)  # 98,304 FP32 terms added atomically in any order
        for l in L:
            sl = slice(l["woff"], l["boff"] + l["cout"])
            e = np.linalg.norm(g1[sl] - g0[sl]) / (np.linalg.norm(g0[sl]) + 1e-30)
            assert e < 1e-5, f"layer gradient differs by {e:.2e}"


def test_net_forward_repeatable():
    """Two forward passes of the same inputs give the same outputs, bit for bit, and a pass of a smaller batch the same
    rows (the epilogue and the GEMM tiles do not depend on the batch's other rows)."""
    net, L, n, pr, x, _ = _net_and_oracle()
    y1 = net.forward(x)
    y2 = net.forward(x)
    assert np.array_equal(y1, y2)
    y3 = net.forward(x[:3])
    assert np.array_equal(y3, y1[:3])
