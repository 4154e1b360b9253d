"""Kernels of the learned warm start: the tcgen05 GEMM (bf16 operands, fp32
accumulation in tensor memory) against a plain PyTorch fp32 matmul of the same
bf16 inputs."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from wavesim_b200 import _lib as L
    return L.lib


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 192), (1000, 32, 1728), (4096, 64, 896), (77, 130, 128)])
def test_gemm_bf16_matches_fp32_matmul(gpu, M, N, K):
    import torch
    lib = _lib()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    Cm = torch.zeros(M, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.ws_gemm_bf16(A.data_ptr(), B.data_ptr(), Cm.data_ptr(), None, None, M, N, K, K, K, N, 0,
                          err.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    ref = A.float() @ B.float().t()
    assert float((Cm - ref).norm() / ref.norm()) < 1e-5


def test_gemm_bias_relu_epilogue(gpu):
    import torch
    lib = _lib()
    M, N, K = 256, 96, 128
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    bias = torch.randn(N, device="cuda")
    out = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16)
    rc = lib.ws_gemm_bf16(A.data_ptr(), B.data_ptr(), None, out.data_ptr(), bias.data_ptr(), M, N, K, K, K, N, 1,
                          None, None)
    torch.cuda.synchronize()
    assert rc == 0
    ref = torch.relu(A.float() @ B.float().t() + bias)
    assert float((out.float() - ref).norm() / ref.norm()) < 1e-2  # bf16 output rounding


def _bf16(t):
    import torch
    return t.to(torch.bfloat16)


def _conv_ref(xin_f32, Wf, bias, C, Cout, vol):
    """torch fp32 conv3d of channels-last [vox][C] with W [Cout][27 C] in tap order ((dz*3+dy)*3+dx)*C + c."""
    import torch
    b, d, h, w = vol
    xin = xin_f32.reshape(b, d, h, w, C).permute(0, 4, 1, 2, 3)
    wt = Wf[:, :27 * C].reshape(Cout, 3, 3, 3, C).permute(0, 4, 1, 2, 3)
    y = torch.nn.functional.conv3d(xin, wt, bias, padding=1)
    return y.permute(0, 2, 3, 4, 1).reshape(-1, Cout)


@pytest.mark.parametrize("C,Cout,vol", [(8, 32, (1, 8, 16, 24)), (32, 32, (2, 8, 8, 8)), (64, 96, (1, 6, 10, 14)),
                                        (96, 128, (1, 4, 8, 8)), (32, 2, (1, 8, 8, 16)), (16, 160, (1, 4, 4, 12)),
                                        (8, 48, (1, 3, 5, 7))])
def test_conv3_matches_torch_conv3d(gpu, C, Cout, vol):
    """The implicit-GEMM convolution (cp.async gather + tcgen05) against torch's
    fp32 conv3d of the same bf16 inputs: fp32 and bf16+ReLU epilogues, ragged
    voxel counts, every output-channel tile."""
    import torch

    from wavesim_b200 import warmstart as W
    b, d, h, w = vol
    nvox = b * d * h * w
    g = torch.Generator(device="cuda").manual_seed(C * 131 + Cout)
    kp = W.pad64(27 * C)
    x = _bf16(torch.randn(nvox, C, device="cuda", generator=g))
    Wt = _bf16(torch.randn(Cout, kp, device="cuda", generator=g) / np.sqrt(27 * C))
    bias = torch.randn(Cout, device="cuda", generator=g)
    ref = _conv_ref(x.float(), Wt.float(), bias, C, Cout, vol)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y32 = torch.full((nvox, Cout), float("nan"), device="cuda")
    W._ck(W.lib().ws_conv3_fwd_bf16(x.data_ptr(), Wt.data_ptr(), bias.data_ptr(), y32.data_ptr(), None, b, d, h, w, C,
                                    Cout, kp, 3, err.data_ptr(), None), "conv")
    yb = torch.empty(nvox, Cout, device="cuda", dtype=torch.bfloat16)
    W._ck(W.lib().ws_conv3_fwd_bf16(x.data_ptr(), Wt.data_ptr(), bias.data_ptr(), None, yb.data_ptr(), b, d, h, w, C,
                                    Cout, kp, 1, err.data_ptr(), None), "conv")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert float((y32 - ref).norm() / ref.norm()) < 1e-5
    rr = torch.relu(ref)
    assert float((yb.float() - rr).norm() / rr.norm()) < 1e-2


@pytest.mark.parametrize("Cu,Cx,Cout,vol", [(64, 32, 32, (1, 8, 8, 16)), (128, 96, 96, (1, 4, 4, 4)),
                                            (96, 64, 64, (2, 4, 6, 8))])
def test_conv3_upcat_matches_torch(gpu, Cu, Cx, Cout, vol):
    """The decoder convolution reading [nearest x2 upsampling of U, X] in place."""
    import torch

    from wavesim_b200 import warmstart as W
    b, d, h, w = vol
    nvox = b * d * h * w
    g = torch.Generator(device="cuda").manual_seed(Cu + 7 * Cx)
    C = Cu + Cx
    kp = W.pad64(27 * C)
    U = _bf16(torch.randn(nvox // 8, Cu, device="cuda", generator=g))
    X = _bf16(torch.randn(nvox, Cx, device="cuda", generator=g))
    Wt = _bf16(torch.randn(Cout, kp, device="cuda", generator=g) / np.sqrt(27 * C))
    bias = torch.randn(Cout, device="cuda", generator=g)
    up = U.float().reshape(b, d // 2, h // 2, w // 2, Cu)
    up = up.repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3).reshape(nvox, Cu)
    ref = torch.relu(_conv_ref(torch.cat([up, X.float()], 1), Wt.float(), bias, C, Cout, vol))
    yb = torch.empty(nvox, Cout, device="cuda", dtype=torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    W._ck(W.lib().ws_conv3_upcat_fwd_bf16(U.data_ptr(), X.data_ptr(), Wt.data_ptr(), bias.data_ptr(), None,
                                          yb.data_ptr(), b, d, h, w, Cu, Cx, Cout, kp, 1, err.data_ptr(), None),
          "conv upcat")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert float((yb.float() - ref).norm() / ref.norm()) < 1e-2


def test_features_and_envelope_kernels(gpu):
    """ws_net_features against its numpy statement, and ws_net_envelope_to_field
    against WaveSim.initial_field's host continuation into the boundary."""
    import torch

    import wavesim_b200 as ws
    from wavesim_b200 import warmstart as W
    rng = np.random.default_rng(4)
    Ny, Nx, Nz = 16, 24, 8
    n = (1.33 + 0.17 * (rng.random((Ny, Nx, Nz)) > 0.7)).astype(np.float32)
    k0, nbg = 2 * np.pi * 0.25, 1.33
    f = W.features(n, k0, nbg, torch, torch.device("cuda")).float().cpu().numpy()
    dn = n.astype(np.float64) - nbg
    phi = k0 * np.cumsum(dn, axis=2)
    src = np.zeros_like(dn)
    src[:, :, 0] = 1
    want = np.stack([dn / 0.2, src, np.cos(phi), np.sin(phi)], -1).reshape(-1, 4, order="F")
    assert np.abs(f[:, :4] - want).max() < 1e-2 and not f[:, 4:].any()

    sim = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [4, 6, 8]})
    env = (rng.standard_normal((Ny, Nx, Nz)) + 1j * rng.standard_normal((Ny, Nx, Nz))).astype(np.complex64)
    pred = torch.from_numpy(np.stack([env.real, env.imag], -1).reshape(-1, 2, order="F").copy()).cuda()
    N = (W.I64 * 3)(*[int(v) for v in sim.N[:3]])
    r0 = (W.I64 * 3)(*[int(sim.roi[0, d]) - 1 for d in range(3)])
    rn = (W.I64 * 3)(Ny, Nx, Nz)
    psi = torch.empty(int(np.prod(sim.N[:3])), dtype=torch.complex64, device="cuda")
    kz = k0 * nbg
    W._ck(W.lib().ws_net_envelope_to_field(pred.data_ptr(), N, r0, rn, 0.5, kz, 0, psi.data_ptr(), None), "env")
    got = psi.cpu().numpy().reshape(tuple(sim.N[:3]), order="F")
    field = 0.5 * env * np.exp(1j * kz * np.arange(Nz))[None, None, :]
    want = np.asarray(sim.initial_field(field))[..., 0]
    assert np.abs(got - want).max() < 1e-4 * np.abs(want).max()
    # the same envelope in the half-resolution (space-to-depth) layout
    half = torch.from_numpy(W.field_to_target(env, 1.0, half=True)).cuda()
    psi2 = torch.empty_like(psi)
    W._ck(W.lib().ws_net_envelope_to_field(half.data_ptr(), N, r0, rn, 0.5, kz, 1, psi2.data_ptr(), None), "env")
    assert float((psi2 - psi).abs().max()) < 1e-5 * float(psi.abs().max())


def test_space_to_depth_matches_numpy(gpu):
    """ws_net_space_to_depth against the host layout of the training targets."""
    import torch

    from wavesim_b200 import warmstart as W
    rng = np.random.default_rng(7)
    shape = (16, 32, 48)  # (Ny, Nx, Nz)
    x = rng.standard_normal((int(np.prod(shape)), 8)).astype(np.float32)
    xb = torch.from_numpy(x).cuda().to(torch.bfloat16)
    y = W.space_to_depth(xb, shape, torch).float().cpu().numpy()
    Ny, Nx, Nz = shape
    v = xb.float().cpu().numpy().reshape(Nz // 2, 2, Nx // 2, 2, Ny // 2, 2, 8)
    want = np.transpose(v, (0, 2, 4, 1, 3, 5, 6)).reshape(-1, 64)
    assert np.array_equal(y, want)


def _gpu_net(widths, seed=0):
    from wavesim_b200.warmstart import WarmStartNet
    return WarmStartNet(widths=widths, seed=seed)


def _run_small_net(widths, seed, vol=(1, 8, 8, 16)):
    import torch

    from wavesim_b200 import warmstart as W
    net = _gpu_net(widths, seed=seed)
    nvox = int(np.prod(vol))
    rng = np.random.default_rng(seed + 1)
    xf = torch.from_numpy(rng.standard_normal((nvox, 8)).astype(np.float32)).cuda()
    x = torch.empty(nvox, 8, device="cuda", dtype=torch.bfloat16)
    W._ck(W.lib().ws_net_f32_to_bf16(xf.data_ptr(), x.data_ptr(), xf.numel(), None), "cvt")
    target = torch.from_numpy(rng.standard_normal((nvox, 2)).astype(np.float32)).cuda()
    for l in net.layers:
        l.zero_grad()
        l.record = []
    out, acts = net.forward(x, vol, keep=True)
    grad = torch.empty_like(out)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    W._ck(W.lib().ws_net_mse(out.data_ptr(), target.data_ptr(), grad.data_ptr(), loss.data_ptr(), nvox, 2, 2, None),
          "mse")
    net.backward(acts, grad, vol)
    torch.cuda.synchronize()
    net._check_err()
    return net, x, out, vol


def test_network_layers_match_fp64_oracle(gpu):
    """Each convolution layer on its own, fed the GPU's input, output and
    incoming gradient: forward output, weight, bias and input gradients of the
    bf16 tensor-core kernels against the FP64 restatement."""
    from oracle import warmstart_oracle as O
    net, x, out, vol = _run_small_net((8, 8, 16, 16), seed=3)
    b, d, h, w = vol
    vols = {k: (b, d >> k, h >> k, w >> k) for k in range(4)}
    for i, l in enumerate(net.layers):
        (xi, yi, dyi, dxi), = l.record
        nv = xi.shape[0]
        v = next(vv for vv in vols.values() if vv[0] * vv[1] * vv[2] * vv[3] == nv)
        W64 = l.wb.float().cpu().numpy()[:, :l.k].astype(np.float64)
        b64 = l.b.cpu().numpy().astype(np.float64)
        col = O.im2col(xi.float().cpu().numpy().astype(np.float64), v, l.cin)
        pre = col @ W64.T + b64
        g = dyi.cpu().numpy().astype(np.float64)
        if l.relu:
            yr = np.maximum(pre, 0)
            assert np.linalg.norm(yi.float().cpu().numpy() - yr) <= 1e-2 * np.linalg.norm(yr), i
            g = g * (yi.float().cpu().numpy() > 0)
        gw = g.T @ col
        gb = g.sum(axis=0)
        ew = np.linalg.norm(l.gw.cpu().numpy()[:, :l.k] - gw) / max(np.linalg.norm(gw), 1e-30)
        eb = np.linalg.norm(l.gb.cpu().numpy() - gb) / max(np.linalg.norm(gb), 1e-30)
        assert ew < 1.5e-2 and eb < 1e-4, (i, ew, eb)
        if dxi is not None:
            dx = O.col2im(g @ W64, v, l.cin)
            ex = np.linalg.norm(dxi.cpu().numpy() - dx) / max(np.linalg.norm(dx), 1e-30)
            assert ex < 1.5e-2, (i, ex)


def test_network_forward_matches_fp64_oracle(gpu):
    from oracle.warmstart_oracle import Net
    net, x, out, vol = _run_small_net((8, 8, 16, 16), seed=5)
    weights = [(l.wb.float().cpu().numpy()[:, :l.k], l.b.cpu().numpy()) for l in net.layers]
    o_out, _ = Net(weights, (8, 8, 16, 16)).forward(x.float().cpu().numpy().astype(np.float64), vol)
    rel_out = np.linalg.norm(out.cpu().numpy() - o_out) / np.linalg.norm(o_out)
    assert rel_out < 3e-2, rel_out


def test_network_training_reduces_loss(gpu):
    """A few Adam steps on a fixed smooth target reduce the loss."""
    import torch

    from wavesim_b200 import warmstart as W
    net = _gpu_net((8, 16, 16, 16), seed=1)
    vol = (1, 16, 16, 16)
    z = np.arange(16)
    f = np.zeros((16, 16, 16, 8), np.float32)
    f[..., 2] = np.cos(1.3 * z)[:, None, None]
    f[..., 3] = np.sin(1.3 * z)[:, None, None]
    xf = torch.from_numpy(f.reshape(-1, 8)).cuda()
    x = torch.empty_like(xf, dtype=torch.bfloat16)
    W._ck(W.lib().ws_net_f32_to_bf16(xf.data_ptr(), x.data_ptr(), xf.numel(), None), "cvt")
    t = torch.from_numpy(np.stack([f[..., 2], f[..., 3]], -1).reshape(-1, 2) * 0.5).cuda()
    losses = [net.train_step(x, t, vol, 3e-3) for _ in range(40)]
    assert losses[-1] < 0.3 * losses[0], losses[::8]


def test_network_warm_start_runs_on_device(gpu):
    """An (untrained) network as the warm start of a solve: the prediction
    stays on the device and the solve still reaches the cold answer."""
    import wavesim_b200 as ws
    from wavesim_b200.warmstart import WarmStart
    from wavesim_b200.workloads import sphere_medium
    n = sphere_medium(32, np.random.default_rng(21))
    sim = ws.WaveSim(n, {"lambda": 1.0, "pixel_size": 0.25, "boundary_widths": [16, 16, 16], "energy_threshold": 1e-4})
    src = ws.Source(np.ones((32, 32)), [1, 1, 1])
    E, st = sim.exec(src)
    Ew, sw = sim.exec(src, warm_start=WarmStart())
    assert float(np.linalg.norm(Ew - E) / np.linalg.norm(E)) < 2e-2
