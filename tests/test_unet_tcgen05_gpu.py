"""The U-Net convolution on the tensor cores (lfts_conv3d_bf16: tcgen05
implicit GEMM, BF16 operands, FP32 accumulation in tensor memory) against
torch's FP32 periodic conv3d of the same BF16-rounded inputs and weights, for
every layer shape of the 24-channel U-Net (channel padding, the padded skip
concatenations, the 1x1x1 output layer, a partial 128-position tile); then the
whole tensor-core U-Net against the FP32 torch model."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference(x, conv, relu):
    import torch
    import torch.nn.functional as F
    w = conv.weight.detach().to(torch.bfloat16).float()
    b = conv.bias.detach().float()
    k = w.shape[-1]
    xp = F.pad(x, (k // 2,) * 6, mode="circular") if k > 1 else x
    y = F.conv3d(xp, w, b)
    return F.relu(y) if relu else y


@pytest.mark.parametrize("cin,cin_pad,cout,k,grid,batch", [
    (2, 16, 24, 3, (8, 8, 8), 2),      # first layer (input channels padded 2 -> 16, outputs 24 -> 32)
    (24, 32, 48, 3, (8, 8, 8), 2),
    (48, 48, 96, 3, (4, 4, 4), 2),
    (144, 144, 48, 3, (8, 8, 8), 1),   # decoder concat, largest K
    (96, 96, 96, 3, (4, 6, 5), 1),     # non-cubic box, 120 positions: one partial tile
    (24, 32, 1, 1, (8, 8, 8), 2),      # 1x1x1 output layer
    # grids with H % 16 == 0 and W % 8 == 0 take the halo-staged kernel
    (2, 16, 24, 3, (16, 16, 16), 2), (24, 32, 48, 3, (16, 16, 16), 1), (144, 144, 48, 3, (8, 16, 8), 2),
    (96, 96, 96, 3, (6, 32, 24), 1),
])
@pytest.mark.parametrize("relu", [True, False])
def test_conv_matches_torch(cin, cin_pad, cout, k, grid, batch, relu):
    import torch
    from langevinfts_b200.learned import conv3d_tcgen05, pack_conv
    torch.manual_seed(cin * 31 + cout)
    conv = torch.nn.Conv3d(cin, cout, k).cuda()
    x = torch.randn(batch, cin, *grid, device="cuda").to(torch.bfloat16).float()
    layer = pack_conv(conv, list(range(cin)), cin_pad)
    h = x.permute(0, 2, 3, 4, 1)
    h = torch.nn.functional.pad(h, (0, cin_pad - cin)).to(torch.bfloat16).contiguous()
    got = conv3d_tcgen05(h, layer, relu).float()
    torch.cuda.synchronize()
    ref = _reference(x, conv, relu).permute(0, 2, 3, 4, 1)
    scale = float(ref.abs().max())
    # BF16 rounding of the output (2^-8 relative) plus FP32 accumulation order
    assert float((got[..., :cout] - ref).abs().max()) <= 8e-3 * scale + 1e-6
    assert float(got[..., cout:].abs().max() if got.shape[-1] > cout else 0) == 0.0  # padded channels stay zero


@pytest.mark.parametrize("tz", ["1", "2"])
@pytest.mark.parametrize("cin,cin_pad,cout,grid,batch", [
    (2, 16, 24, (16, 16, 16), 2), (24, 32, 48, (8, 32, 16), 1), (48, 48, 48, (4, 16, 8), 3),
    (96, 96, 96, (6, 32, 24), 1), (72, 80, 24, (2, 16, 8), 2)])
def test_conv_halo_tiles(monkeypatch, tz, cin, cin_pad, cout, grid, batch):
    """The halo kernel with one and with two output planes per CTA (the
    LFTS_CONV_TZ override), each with the ring depth its shared memory allows."""
    import torch
    from langevinfts_b200.learned import conv3d_tcgen05, pack_conv
    monkeypatch.setenv("LFTS_CONV_KSLICE", "0")
    monkeypatch.setenv("LFTS_CONV_TZ", tz)
    torch.manual_seed(cin * 17 + cout)
    conv = torch.nn.Conv3d(cin, cout, 3).cuda()
    x = torch.randn(batch, cin, *grid, device="cuda").to(torch.bfloat16).float()
    layer = pack_conv(conv, list(range(cin)), cin_pad)
    h = torch.nn.functional.pad(x.permute(0, 2, 3, 4, 1), (0, cin_pad - cin)).to(torch.bfloat16).contiguous()
    got = conv3d_tcgen05(h, layer, True).float()
    torch.cuda.synchronize()
    ref = _reference(x, conv, True).permute(0, 2, 3, 4, 1)
    assert float((got[..., :cout] - ref).abs().max()) <= 8e-3 * float(ref.abs().max()) + 1e-6


@pytest.mark.parametrize("tz", ["1", "2", "4"])
@pytest.mark.parametrize("cin,cin_pad,cout,grid,batch,relu", [
    (24, 32, 24, (8, 16, 16), 2, True), (72, 80, 24, (4, 32, 8), 2, False), (48, 48, 48, (4, 16, 24), 1, True),
    (144, 144, 48, (8, 16, 8), 1, True), (96, 96, 48, (4, 16, 8), 3, False)])
def test_conv_kslice(monkeypatch, tz, cin, cin_pad, cout, grid, batch, relu):
    """The kernel that stages the halo and all 27 taps' weights by slices of 16
    input channels, with 1, 2 and 4 output planes per CTA (the
    LFTS_CONV_KSLICE_TZ override), against torch."""
    import torch
    from langevinfts_b200.learned import conv3d_tcgen05, pack_conv
    monkeypatch.setenv("LFTS_CONV_KSLICE", "1")
    monkeypatch.setenv("LFTS_CONV_KSLICE_TZ", tz)
    torch.manual_seed(cin * 13 + cout + int(tz))
    conv = torch.nn.Conv3d(cin, cout, 3).cuda()
    x = torch.randn(batch, cin, *grid, device="cuda").to(torch.bfloat16).float()
    layer = pack_conv(conv, list(range(cin)), cin_pad)
    h = torch.nn.functional.pad(x.permute(0, 2, 3, 4, 1), (0, cin_pad - cin)).to(torch.bfloat16).contiguous()
    got = conv3d_tcgen05(h, layer, relu).float()
    torch.cuda.synchronize()
    ref = _reference(x, conv, relu).permute(0, 2, 3, 4, 1)
    assert float((got[..., :cout] - ref).abs().max()) <= 8e-3 * float(ref.abs().max()) + 1e-6
    assert float(got[..., cout:].abs().max() if got.shape[-1] > cout else 0) == 0.0


@pytest.mark.parametrize("ws", ["2", "3", "4"])
@pytest.mark.parametrize("cin,cout,k,grid,batch", [
    (32, 32, 3, (16, 16, 16), 2), (48, 96, 3, (16, 16, 16), 1), (80, 32, 3, (6, 16, 16), 3), (32, 16, 1, (8, 8, 8), 1),
    (32, 16, 3, (2, 8, 64), 2), (32, 32, 3, (2, 4, 96), 3), (16, 16, 3, (4, 8, 24), 2),  # row segments of 64, 32, 8
    (16, 32, 3, (4, 6, 12), 2)])  # W % 8 != 0: per-tap gathers
def test_wgrad_ring_depths(monkeypatch, ws, cin, cout, k, grid, batch):
    """lfts_conv3d_wgrad_bf16 with every ring depth (the LFTS_CONV_WGRAD_RING
    override) against torch's FP32 weight gradient of the same BF16 operands,
    over several 2048-position chunks and a ragged last chunk, for x staged as
    row segments of every length and as per-tap gathers."""
    import torch
    import torch.nn.functional as F
    from langevinfts_b200.capi import check, lib
    monkeypatch.setenv("LFTS_CONV_WGRAD_RING", ws)
    torch.manual_seed(cin + cout + k)
    x = torch.randn(batch, *grid, cin, device="cuda").to(torch.bfloat16)
    gy = torch.randn(batch, *grid, cout, device="cuda").to(torch.bfloat16)
    taps = k ** 3
    dw = torch.zeros(taps, cout, cin, device="cuda")
    check(lib().lfts_conv3d_wgrad_bf16(torch.cuda.current_stream().cuda_stream, x.data_ptr(), gy.data_ptr(), dw.data_ptr(),
                                       batch, *grid, cin, cout, taps))
    torch.cuda.synchronize()
    xc = x.float().permute(0, 4, 1, 2, 3)
    xp = F.pad(xc, (k // 2,) * 6, mode="circular") if k > 1 else xc
    # dw[co][ci][kz][ky][kx] = sum_p gy[p][co] x[p + tap - 1][ci]
    ref = torch.nn.grad.conv3d_weight(xp, (cout, cin, k, k, k), gy.float().permute(0, 4, 1, 2, 3))
    ref = ref.permute(2, 3, 4, 0, 1).reshape(taps, cout, cin)
    assert _rel(dw, ref) < 1e-4


@pytest.mark.parametrize("stages", ["64", "100", "256"])
def test_wgrad_stage_counts(monkeypatch, stages):
    """lfts_conv3d_wgrad_bf16 with more stages of 64 positions per CTA (the
    LFTS_CONV_WGRAD_STAGES override), ragged last chunk, against torch."""
    import torch
    import torch.nn.functional as F
    from langevinfts_b200.capi import check, lib
    monkeypatch.setenv("LFTS_CONV_WGRAD_STAGES", stages)
    torch.manual_seed(int(stages))
    cin, cout, grid, batch = 32, 16, (6, 16, 32), 5
    x = torch.randn(batch, *grid, cin, device="cuda").to(torch.bfloat16)
    gy = torch.randn(batch, *grid, cout, device="cuda").to(torch.bfloat16)
    dw = torch.zeros(27, cout, cin, device="cuda")
    check(lib().lfts_conv3d_wgrad_bf16(torch.cuda.current_stream().cuda_stream, x.data_ptr(), gy.data_ptr(), dw.data_ptr(),
                                       batch, *grid, cin, cout, 27))
    torch.cuda.synchronize()
    xp = F.pad(x.float().permute(0, 4, 1, 2, 3), (1,) * 6, mode="circular")
    ref = torch.nn.grad.conv3d_weight(xp, (cout, cin, 3, 3, 3), gy.float().permute(0, 4, 1, 2, 3))
    assert _rel(dw, ref.permute(2, 3, 4, 0, 1).reshape(27, cout, cin)) < 1e-4


@pytest.mark.parametrize("cpad,co", [(32, 24), (48, 48), (16, 1), (144, 144), (256, 200)])
def test_relu_grad_kernel(cpad, co):
    """lfts_relu_grad_bf16 against torch: g = gy * (y > 0) value for value
    (zeros, negative zeros, infinities and NaN in y included; the kernel writes
    +0 where torch's product gives -0) and the bias gradient against a float64
    sum."""
    import torch
    from langevinfts_b200.capi import check, lib
    torch.manual_seed(cpad + co)
    npos = 3 * 17 * 19 + 5
    gy = torch.randn(npos, cpad, device="cuda").to(torch.bfloat16)
    y = torch.randn(npos, cpad, device="cuda").to(torch.bfloat16)
    special = torch.tensor([0.0, -0.0, float("inf"), float("-inf"), float("nan"), 1e-40], device="cuda").to(torch.bfloat16)
    y.view(-1)[:special.numel() * 7:7] = special.repeat(1)
    g = torch.empty_like(gy)
    db = torch.zeros(cpad, device="cuda")
    check(lib().lfts_relu_grad_bf16(torch.cuda.current_stream().cuda_stream, gy.data_ptr(), y.data_ptr(), g.data_ptr(),
                                    db.data_ptr(), npos, cpad, co))
    torch.cuda.synchronize()
    ref = gy * (y > 0)
    assert torch.equal(g.float(), ref.float())
    want = ref[:, :co].double().sum(0)
    assert float((db[:co].double() - want).abs().max()) <= 1e-5 * float(want.abs().max()) + 1e-6
    assert float(db[co:].abs().max() if co < cpad else 0) == 0.0


def test_tcgen05_unet_matches_torch_model():
    import torch
    from langevinfts_b200.learned import TcgenUNet, UNet3D
    torch.manual_seed(3)
    net = UNet3D(cin=2, cout=1, base=24).cuda()
    for p in net.parameters():  # non-zero last layer
        if p.dim() == 1:
            torch.nn.init.normal_(p, 0, 0.05)
    torch.nn.init.normal_(net.out.weight, 0, 0.2)
    x = torch.randn(2, 2, 16, 16, 16, device="cuda")
    with torch.no_grad():
        ref = net(x)
    got = TcgenUNet(net)(x)
    torch.cuda.synchronize()
    rel = float((got - ref).abs().max() / ref.abs().max())
    assert rel < 5e-2, rel  # BF16 activations through 11 layers
    assert np.corrcoef(got.flatten().cpu().numpy(), ref.flatten().cpu().numpy())[0, 1] > 0.999


def _rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("cin,cin_pad,cout,k,grid,batch", [
    (2, 16, 24, 3, (8, 8, 8), 2), (24, 32, 48, 3, (8, 8, 8), 1), (144, 144, 48, 3, (4, 4, 4), 2),
    (96, 96, 96, 3, (4, 6, 5), 1), (24, 32, 1, 1, (8, 8, 8), 2),
    (48, 48, 96, 3, (32, 32, 32), 2),  # 65536 positions: 32 weight-gradient chunks (input gradient: halo kernel)
    (24, 32, 24, 3, (16, 16, 16), 2)])
def test_conv_backward_matches_torch(cin, cin_pad, cout, k, grid, batch):
    """Input gradient (the forward kernel with transposed, mirrored weights)
    and weight gradient (lfts_conv3d_wgrad_bf16) against torch autograd on the
    same BF16-rounded operands."""
    import torch
    import torch.nn.functional as F
    from langevinfts_b200.learned import _ConvFn
    torch.manual_seed(cin + 7 * cout)
    conv = torch.nn.Conv3d(cin, cout, k).cuda()
    with torch.no_grad():
        conv.weight.copy_(conv.weight.to(torch.bfloat16).float())
    relu = cout > 1
    x = torch.randn(batch, cin, *grid, device="cuda").to(torch.bfloat16).float()
    gy = torch.randn(batch, *grid, cout, device="cuda").to(torch.bfloat16).float()
    h = F.pad(x.permute(0, 2, 3, 4, 1), (0, cin_pad - cin)).to(torch.bfloat16).contiguous().requires_grad_(True)
    y = _ConvFn.apply(h, conv.weight, conv.bias, list(range(cin)), cin_pad, relu)
    (y[..., :cout].float() * gy).sum().backward()
    xr = x.clone().requires_grad_(True)
    wr = conv.weight.detach().clone().requires_grad_(True)
    br = conv.bias.detach().clone().requires_grad_(True)
    yr = F.conv3d(F.pad(xr, (k // 2,) * 6, mode="circular") if k > 1 else xr, wr, br)
    yr = F.relu(yr) if relu else yr
    (yr.permute(0, 2, 3, 4, 1) * gy).sum().backward()
    torch.cuda.synchronize()
    assert _rel(h.grad[..., :cin].float(), xr.grad.permute(0, 2, 3, 4, 1)) < 1e-2
    assert float(h.grad[..., cin:].float().abs().max() if cin_pad > cin else 0) == 0.0
    assert _rel(conv.weight.grad, wr.grad) < 1e-2
    assert _rel(conv.bias.grad, br.grad) < 1e-2


def test_tcgen05_unet_gradients_match_torch_model():
    """Gradients of the whole 24-channel network (32^3, batch 2: the weight
    gradients reduce over many position chunks) against the FP32 torch model:
    as close as torch's own BF16 autocast gets, parameter by parameter."""
    import torch
    import torch.nn.functional as F
    from langevinfts_b200.learned import TcgenUNetTrain, UNet3D
    torch.manual_seed(0)
    net = UNet3D(cin=2, cout=1, base=24).cuda()
    torch.nn.init.normal_(net.out.weight, 0, 0.05)
    x = torch.randn(2, 2, 32, 32, 32, device="cuda")
    t = 0.1 * torch.randn(2, 1, 32, 32, 32, device="cuda")

    def grads(fn):
        net.zero_grad()
        F.mse_loss(fn(x), t).backward()
        return {n: p.grad.clone() for n, p in net.named_parameters()}

    def autocast(z):
        with torch.autocast("cuda", dtype=torch.bfloat16):
            return net(z).float()

    g32, gac, gtc = grads(net), grads(autocast), grads(TcgenUNetTrain(net))
    for n in g32:
        cos = float((gtc[n] * g32[n]).sum() / (gtc[n].norm() * g32[n].norm()))
        assert cos > 0.98 and _rel(gtc[n], g32[n]) <= max(2 * _rel(gac[n], g32[n]), 0.03), (n, cos, _rel(gtc[n], g32[n]),
                                                                                          _rel(gac[n], g32[n]))


def test_training_on_the_tensor_cores_lowers_the_loss():
    import torch
    from langevinfts_b200.learned import train
    g = torch.Generator().manual_seed(1)
    X = torch.randn(8, 2, 16, 16, 16, generator=g).numpy()
    Y = X[:, 1:] + 0.5 * np.roll(X[:, :1], 1, axis=-1)  # a learnable residual
    start, hist = train(X, Y, base=8, seconds=120, epochs=40, batch=4, lr=3e-3, tcgen05=True)
    assert start.net is not None
    assert hist[-1][1] < 0.6 * hist[0][1], hist[:: max(1, len(hist) // 6)]


def test_adamw_kernel_matches_torch_adamw():
    """lfts_adamw_f32 (FlatAdamW) against torch.optim.AdamW in FP32 on the same
    parameters and gradients, six steps."""
    import torch
    from langevinfts_b200.learned import FlatAdamW
    torch.manual_seed(9)
    shapes = [(24, 2, 3, 3, 3), (24,), (48, 24, 3, 3, 3), (1, 24, 1, 1, 1)]
    a = [torch.nn.Parameter(torch.randn(s, device="cuda")) for s in shapes]
    b = [torch.nn.Parameter(p.detach().clone()) for p in a]
    ours = FlatAdamW(a, lr=2e-3, weight_decay=1e-2)
    ref = torch.optim.AdamW(b, lr=2e-3, weight_decay=1e-2)
    for _ in range(6):
        for pa, pb in zip(a, b):
            g = torch.randn_like(pa)
            pa.grad, pb.grad = g.clone(), g.clone()
        ours.step()
        ref.step()
    for pa, pb in zip(a, b):
        assert float((pa.detach() - pb.detach()).abs().max()) <= 1e-5 * float(pb.detach().abs().max())


@pytest.mark.parametrize("cin,cin_pad,cout,grid", [(24, 32, 48, (8, 8, 8)), (2, 16, 24, (16, 16, 16))])
def test_conv_gradients_match_cpu_float64(cin, cin_pad, cout, grid):
    """Input, weight and bias gradients of the tensor-core convolution
    (_ConvFn: lfts_conv3d_bf16 with mirrored taps, lfts_conv3d_wgrad_bf16)
    against float64 autograd of torch's CPU periodic conv3d on the same
    BF16-rounded input, weights and output gradient."""
    import torch
    import torch.nn.functional as F
    from langevinfts_b200.learned import _ConvFn
    torch.manual_seed(cin + cout)
    B = 2
    w = (0.2 * torch.randn(cout, cin, 3, 3, 3)).to(torch.bfloat16).float()
    bias = torch.randn(cout)
    x = torch.randn(B, cin, *grid).to(torch.bfloat16).float()
    gy = torch.randn(B, cout, *grid).to(torch.bfloat16).float()
    # reference: float64 on the CPU
    xr = x.double().requires_grad_(True)
    wr = w.double().requires_grad_(True)
    br = bias.double().requires_grad_(True)
    F.conv3d(F.pad(xr, (1,) * 6, mode="circular"), wr, br).backward(gy.double())
    # tensor cores: channels-last BF16 with padded input channels, no ReLU
    xc = torch.nn.functional.pad(x.permute(0, 2, 3, 4, 1), (0, cin_pad - cin)).to(torch.bfloat16).cuda().contiguous()
    xc.requires_grad_(True)
    wc = w.cuda().requires_grad_(True)
    bc = bias.cuda().requires_grad_(True)
    y = _ConvFn.apply(xc, wc, bc, list(range(cin)), cin_pad, False)
    gyc = torch.nn.functional.pad(gy.permute(0, 2, 3, 4, 1), (0, y.shape[-1] - cout)).to(torch.bfloat16).cuda()
    y.backward(gyc)
    torch.cuda.synchronize()
    dx = xc.grad[..., :cin].float().cpu().permute(0, 4, 1, 2, 3).double()
    dw, db = wc.grad.double().cpu(), bc.grad.double().cpu()
    # FP32 accumulation of exact BF16 products: the weight and bias gradients to
    # 1e-5 of their scale; the input gradient is a BF16 output (2^-8 relative)
    assert float((dw - wr.grad).abs().max()) <= 1e-5 * float(wr.grad.abs().max())
    assert float((db - br.grad).abs().max()) <= 1e-5 * float(br.grad.abs().max())
    assert float((dx - xr.grad).abs().max()) <= 8e-3 * float(xr.grad.abs().max())
