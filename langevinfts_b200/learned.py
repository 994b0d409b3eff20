"""Learned saddle-point start for batched L-FTS.

After the Langevin update of the real (exchange) fields w_-, the saddle-point
search over the imaginary (pressure) fields w_+ normally starts from the
previous step's saddle point.  Here a 3-level periodic 3D U-Net predicts the
new saddle point from the new w_-, the previous w_+ and the step's change of
w_- (dw_- = w_- - w_-prev, which drives the shift of the saddle point), and
the search starts there:

    w_+start = w_+prev + s_out * UNet([w_- / s_in, w_+prev / s_out, dw_- / s_d])

The network adds a residual to the warm start; its last layer starts at zero,
so an untrained model reproduces the plain warm start exactly.  The search
itself (Anderson mixing to the same tolerance) is unchanged, so the learned
start can only change how many iterations a step needs, not where it ends.

Pieces:
  UNet3D            3 levels (N, N/2, N/4), 24 base channels, 3^3 kernels with
                    circular padding (the box is periodic), ReLU, average
                    pooling down, nearest upsampling, skip concatenation; the
                    parameter holder, and the torch form (BF16 autocast).
  TcgenUNet         inference with every convolution on this library's
                    tensor-core kernel (lfts_conv3d_bf16: tcgen05 implicit
                    GEMM, BF16 operands, FP32 accumulation in tensor memory).
  TcgenUNetTrain    training form: forward and backward of every convolution
                    on the tensor cores (_ConvFn: input gradient by the forward
                    kernel with mirrored taps, weight gradient by
                    lfts_conv3d_wgrad_bf16).
  generate_pairs    training pairs from the plain solver: inputs (w_-, w_+prev,
                    dw_-) and target w_+ of every replica and step.
  FlatAdamW         AdamW on this library's kernel (lfts_adamw_f32): the
                    parameters live in one flat FP32 buffer, one launch a step.
  train             AdamW on the mean-squared error of the residual; by default
                    every convolution's forward and backward on the tensor
                    cores and the update by FlatAdamW (tcgen05=False: torch's
                    convolutions under BF16 autocast and torch's AdamW, kept as
                    the comparison).
  LearnedStart      the callable BatchedLFTS.step(start=...) uses: keeps a
                    device copy of w_- before each Langevin update
                    (before_update), reads w_aux on the device (zero copy),
                    writes the predicted w_+ in place on the engine's stream;
                    inference on the tensor cores by default.

Pooling, upsampling and concatenation are torch tensor operations between the
convolutions.  Grids must have extents divisible by 4.
"""
import time

import numpy as np
import torch
import torch.nn as nn
import torch.nn.functional as F


class _DeviceArray:
    """Zero-copy view of device memory for torch.as_tensor (__cuda_array_interface__)."""

    def __init__(self, ptr, shape, typestr="<f8"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _conv(cin, cout, k=3):
    return nn.Conv3d(cin, cout, k, padding=k // 2, padding_mode="circular")


def _block(cin, cout):
    return nn.Sequential(_conv(cin, cout), nn.ReLU(inplace=True), _conv(cout, cout), nn.ReLU(inplace=True))


class UNet3D(nn.Module):
    """3-level periodic 3D U-Net (base channels b: b, 2b, 4b by level)."""

    def __init__(self, cin=2, cout=1, base=24):
        super().__init__()
        b = base
        self.e1, self.e2, self.e3 = _block(cin, b), _block(b, 2 * b), _block(2 * b, 4 * b)
        self.d2, self.d1 = _block(6 * b, 2 * b), _block(3 * b, b)
        self.out = nn.Conv3d(b, cout, 1)
        nn.init.zeros_(self.out.weight)
        nn.init.zeros_(self.out.bias)

    def forward(self, x):
        x1 = self.e1(x)
        x2 = self.e2(F.avg_pool3d(x1, 2))
        x3 = self.e3(F.avg_pool3d(x2, 2))
        y2 = self.d2(torch.cat([F.interpolate(x3, scale_factor=2, mode="nearest"), x2], 1))
        y1 = self.d1(torch.cat([F.interpolate(y2, scale_factor=2, mode="nearest"), x1], 1))
        return self.out(y1)


def generate_pairs(sim, nsteps):
    """Run nsteps plain Langevin steps of a started BatchedLFTS and collect, per
    replica and step that met the tolerance, the network inputs (w_- after the
    update, w_+ before the search, and the update's change of w_-) and the
    target (w_+ at the saddle point).  Returns float32 arrays X [n, 3, nx, ny,
    nz], Y [n, 1, nx, ny, nz] and the saddle iterations of the steps."""
    shape = list(sim.cb.get_nx())
    ri, ii = sim.mpt.aux_fields_real_idx, sim.mpt.aux_fields_imag_idx
    if len(ri) != 1 or len(ii) != 1:
        raise ValueError("the learned start handles one real and one imaginary auxiliary field")
    X, Y, iters = [], [], []
    w_prev = sim.fields()
    for _ in range(nsteps):
        st = sim.step()
        w = sim.fields()
        for r in range(sim.R):
            if st["failed"][r]:
                continue
            X.append(np.stack([w[r, ri[0]], w_prev[r, ii[0]], w[r, ri[0]] - w_prev[r, ri[0]]]).reshape([3] + shape)
                     .astype(np.float32))
            Y.append(w[r, ii[0]].reshape([1] + shape).astype(np.float32))
        iters += list(st["iterations"])
        w_prev = w
    return np.array(X), np.array(Y), iters


def _pad16(c):
    return (c + 15) // 16 * 16


def pack_conv(conv, in_map, cin_pad):
    """Weights of an nn.Conv3d (kernel 3 or 1) in the layout lfts_conv3d_bf16
    reads: [taps][cin_pad/8][cout_pad][8] BF16, tap = 9 kz + 3 ky + kx; real
    input channel i sits at padded position in_map[i].  Returns (packed
    weights, FP32 bias [cout_pad], cout_pad, taps)."""
    w = conv.weight.detach().float().cpu()
    co, ci, k = w.shape[0], w.shape[1], w.shape[2]
    taps, cout_pad = k ** 3, _pad16(co)
    full = torch.zeros(taps, cout_pad, cin_pad)
    full[:, :co, torch.as_tensor(in_map)] = w.permute(2, 3, 4, 0, 1).reshape(taps, co, ci)
    packed = full.reshape(taps, cout_pad, cin_pad // 8, 8).permute(0, 2, 1, 3).contiguous()
    bias = torch.zeros(cout_pad)
    if conv.bias is not None:
        bias[:co] = conv.bias.detach().float().cpu()
    return packed.to(torch.bfloat16).cuda(), bias.cuda(), cout_pad, taps


def conv3d_tcgen05(x, layer, relu):
    """Periodic convolution of a channels-last BF16 tensor [B, D, H, W, cin_pad]
    with a packed layer, by lfts_conv3d_bf16 on torch's current stream."""
    from langevinfts_b200.capi import check, lib
    wpk, bias, cout_pad, taps = layer
    B, D, H, W, cin = x.shape
    out = torch.empty([B, D, H, W, cout_pad], dtype=torch.bfloat16, device=x.device)
    check(lib().lfts_conv3d_bf16(torch.cuda.current_stream().cuda_stream, x.data_ptr(), wpk.data_ptr(), bias.data_ptr(),
                                 out.data_ptr(), B, D, H, W, cin, cout_pad, taps, 1 if relu else 0))
    return out


def _full_weights(w, in_map, cin_pad, cout_pad):
    """[taps, cout_pad, cin_pad] FP32 from a torch conv weight [co, ci, k, k, k]."""
    co, ci, k = w.shape[0], w.shape[1], w.shape[2]
    full = torch.zeros(k ** 3, cout_pad, cin_pad, device=w.device)
    full[:, :co, torch.as_tensor(in_map, device=w.device)] = w.detach().float().permute(2, 3, 4, 0, 1).reshape(k ** 3, co, ci)
    return full


def _pack_full(full):
    taps, cout_pad, cin_pad = full.shape
    return full.reshape(taps, cout_pad, cin_pad // 8, 8).permute(0, 2, 1, 3).contiguous().to(torch.bfloat16)


class _ConvFn(torch.autograd.Function):
    """Periodic conv (+ ReLU) on the tensor cores with its backward: the input
    gradient by lfts_conv3d_bf16 with transposed, tap-mirrored weights, the
    weight gradient by lfts_conv3d_wgrad_bf16."""

    @staticmethod
    def forward(ctx, x, w, b, in_map, cin_pad, relu):
        from langevinfts_b200.capi import check, lib
        co, k = w.shape[0], w.shape[2]
        cout_pad, taps = _pad16(co), k ** 3
        full = _full_weights(w, in_map, cin_pad, cout_pad)
        bias = torch.zeros(cout_pad, device=w.device)
        bias[:co] = b.detach().float()
        y = conv3d_tcgen05(x, (_pack_full(full), bias, cout_pad, taps), relu)
        ctx.save_for_backward(x, y, full)
        ctx.meta = (co, w.shape[1], k, in_map, cin_pad, cout_pad, taps, relu)
        return y

    @staticmethod
    def backward(ctx, gy):
        from langevinfts_b200.capi import check, lib
        x, y, full = ctx.saved_tensors
        co, ci, k, in_map, cin_pad, cout_pad, taps, relu = ctx.meta
        gy = gy.to(torch.bfloat16).contiguous()
        if relu:
            # ReLU mask and bias gradient in one pass (lfts_relu_grad_bf16)
            g = torch.empty_like(y)
            dbp = torch.zeros(cout_pad, device=gy.device)
            check(lib().lfts_relu_grad_bf16(torch.cuda.current_stream().cuda_stream, gy.data_ptr(), y.data_ptr(), g.data_ptr(),
                                            dbp.data_ptr(), y.numel() // cout_pad, cout_pad, co))
            db = dbp[:co]
        else:
            g = gy
            db = g[..., :co].float().sum((0, 1, 2, 3))
        # input gradient: the same convolution of g, weights transposed, taps mirrored
        back = full.flip(0).transpose(1, 2).contiguous()  # [taps, cin_pad, cout_pad]
        dx = conv3d_tcgen05(g, (_pack_full(back), torch.zeros(cin_pad, device=g.device), cin_pad, taps), False)
        dwp = torch.zeros(taps, cout_pad, cin_pad, device=g.device)
        B, D, H, W, _ = x.shape
        check(lib().lfts_conv3d_wgrad_bf16(torch.cuda.current_stream().cuda_stream, x.data_ptr(), g.data_ptr(), dwp.data_ptr(),
                                           B, D, H, W, cin_pad, cout_pad, taps))
        dw = dwp[:, :co, torch.as_tensor(in_map, device=g.device)].reshape(k, k, k, co, ci).permute(3, 4, 0, 1, 2).contiguous()
        return dx, dw, db, None, None, None


class TcgenUNetTrain(torch.nn.Module):
    """Training form of a UNet3D with every convolution, forward and backward,
    on the tensor cores (_ConvFn); the UNet3D's parameters receive the
    gradients, so torch's AdamW steps them and TcgenUNet / the torch model
    both run the result."""

    def __init__(self, net):
        super().__init__()
        self.net = net
        b = net.e1[0].out_channels
        self.pb, self.p2, self.p4 = _pad16(b), _pad16(2 * b), _pad16(4 * b)
        self.cin = net.e1[0].in_channels
        self.cin_pad = _pad16(self.cin)
        # channel maps as device tensors, made once (no host upload inside a step, so a step can be graph-captured)
        dev = net.e1[0].weight.device
        r = lambda n: torch.arange(n, device=dev)
        cat = lambda a, off, n: torch.cat([a, torch.arange(off, off + n, device=dev)])
        pb, p2, p4 = self.pb, self.p2, self.p4
        self.maps = {"e1": (r(self.cin), self.cin_pad, r(b), pb), "e2": (r(b), pb, r(2 * b), p2),
                     "e3": (r(2 * b), p2, r(4 * b), p4),
                     "d2": (cat(r(4 * b), p4, 2 * b), p4 + p2, r(2 * b), p2),
                     "d1": (cat(r(2 * b), p2, b), p2 + pb, r(b), pb)}
        self.out_map = r(net.out.in_channels)

    def _block(self, h, name):
        blk = getattr(self.net, name)
        m0, c0, m1, c1 = self.maps[name]
        h = _ConvFn.apply(h, blk[0].weight, blk[0].bias, m0, c0, True)
        return _ConvFn.apply(h, blk[2].weight, blk[2].bias, m1, c1, True)

    @staticmethod
    def _pool(x):
        B, D, H, W, C = x.shape
        return x.float().reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean((2, 4, 6)).to(torch.bfloat16).contiguous()

    @staticmethod
    def _up(x):
        return x.repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3).contiguous()

    def forward(self, x):
        h = x.permute(0, 2, 3, 4, 1).to(torch.bfloat16)
        h = torch.nn.functional.pad(h, (0, self.cin_pad - h.shape[-1])).contiguous()
        x1 = self._block(h, "e1")
        x2 = self._block(self._pool(x1), "e2")
        x3 = self._block(self._pool(x2), "e3")
        y2 = self._block(torch.cat([self._up(x3), x2], -1).contiguous(), "d2")
        y1 = self._block(torch.cat([self._up(y2), x1], -1).contiguous(), "d1")
        o = _ConvFn.apply(y1, self.net.out.weight, self.net.out.bias, self.out_map, self.pb,
                          False)[..., :self.net.out.out_channels]
        return o.permute(0, 4, 1, 2, 3).float()


class TcgenUNet:
    """Inference of a trained UNet3D with every convolution on the tensor cores
    (lfts_conv3d_bf16: tcgen05 implicit GEMM, BF16 operands, FP32 accumulate);
    activations channels-last BF16 with channels padded to multiples of 16,
    pooling / upsampling / concatenation as torch glue."""

    def __init__(self, net):
        b = net.e1[0].out_channels
        pb, p2, p4 = _pad16(b), _pad16(2 * b), _pad16(4 * b)
        cin = net.e1[0].in_channels
        rng = lambda n: list(range(n))
        self.cin_pad = _pad16(cin)
        self.e1 = (pack_conv(net.e1[0], rng(cin), self.cin_pad), pack_conv(net.e1[2], rng(b), pb))
        self.e2 = (pack_conv(net.e2[0], rng(b), pb), pack_conv(net.e2[2], rng(2 * b), p2))
        self.e3 = (pack_conv(net.e3[0], rng(2 * b), p2), pack_conv(net.e3[2], rng(4 * b), p4))
        # concatenations: upsampled part first, then the skip (each padded)
        self.d2 = (pack_conv(net.d2[0], rng(4 * b) + [p4 + i for i in range(2 * b)], p4 + p2),
                   pack_conv(net.d2[2], rng(2 * b), p2))
        self.d1 = (pack_conv(net.d1[0], rng(2 * b) + [p2 + i for i in range(b)], p2 + pb), pack_conv(net.d1[2], rng(b), pb))
        self.out = pack_conv(net.out, rng(b), pb)
        self.cout = net.out.out_channels

    @staticmethod
    def _pool(x):
        B, D, H, W, C = x.shape
        return x.float().reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean((2, 4, 6)).to(torch.bfloat16).contiguous()

    @staticmethod
    def _up(x):
        return x.repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3).contiguous()

    def _block(self, x, pair):
        return conv3d_tcgen05(conv3d_tcgen05(x, pair[0], True), pair[1], True)

    @torch.no_grad()
    def __call__(self, x):
        """x: [B, cin, D, H, W] float -> [B, cout, D, H, W] float32."""
        h = x.permute(0, 2, 3, 4, 1).to(torch.bfloat16)
        h = torch.nn.functional.pad(h, (0, self.cin_pad - h.shape[-1])).contiguous()
        x1 = self._block(h, self.e1)
        x2 = self._block(self._pool(x1), self.e2)
        x3 = self._block(self._pool(x2), self.e3)
        y2 = self._block(torch.cat([self._up(x3), x2], -1).contiguous(), self.d2)
        y1 = self._block(torch.cat([self._up(y2), x1], -1).contiguous(), self.d1)
        o = conv3d_tcgen05(y1, self.out, False)[..., :self.cout]
        return o.permute(0, 4, 1, 2, 3).float().contiguous()


class FlatAdamW:
    """AdamW whose update runs on this library's kernel (lfts_adamw_f32).  The
    parameters are moved into one flat FP32 buffer (each parameter becomes a
    view of it), the gradients are gathered into a second one, and one launch
    updates everything; the moments m and v live beside them."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=1e-2):
        self.params = [p for p in params if p.requires_grad]
        n = sum(p.numel() for p in self.params)
        dev = self.params[0].device
        self.flat = torch.empty(n, dtype=torch.float32, device=dev)
        off = 0
        for p in self.params:
            k = p.numel()
            self.flat[off:off + k].copy_(p.detach().reshape(-1))
            p.data = self.flat[off:off + k].view_as(p)
            off += k
        self.grad = torch.zeros_like(self.flat)
        self.m = torch.zeros_like(self.flat)
        self.v = torch.zeros_like(self.flat)
        self.lr, self.betas, self.eps, self.weight_decay, self.t = lr, betas, eps, weight_decay, 0

    def zero_grad(self, set_to_none=True):
        for p in self.params:
            p.grad = None

    def step(self):
        from langevinfts_b200.capi import check, lib
        torch.cat([(p.grad if p.grad is not None else torch.zeros_like(p)).reshape(-1) for p in self.params], out=self.grad)
        self.t += 1
        check(lib().lfts_adamw_f32(torch.cuda.current_stream().cuda_stream, self.flat.data_ptr(), self.grad.data_ptr(),
                                   self.m.data_ptr(), self.v.data_ptr(), self.flat.numel(), self.lr, self.betas[0],
                                   self.betas[1], self.eps, self.weight_decay, self.t))


class LearnedStart:
    """Callable for BatchedLFTS.step(start=...): predicts the imaginary field
    of every replica from the fields on the device and writes it in place.
    tcgen05=True (default): every convolution on this library's tensor-core
    kernel; False: torch's convolutions under BF16 autocast."""

    def __init__(self, model, s_in, s_out, s_d=None, batch=8, tcgen05=True):
        self.model, self.s_in, self.s_out, self.batch = model.eval(), float(s_in), float(s_out), batch
        # s_d: scale of the third input channel, the update's change of w_- (None: a two-channel network)
        self.s_d = None if s_d is None else float(s_d)
        self._wm_prev = None
        # tcgen05=True: the convolutions run on this library's tensor-core kernel
        self.net = TcgenUNet(self.model) if tcgen05 else None

    @torch.no_grad()
    def before_update(self, sim):
        """Device copy of every replica's w_- before the Langevin update, on the
        engine's stream (BatchedLFTS.step calls it when the start has it)."""
        if self.s_d is None:
            return
        ri = sim.mpt.aux_fields_real_idx[0]
        with torch.cuda.stream(torch.cuda.ExternalStream(sim.engine.stream_ptr())):
            w = torch.as_tensor(_DeviceArray(sim.engine.w_aux_ptr(), (sim.R, sim.S, sim.M)), device="cuda")
            self._wm_prev = w[:, ri].clone()

    @torch.no_grad()
    def __call__(self, sim):
        shape = list(sim.cb.get_nx())
        R, S, M = sim.R, sim.S, sim.M
        ri, ii = sim.mpt.aux_fields_real_idx[0], sim.mpt.aux_fields_imag_idx[0]
        if self.s_d is not None and (self._wm_prev is None or self._wm_prev.shape != (R, M)):
            raise RuntimeError("LearnedStart: no copy of w_- from before this step's update (before_update)")
        stream = torch.cuda.ExternalStream(sim.engine.stream_ptr())
        with torch.cuda.stream(stream):
            w = torch.as_tensor(_DeviceArray(sim.engine.w_aux_ptr(), (R, S, M)), device="cuda")
            for r0 in range(0, R, self.batch):
                wr = w[r0:r0 + self.batch]
                ch = [wr[:, ri] / self.s_in, wr[:, ii] / self.s_out]
                if self.s_d is not None:
                    ch.append((wr[:, ri] - self._wm_prev[r0:r0 + self.batch]) / self.s_d)
                x = torch.stack(ch, 1).float().reshape([-1, len(ch)] + shape)
                if self.net is not None:
                    d = self.net(x)
                else:
                    with torch.autocast("cuda", dtype=torch.bfloat16):
                        d = self.model(x).float()
                d = d.reshape(-1, M).double() * self.s_out
                d -= d.mean(1, keepdim=True)  # the pressure field keeps zero mean
                wr[:, ii] += d


def ablation(sim, starts, nsteps):
    """Run the same nsteps Langevin steps of a started BatchedLFTS once per entry
    of starts (None: the plain warm start; else a LearnedStart): each run
    begins from the fields, previous noise and PCG64 states the simulation has
    now, so every run sees the same noise.  Returns, per entry, a dict of the
    mean saddle iterations, the failed steps, the iterations per step and the
    wall time; the simulation is left at the end of the last run."""
    import torch
    w0, xi0 = sim.fields(), sim.engine.get_noise_prev()
    rng0 = [g.bit_generator.state for g in sim.rngs]
    step0 = sim.langevin_step
    out = []
    for st in starts:
        sim.engine.set_fields(w0)
        sim.engine.find_saddle_point()  # concentrations at w0, a saddle point already
        sim.engine.set_noise_prev(xi0)
        for g, s0 in zip(sim.rngs, rng0):
            g.bit_generator.state = s0
        sim.langevin_step = step0
        iters, fails = [], 0
        torch.cuda.synchronize()
        t = time.time()
        for _ in range(nsteps):
            r = sim.step(start=st) if st is not None else sim.step()
            iters.append(list(r["iterations"]))
            fails += int(sum(r["failed"]))
        torch.cuda.synchronize()
        out.append({"mean_iterations": float(np.mean(iters)), "failed": fails, "iterations": iters,
                    "seconds": time.time() - t})
    return out


def train(X, Y, base=24, seconds=60.0, epochs=1000, batch=4, lr=1e-3, weight_decay=1e-4, seed=0, log=None, tcgen05=True,
          schedule="cosine", graph=True):
    """AdamW on MSE of the scaled residual target (Y - w_+prev) / s_out until
    `seconds` or `epochs` run out.  X holds 2 input channels (w_-, w_+prev) or
    3 (and dw_-), each scaled by its standard deviation.  schedule "cosine":
    the learning rate falls from lr to 0 over the time budget (half a cosine
    in elapsed time); "constant": lr throughout.  graph (tensor-core path): the
    forward and backward of a batch are captured once as a CUDA graph and
    replayed on static batch buffers (full batches only); the AdamW step runs
    after each replay.  tcgen05=True (default): every convolution's
    forward and backward on this library's tensor-core kernels and the update
    by FlatAdamW (lfts_adamw_f32); False: BF16 autocast over torch's
    convolutions and torch's AdamW.  Returns (LearnedStart, history of (epoch,
    mean loss))."""
    torch.manual_seed(seed)
    scales = [float(np.std(X[:, c])) or 1.0 for c in range(X.shape[1])]
    s_in, s_out = scales[0], scales[1]
    s_d = scales[2] if X.shape[1] > 2 else None
    xin = torch.from_numpy(np.concatenate([X[:, c:c + 1] / scales[c] for c in range(X.shape[1])], 1)).cuda()
    tgt = torch.from_numpy((Y - X[:, 1:2]) / s_out).cuda()
    model = UNet3D(cin=X.shape[1], cout=1, base=base).cuda()
    fwd = TcgenUNetTrain(model) if tcgen05 else None
    if tcgen05:
        opt = FlatAdamW(model.parameters(), lr=lr, weight_decay=weight_decay)
    else:
        opt = torch.optim.AdamW(model.parameters(), lr=lr, weight_decay=weight_decay)
    if schedule not in ("cosine", "constant"):
        raise ValueError('schedule must be "cosine" or "constant"')

    def set_lr(v):
        if tcgen05:
            opt.lr = v
        else:
            for g in opt.param_groups:
                g["lr"] = v
    n = xin.shape[0]
    step_graph = None
    if tcgen05 and graph and n >= batch:
        xs, ts = xin[:batch].clone(), tgt[:batch].clone()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):  # warm-up outside the capture (allocations, kernel attributes)
            for _ in range(2):
                model.zero_grad(set_to_none=True)
                F.mse_loss(fwd(xs), ts).backward()
        torch.cuda.current_stream().wait_stream(side)
        model.zero_grad(set_to_none=True)
        step_graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(step_graph):
            static_loss = F.mse_loss(fwd(xs), ts)
            static_loss.backward()
    hist, t0, out_of_time = [], time.time(), False
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda")
        tot, seen = torch.zeros((), device="cuda"), 0  # summed on the device: no synchronisation per batch
        for k in range(0, n, batch):
            elapsed = time.time() - t0
            if elapsed > seconds:
                out_of_time = True
                break
            if schedule == "cosine":
                set_lr(lr * 0.5 * (1.0 + np.cos(np.pi * elapsed / seconds)))
            idx = perm[k:k + batch]
            if step_graph is not None:
                if len(idx) < batch:
                    break  # full batches only
                torch.index_select(xin, 0, idx, out=xs)
                torch.index_select(tgt, 0, idx, out=ts)
                step_graph.replay()  # gradients into the parameters' captured .grad tensors
                opt.step()
                loss = static_loss
            else:
                if fwd is not None:
                    loss = F.mse_loss(fwd(xin[idx]), tgt[idx])
                else:
                    with torch.autocast("cuda", dtype=torch.bfloat16):
                        loss = F.mse_loss(model(xin[idx]).float(), tgt[idx])
                opt.zero_grad(set_to_none=True)
                loss.backward()
                opt.step()
            tot += loss.detach() * len(idx)
            seen += len(idx)
        if seen:
            hist.append((ep, float(tot) / seen))
            if log:
                log(f"epoch {ep} loss {hist[-1][1]:.4e}")
        if out_of_time:
            break
    return LearnedStart(model, s_in, s_out, s_d, tcgen05=tcgen05), hist
