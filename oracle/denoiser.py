"""Oracle (test infrastructure only) of the learned moment denoiser: the
network of rhybrid_b200/csrc/k_denoise.cuh restated in numpy, forward and
backward, for checking the GPU kernels. With bf16=True it rounds what the GPU
stores in BF16 (the network input, the weights, the hidden activations and the
output gradients) the same way (round to nearest even) and accumulates in
float64; with bf16=False it is the exact float64 network, whose backward is
checked here against finite differences.

Layout: moments x[nz, ny, nx, 4] (normalized rho, Jx, Jy, Jz); parameters as
the C ABI's RHGPU_DN_PARAMS vector: per layer W[27][16 cin][16 cout] then
b[16], tap t = (dx+1) + 3 (dy+1) + 9 (dz+1)."""
import numpy as np

C = 16
TAPS = 27
LEAK = 0.125   # leaky ReLU slope below zero
LAYER = TAPS * C * C + C
PARAMS = 3 * LAYER


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def unpack(p):
    p = np.asarray(p)
    Ws, bs = [], []
    for l in range(3):
        base = l * LAYER
        Ws.append(p[base:base + TAPS * C * C].reshape(TAPS, C, C))
        bs.append(p[base + TAPS * C * C:base + LAYER])
    return Ws, bs


def shift(a, d, periodic):
    """out[z, y, x] = a[z + dz, y + dy, x + dx] (zero outside a non-periodic box)."""
    out = a
    for axis, (dd, per) in zip((2, 1, 0), zip(d, periodic)):
        if dd == 0:
            continue
        if per:
            out = np.roll(out, -dd, axis=axis)
        else:
            r = np.zeros_like(out)
            n = out.shape[axis]
            src = [slice(None)] * out.ndim
            dst = [slice(None)] * out.ndim
            if dd > 0:
                src[axis], dst[axis] = slice(dd, n), slice(0, n - dd)
            else:
                src[axis], dst[axis] = slice(0, n + dd), slice(-dd, n)
            r[tuple(dst)] = out[tuple(src)]
            out = r
    return out


def taps():
    for t in range(TAPS):
        yield t, (t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1)


def conv(a, W, periodic, transposed=False):
    """sum over taps of shift(a, +-d) @ W[t] (W^T when transposed)."""
    out = np.zeros(a.shape[:3] + (C,), dtype=np.float64)
    for t, d in taps():
        s = shift(a, tuple(-x for x in d) if transposed else d, periodic).astype(np.float64)
        out += s @ (W[t].T if transposed else W[t]).astype(np.float64)
    return out


def forward(p, x, periodic, bf16_mode=True):
    """Returns (output [.., 4] float64, activations list) of the network."""
    Ws, bs = unpack(p)
    rnd = bf16 if bf16_mode else (lambda v: np.asarray(v, dtype=np.float64))
    Wr = [rnd(W) for W in Ws]
    x = np.asarray(x, dtype=np.float32 if bf16_mode else np.float64)
    a0 = np.zeros(x.shape[:3] + (C,), dtype=np.float64)
    a0[..., :4] = rnd(x)
    lrelu = lambda h: np.where(h > 0, h, LEAK * h)   # noqa: E731
    h1 = lrelu(conv(a0, Wr[0], periodic) + bs[0])
    a1 = rnd(h1.astype(np.float32)) if bf16_mode else h1
    h2 = lrelu(conv(a1, Wr[1], periodic) + bs[1])
    a2 = rnd(h2.astype(np.float32)) if bf16_mode else h2
    y = conv(a2, Wr[2], periodic) + bs[2]
    out = y[..., :4] + x.astype(np.float64)
    return out, (a0, a1, a2, Wr)


def loss_grad(p, x, target, periodic, bf16_mode=True):
    """Mean squared error over the 4 channels and its gradient (PARAMS,)."""
    out, (a0, a1, a2, Wr) = forward(p, x, periodic, bf16_mode)
    n = out.shape[0] * out.shape[1] * out.shape[2] * 4
    d = out - np.asarray(target, dtype=np.float64)
    loss = float((d * d).sum() / n)
    rnd = bf16 if bf16_mode else (lambda v: np.asarray(v, dtype=np.float64))
    dY = np.zeros(a0.shape, dtype=np.float64)
    dY[..., :4] = 2.0 * d / n
    if bf16_mode:
        dY = rnd(dY.astype(np.float32))
    g = np.zeros(PARAMS, dtype=np.float64)
    acts = [a0, a1, a2]
    for l in (2, 1, 0):
        gW = np.zeros((TAPS, C, C))
        for t, dd in taps():
            gW[t] = np.einsum("zyxi,zyxo->io", shift(acts[l], dd, periodic), dY)
        base = l * LAYER
        g[base:base + TAPS * C * C] = gW.reshape(-1)
        g[base + TAPS * C * C:base + LAYER] = dY.reshape(-1, C).sum(0)
        if l > 0:
            dX = conv(dY, Wr[l], periodic, transposed=True) * np.where(acts[l] > 0, 1.0, LEAK)
            dY = rnd(dX.astype(np.float32)) if bf16_mode else dX
    # untrainable entries (padding channels) are zero
    for l in range(3):
        base = l * LAYER
        gw = g[base:base + TAPS * C * C].reshape(TAPS, C, C)
        if l == 0:
            gw[:, 4:, :] = 0.0
        if l == 2:
            gw[:, :, 4:] = 0.0
            g[base + TAPS * C * C + 4:base + LAYER] = 0.0
    return loss, g
