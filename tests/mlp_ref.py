"""NumPy reference of the opacity-surrogate network, used as the checker of
the tensor-core kernels: the same layers, with the BF16 roundings the
kernels apply (activations and weights of the 256-wide layers, the
back-propagated dZ), FP32 elsewhere.  `emulate=False` gives the plain
float64 network for finite-difference checks of the formulas."""
import numpy as np

IN, H, OUT = 6, 256, 64
NP = H * IN + H + 3 * H * H + 3 * H + OUT * H + OUT


def bf16(a):
    """round-to-nearest-even to bfloat16, returned as float32"""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_bits(a):
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def unpack(p):
    p = np.asarray(p)
    o = 0
    W0 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b0 = p[o:o + H]; o += H
    W = p[o:o + 3 * H * H].reshape(3, H, H); o += 3 * H * H
    b = p[o:o + 3 * H].reshape(3, H); o += 3 * H
    W4 = p[o:o + OUT * H].reshape(OUT, H); o += OUT * H
    b4 = p[o:o + OUT]
    return W0, b0, W, b, W4, b4


def pack(W0, b0, W, b, W4, b4):
    return np.concatenate([W0.ravel(), b0.ravel(), W.ravel(), b.ravel(), W4.ravel(), b4.ravel()])


def init(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    W0 = rng.normal(0, scale / np.sqrt(IN), (H, IN))
    W = rng.normal(0, scale / np.sqrt(H), (3, H, H))
    W4 = rng.normal(0, scale / np.sqrt(H), (OUT, H))
    b0 = rng.normal(0, 0.1, H)
    b = rng.normal(0, 0.1, (3, H))
    b4 = rng.normal(0, 0.1, OUT)
    return pack(W0, b0, W, b, W4, b4).astype(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, emulate=True):
    dt = np.float32 if emulate else np.float64
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    W0, b0, W, b, W4, b4 = [np.asarray(a, dt) for a in unpack(p)]
    x = np.asarray(x, dt)
    zs, hs = [], []
    z = x @ W0.T + b0
    zs.append(z)
    h = r(silu(z))
    hs.append(h)
    for l in range(3):
        z = (h @ r(W[l]).T).astype(dt) + b[l]
        zs.append(z)
        h = r(silu(z))
        hs.append(h)
    y = (h @ r(W4).T).astype(dt) + b4
    return y, zs, hs


def gradient(p, x, t, w, emulate=True):
    dt = np.float32 if emulate else np.float64
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    W0, b0, W, b, W4, b4 = [np.asarray(a, dt) for a in unpack(p)]
    x = np.asarray(x, dt)
    n = x.shape[0]
    y, zs, hs = forward(p, x, emulate)
    d = y - np.asarray(t, dt)
    w = np.asarray(w, dt)
    loss = float((w * d * d).sum() / n)
    dy = 2 * w * d / n
    gW4 = dy.T @ hs[3]
    gb4 = dy.sum(0)
    dz = r((dy @ W4) * dsilu(zs[3]))
    gW, gb = np.zeros_like(W), np.zeros_like(b)
    for l in (2, 1, 0):
        gW[l] = dz.T @ hs[l]
        gb[l] = dz.sum(0)
        dz = r((dz @ r(W[l])) * dsilu(zs[l]))
    gW0 = dz.T @ x
    gb0 = dz.sum(0)
    return pack(gW0, gb0, gW, gb, gW4, gb4), loss
