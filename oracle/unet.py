"""unet.py -- numpy restatement of the learned p' preconditioner's U-Net
(mach2d_b200/csrc/m2d_unet.cu): forward pass, backward pass and the p'
system <-> image adapters.  TEST INFRASTRUCTURE ONLY: the tests use it as the
checker of the CUDA kernels; nothing in the library calls it.

The network has no counterpart in the reference, so this file is its
specification.  Arithmetic is float64; with `bf16=True` the values are
rounded to BF16 exactly where the device rounds them (input planes,
weights, activations after GELU, pooled means, dZ), so that the device
result differs from this one only by FP32 accumulation order.  With
`bf16=False` the backward pass is the exact gradient of the forward pass,
which the CPU tests check by finite differences.
"""
import numpy as np

# (cin, cout, level) of the 14 convolutions in network order
LAYERS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 128, 3),
          (128, 128, 3), (192, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]
K = 0.7978845608028654
C3 = 0.044715


def param_count():
    return sum(co * 9 * ci + co for ci, co, _ in LAYERS) + 17


def split(p):
    """[(W [cout, 9, cin], b [cout]) per layer], wh [16], bh."""
    out, off = [], 0
    for ci, co, _ in LAYERS:
        w = p[off:off + co * 9 * ci].reshape(co, 9, ci)
        off += co * 9 * ci
        out.append((w, p[off:off + co]))
        off += co
    return out, p[off:off + 16], p[off + 16]


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def _id(x):
    return np.asarray(x, dtype=np.float64)


def conv3x3(x, w):
    """'same' 3x3 convolution, zero padding; x [n, H, W, cin], w [cout, 9, cin]."""
    n, H, W, _ = x.shape
    xp = np.zeros((n, H + 2, W + 2, x.shape[3]))
    xp[:, 1:-1, 1:-1] = x
    y = np.zeros((n, H, W, w.shape[0]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        y += np.einsum("nhwc,oc->nhwo", xp[:, dy:dy + H, dx:dx + W], w[:, t, :], optimize=True)
    return y


def conv3x3_wgrad(x, dz):
    """dW[o, t, c] = sum_p dz[p, o] x[p + offset(t), c]."""
    n, H, W, _ = x.shape
    xp = np.zeros((n, H + 2, W + 2, x.shape[3]))
    xp[:, 1:-1, 1:-1] = x
    return np.stack([np.einsum("nhwo,nhwc->oc", dz, xp[:, t // 3:t // 3 + H, t % 3:t % 3 + W], optimize=True)
                     for t in range(9)], axis=1)


def conv3x3_dgrad(dz, w):
    """Adjoint of conv3x3 in its input: the transposed kernel with the taps reversed."""
    wt = np.transpose(w[:, ::-1, :], (2, 1, 0))
    return conv3x3(dz, wt)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K * (x + C3 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K * (x + C3 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K * (1.0 + 3.0 * C3 * x * x)


def pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])


def pool_bwd(dy):
    return 0.25 * np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2)


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_bwd(dy):
    return dy[:, 0::2, 0::2] + dy[:, 0::2, 1::2] + dy[:, 1::2, 0::2] + dy[:, 1::2, 1::2]


def forward(p, feat, bf16_rounding=True):
    """feat [n, 11, H, W] -> out [n, H, W] and the cache for backward."""
    r = bf16 if bf16_rounding else _id
    layers, wh, bh = split(np.asarray(p, dtype=np.float64))
    n, _, H, W = feat.shape
    x0 = np.zeros((n, H, W, 16))
    x0[..., :11] = np.transpose(feat, (0, 2, 3, 1))
    x0 = r(x0)
    cache = {"x": [None] * 14, "z": [None] * 14}

    def layer(k, x):
        w, b = layers[k]
        z = conv3x3(x, r(w)) + b
        cache["x"][k], cache["z"][k] = x, z
        return r(gelu(z))

    s, h = [], x0
    for lv in range(3):
        h = layer(2 * lv + 1, layer(2 * lv, h))
        s.append(h)
        h = r(pool(h))
    h = layer(7, layer(6, h))
    for lv in (2, 1, 0):
        d = np.concatenate([up(h), s[lv]], axis=3)
        k = 8 + 2 * (2 - lv)
        h = layer(k + 1, layer(k, d))
    cache["U0"] = h
    out = h @ wh + bh
    return out, cache


def backward(p, cache, dout, bf16_rounding=True):
    """Gradient of sum(dout * out) with respect to the parameters."""
    r = bf16 if bf16_rounding else _id
    layers, wh, _ = split(np.asarray(p, dtype=np.float64))
    grads = [None] * 14

    def back(k, da, need_dx=True):
        w, _ = layers[k]
        g = da * gelu_grad(cache["z"][k])
        dz = r(g)
        grads[k] = (conv3x3_wgrad(cache["x"][k], dz), g.sum(axis=(0, 1, 2)))
        return conv3x3_dgrad(dz, r(w)) if need_dx else None

    U0 = cache["U0"]
    dwh = np.einsum("nhw,nhwc->c", dout, U0)
    dbh = dout.sum()
    dh = dout[..., None] * wh
    upch = {0: 32, 1: 64, 2: 128}
    dD = {}
    for lv in (0, 1, 2):
        k = 8 + 2 * (2 - lv)
        dD[lv] = back(k, back(k + 1, dh))
        dh = up_bwd(dD[lv][..., :upch[lv]])
    dh = back(6, back(7, dh))
    for lv in (2, 1, 0):
        dskip = dD[lv][..., upch[lv]:] + pool_bwd(dh)
        dh = back(2 * lv, back(2 * lv + 1, dskip), need_dx=lv > 0)
    out = []
    for k in range(14):
        out.append(grads[k][0].reshape(-1))
        out.append(grads[k][1])
    out.append(dwh)
    out.append([dbh])
    return np.concatenate(out)


def loss_grad(p, feat, target, mask, scale, bf16_rounding=True):
    out, cache = forward(p, feat, bf16_rounding)
    d = (out - target) * mask
    loss = scale * np.sum(d * d)
    return loss, backward(p, cache, 2.0 * scale * d, bf16_rounding), out


def init_params(seed):
    """He-normal convolution weights, zero biases, small head."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co, _ in LAYERS:
        out.append(rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)))
        out.append(np.zeros(co))
    out.append(rng.standard_normal(16) * 0.25)
    out.append([0.0])
    return np.concatenate(out).astype(np.float32)


# ------------------------------------------------------------ p' adapters
def features(nx, ny, H, W, a5, r, Jp):
    """11 planes [11, H, W] and (sigma, mean log Jp, std log Jp)."""
    A = a5.reshape(5, ny, nx)[:, 1:-1, 1:-1]
    rr = r.reshape(ny, nx)[1:-1, 1:-1]
    lj = np.log(Jp.reshape(ny, nx)[1:-1, 1:-1])
    ap = A[2]
    rh = rr / ap
    sig = np.sqrt(np.mean(rh * rh))
    sig = sig if sig > 0 else 1.0
    mean = lj.mean()
    var = np.mean(lj * lj) - mean * mean
    std = np.sqrt(var) if var > 1e-24 else 1.0
    f = np.zeros((11, H, W))
    h, w = ny - 2, nx - 2
    f[0, :h, :w] = rh / sig
    f[2, :h, :w] = A[0] / ap
    f[4, :h, :w] = A[1] / ap
    f[5, :h, :w] = 1.0
    f[6, :h, :w] = A[3] / ap
    f[8, :h, :w] = A[4] / ap
    f[10, :h, :w] = (lj - mean) / std
    return f, (sig, mean, std)


def residual5(nx, ny, a5, b, x):
    """b - A x on every cell; neighbours outside the grid contribute nothing."""
    A = a5.reshape(5, ny, nx)
    X = x.reshape(ny, nx)
    ax = A[2] * X
    ax[1:, :] += A[0, 1:, :] * X[:-1, :]
    ax[:, 1:] += A[1, :, 1:] * X[:, :-1]
    ax[:, :-1] += A[3, :, :-1] * X[:, 1:]
    ax[:-1, :] += A[4, :-1, :] * X[1:, :]
    return (b.reshape(ny, nx) - ax).reshape(-1)


def apply(nx, ny, H, W, a5, b, y, sigma, x):
    """x + sigma y on the real cells; each ghost cell solves its own row with
    the corrected real neighbours and the old ghost values."""
    X = x.reshape(ny, nx)
    C = X.copy()
    C[1:-1, 1:-1] += sigma * y[:ny - 2, :nx - 2]
    A = a5.reshape(5, ny, nx)
    B = b.reshape(ny, nx)
    out = C.copy()
    for j in range(ny):
        for i in range(nx):
            if 0 < i < nx - 1 and 0 < j < ny - 1:
                continue
            ap = A[2, j, i]
            if ap == 0.0:
                out[j, i] = X[j, i]
                continue
            v = B[j, i]
            if j > 0:
                v -= A[0, j, i] * C[j - 1, i]
            if i > 0:
                v -= A[1, j, i] * C[j, i - 1]
            if i < nx - 1:
                v -= A[3, j, i] * C[j, i + 1]
            if j < ny - 1:
                v -= A[4, j, i] * C[j + 1, i]
            out[j, i] = v / ap
    return out.reshape(-1)
