"""CPU reference of the scenario surrogate's network: forward pass, loss and
analytic gradients in numpy.

TEST INFRASTRUCTURE: the surrogate tests and nothing else use this file.  It
restates the network that covid-sim_b200/csrc/cs_surrogate.cu trains (no
counterpart in the reference, which has no learned model):

    x [B, 8] -> 4 x (Linear 512 + ReLU) -> Linear 256 + ReLU        (MLP, latent 256)
    -> Linear 64*46 + ReLU -> [B, 46, 64]                            (time-major)
    -> 3 x (nearest upsample x2 -> Conv1d k=5, pad 2)  channels 64 -> 64 -> 32 -> 4,
       ReLU after the first two
    -> first 365 of 368 time points -> y [B, 365, 4]
    loss = mean((y - target)^2)

Weights are stored [out, in] (a Conv1d weight [out, k * in + c] for tap k and
input channel c).  `bf16` rounds to bfloat16 (round to nearest even) at the
points where the GPU stores bfloat16: weights, the input, and every activation
that feeds a matrix product.
"""
import numpy as np

N_IN = 8
WIDTH = 512
LATENT = 256
T0, C0 = 46, 64
CONV = ((64, 64, True), (64, 32, True), (32, 4, False))   # (in, out, relu)
T_OUT, N_OUT = 365, 4
KTAP = 5


def layer_shapes():
    """[(name, weight shape [out, in]), ...] in the flat parameter order (each
    weight is followed by its bias [out])."""
    shapes = [("W1", (WIDTH, N_IN)), ("W2", (WIDTH, WIDTH)), ("W3", (WIDTH, WIDTH)), ("W4", (WIDTH, WIDTH)),
              ("W5", (LATENT, WIDTH)), ("D0", (T0 * C0, LATENT))]
    for i, (ci, co, _) in enumerate(CONV):
        shapes.append(("C%d" % (i + 1), (co, KTAP * ci)))
    return shapes


def n_params():
    return sum(o * i + o for _, (o, i) in layer_shapes())


def unflatten(flat):
    out, k = [], 0
    for name, (o, i) in layer_shapes():
        W = flat[k:k + o * i].reshape(o, i); k += o * i
        b = flat[k:k + o]; k += o
        out.append((W, b))
    return out


def flatten(params):
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in params])


def init_params(seed):
    """He-uniform weights, zero biases (the same draws the GPU library is given)."""
    rng = np.random.default_rng(seed)
    out = []
    for name, (o, i) in layer_shapes():
        lim = np.sqrt(6.0 / i)
        out.append((rng.uniform(-lim, lim, size=(o, i)).astype(np.float32), np.zeros(o, np.float32)))
    return flatten(out)


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def _im2col_up(x):
    """x [B, T, C] -> columns [B, 2T, KTAP*C] of the x2 nearest-upsampled, zero-padded input."""
    B, T, C = x.shape
    up = np.repeat(x, 2, axis=1)                       # [B, 2T, C]
    pad = np.zeros((B, 2 * T + KTAP - 1, C), x.dtype)
    pad[:, KTAP // 2:KTAP // 2 + 2 * T] = up
    cols = np.concatenate([pad[:, k:k + 2 * T] for k in range(KTAP)], axis=2)
    return cols


def _col2im_up(dcols, T, C):
    """Adjoint of _im2col_up: dcols [B, 2T, KTAP*C] -> dx [B, T, C]."""
    B = dcols.shape[0]
    dpad = np.zeros((B, 2 * T + KTAP - 1, C), dcols.dtype)
    for k in range(KTAP):
        dpad[:, k:k + 2 * T] += dcols[:, :, k * C:(k + 1) * C]
    dup = dpad[:, KTAP // 2:KTAP // 2 + 2 * T]
    return dup[:, 0::2] + dup[:, 1::2]


def forward(flat, x, round_bf16=False, keep=False):
    """y [B, 365, 4]; with keep, also the intermediate values backward needs."""
    rnd = bf16 if round_bf16 else (lambda a: a)
    dt = np.float32 if round_bf16 else np.float64
    P = [(rnd(W.astype(dt)).astype(dt), b.astype(dt)) for W, b in unflatten(np.asarray(flat))]
    h = rnd(np.asarray(x, dt))
    acts = [h]
    for li in range(6):
        W, b = P[li]
        z = h @ W.T + b
        h = rnd(np.maximum(z, 0))
        acts.append(h)
    B = h.shape[0]
    h = h.reshape(B, T0, C0)
    conv_in = []
    for ci, (cin, cout, relu) in enumerate(CONV):
        W, b = P[6 + ci]
        cols = _im2col_up(h)
        conv_in.append((h, cols))
        z = cols @ W.T + b
        h = rnd(np.maximum(z, 0)) if relu else z
    y = h[:, :T_OUT, :]
    if keep:
        return y, dict(P=P, acts=acts, conv_in=conv_in, conv_out=h)
    return y


def loss_and_grads(flat, x, target, round_bf16=False):
    """(loss, flat gradient) of mean((y - target)^2)."""
    y, st = forward(flat, x, round_bf16, keep=True)
    P = st["P"]
    B = y.shape[0]
    n = y.size
    diff = y - target
    loss = float(np.mean(diff * diff))
    dh = np.zeros_like(st["conv_out"])
    dh[:, :T_OUT, :] = 2.0 * diff / n
    grads = [None] * len(P)
    for ci in reversed(range(len(CONV))):
        cin, cout, relu = CONV[ci]
        W, b = P[6 + ci]
        h_in, cols = st["conv_in"][ci]
        h_out = st["conv_out"] if ci == len(CONV) - 1 else st["conv_in"][ci + 1][0]
        dz = dh * (h_out > 0) if relu else dh
        dz2 = dz.reshape(-1, cout)
        grads[6 + ci] = (dz2.T @ cols.reshape(-1, KTAP * cin), dz2.sum(0))
        dcols = (dz2 @ W).reshape(B, -1, KTAP * cin)
        dh = _col2im_up(dcols, h_in.shape[1], cin)
    dh = dh.reshape(B, T0 * C0)
    for li in reversed(range(6)):
        W, b = P[li]
        h_out, h_in = st["acts"][li + 1], st["acts"][li]
        dz = dh * (h_out > 0)
        grads[li] = (dz.T @ h_in, dz.sum(0))
        dh = dz @ W
    return loss, flatten(grads)
