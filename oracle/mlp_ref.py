"""CPU reference of the warm-start MLP (test infrastructure only).

The network the GPU trains with its tcgen05 BF16 kernels, restated in numpy
float64: n_in inputs (zero-padded to 64) -> `depth` tanh layers of `width`
-> n_out linear outputs, mean-squared-error loss.  There is no network in
the reference code (the warm start is new), so this restatement is the
whole oracle for it; it mirrors the flat parameter layout of
dgbgk_mlp_get_params (per layer W [out][in] row-major, then b [out]).

`bf16=True` rounds every tensor the GPU holds in BF16 (weights, hidden
activations, output-loss gradient and hidden gradients) to BF16 at the same
points, so the GPU result differs from it only by FP32 accumulation order
and by the odd BF16 tie that falls the other way; `bf16=False` is the exact
float64 network the BF16 one approximates.
"""
import numpy as np

KPAD = 64


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def shapes(n_in, width, depth, n_out):
    """(out, in, live_in) per layer, as the GPU lays them out."""
    out = []
    for l in range(depth + 1):
        i = KPAD if l == 0 else width
        out.append((n_out if l == depth else width, i, n_in if l == 0 else width))
    return out


def unflatten(p, n_in, width, depth, n_out):
    Ws, bs, o = [], [], 0
    for (no, ni, _) in shapes(n_in, width, depth, n_out):
        Ws.append(np.asarray(p[o:o + no * ni], dtype=np.float64).reshape(no, ni))
        o += no * ni
        bs.append(np.asarray(p[o:o + no], dtype=np.float64))
        o += no
    return Ws, bs


def flatten(Ws, bs):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in zip(Ws, bs)])


def _pad(x):
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((x.shape[0], KPAD))
    out[:, :x.shape[1]] = x
    return out


def forward(p, x, n_in, width, depth, n_out, bf16_points=True):
    """Network outputs for rows x [n][n_in]; returns (y, hidden list)."""
    rnd = bf16 if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    Ws, bs = unflatten(p, n_in, width, depth, n_out)
    h = rnd(_pad(x))
    H = [h]
    for l in range(depth):
        h = rnd(np.tanh(h @ rnd(Ws[l]).T + bs[l]))
        H.append(h)
    y = h @ rnd(Ws[depth]).T + bs[depth]
    return y, H


def loss_and_grad(p, x, t, n_in, width, depth, n_out, bf16_points=True):
    """Mean squared error over the batch and its gradient (flat layout)."""
    rnd = bf16 if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    Ws, bs = unflatten(p, n_in, width, depth, n_out)
    y, H = forward(p, x, n_in, width, depth, n_out, bf16_points)
    t = np.asarray(t, dtype=np.float64)
    d = y - t
    loss = float(np.mean(d * d))
    g = rnd(2.0 * d / d.size)
    gW, gb = [None] * (depth + 1), [None] * (depth + 1)
    for l in range(depth, -1, -1):
        gW[l] = g.T @ H[l]
        gb[l] = g.sum(axis=0)
        if l > 0:
            g = rnd((g @ rnd(Ws[l])) * (1.0 - H[l] * H[l]))
    gW[0][:, n_in:] = 0.0
    return loss, flatten(gW, gb)
