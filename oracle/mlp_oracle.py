"""CPU restatement of the warm-start network (multiphaselb_b200/csrc/mplb_mlp.cu).
TEST INFRASTRUCTURE ONLY: tests use it to check the device forward pass and
gradients; the product never imports it.

The network has no counterpart in the reference.  What is restated here:
  * the parameter layout W1[64][5], b1, W2[64][64], b2, W3[64][64], b3,
    W4[64], b4 (8769 floats);
  * the input features (T/Tc, a, b, r, R) -> (T/Tc, a, b, (r - R)/5 clamped
    to [-6, 6], 5/R), normalised, BF16-rounded;
  * the forward pass: BF16 weights, tanh hidden units whose outputs are
    rounded to BF16, FP32 biases, a linear output (b * rho);
  * the gradient of the mean squared error, with the BF16 roundings treated
    as identities in the backward pass (as the device does: it
    differentiates through the stored, rounded activations).
Arithmetic here is FP64; the device accumulates in FP32, so the two agree
to FP32 rounding, not bit for bit.
"""
import numpy as np

NIN, NH = 5, 64
OFF = {}
_o = 0
for _name, _size in (("W1", NH * NIN), ("b1", NH), ("W2", NH * NH), ("b2", NH), ("W3", NH * NH), ("b3", NH),
                     ("W4", NH), ("b4", 1)):
    OFF[_name] = (_o, _size)
    _o += _size
NPARAM = _o


def bf16(x):
    """Round float32 values to the nearest BF16 value, ties to even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def features(t_ratio, a, b, r, R):
    """Network inputs (multiphaselb_b200/csrc/mplb_mlp.cu features()); R = +inf
    marks a flat interface, r then being the signed distance to it."""
    R = np.asarray(R, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    flat = np.isinf(R)
    d = np.clip(np.where(flat, r, r - np.where(flat, 0.0, R)) / 5.0, -6.0, 6.0)
    cols = [(np.asarray(t_ratio, dtype=np.float64) - 0.775) / 0.175,
            np.asarray(a, dtype=np.float64) - 1.0,
            np.asarray(b, dtype=np.float64) * 0.25 - 1.0,
            d / 6.0,
            (5.0 / R - 0.3) / 0.3]
    return np.stack([bf16(np.asarray(c, dtype=np.float32)) for c in np.broadcast_arrays(*cols)], axis=-1)


def unpack(params, quantize=True):
    p = np.asarray(params, dtype=np.float32 if quantize else np.float64)
    get = lambda k: p[OFF[k][0]:OFF[k][0] + OFF[k][1]]  # noqa: E731
    q = bf16 if quantize else (lambda v: v)
    W = dict(W1=q(get("W1")).reshape(NH, NIN), W2=q(get("W2")).reshape(NH, NH), W3=q(get("W3")).reshape(NH, NH),
             W4=q(get("W4")).reshape(NH))
    B = dict(b1=get("b1"), b2=get("b2"), b3=get("b3"), b4=get("b4")[0])
    return {k: v.astype(np.float64) for k, v in {**W, **B}.items()}


def forward(params, X, quantize=True):
    """Activations (x, h1, h2, h3) and outputs for inputs X [n][4]."""
    w = unpack(params, quantize)
    act = (lambda z: bf16(np.tanh(z).astype(np.float32)).astype(np.float64)) if quantize else np.tanh
    x = np.asarray(X, dtype=np.float64)
    h1 = act(x @ w["W1"].T + w["b1"])
    h2 = act(h1 @ w["W2"].T + w["b2"])
    h3 = act(h2 @ w["W3"].T + w["b3"])
    out = h3 @ w["W4"] + w["b4"]
    return (x, h1, h2, h3), out


def loss_and_grad(params, X, Y, quantize=True):
    """Mean squared error and its gradient (FP64, parameter layout above)."""
    w = unpack(params, quantize)
    (x, h1, h2, h3), out = forward(params, X, quantize)
    n = x.shape[0]
    d = out - np.asarray(Y, dtype=np.float64)
    loss = float(np.mean(d * d))
    dout = 2.0 * d / n
    g = np.zeros(NPARAM)

    def put(k, v):
        g[OFF[k][0]:OFF[k][0] + OFF[k][1]] = np.ravel(v)

    put("b4", [dout.sum()])
    put("W4", dout @ h3)
    dz3 = np.outer(dout, w["W4"]) * (1.0 - h3 * h3)
    put("W3", dz3.T @ h2)
    put("b3", dz3.sum(axis=0))
    dz2 = (dz3 @ w["W3"]) * (1.0 - h2 * h2)
    put("W2", dz2.T @ h1)
    put("b2", dz2.sum(axis=0))
    dz1 = (dz2 @ w["W2"]) * (1.0 - h1 * h1)
    put("W1", dz1.T @ x)
    put("b1", dz1.sum(axis=0))
    return loss, g


def finite_difference(params, X, Y, idx, h=1e-6):
    """Central differences of the unrounded FP64 loss for parameters idx."""
    p = np.asarray(params, dtype=np.float64)
    out = []
    for i in idx:
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        la = _loss64(a, X, Y)
        lb = _loss64(b, X, Y)
        out.append((la - lb) / (2 * h))
    return np.array(out)


def _loss64(p, X, Y):
    get = lambda k: p[OFF[k][0]:OFF[k][0] + OFF[k][1]]  # noqa: E731
    x = np.asarray(X, dtype=np.float64)
    h1 = np.tanh(x @ get("W1").reshape(NH, NIN).T + get("b1"))
    h2 = np.tanh(h1 @ get("W2").reshape(NH, NH).T + get("b2"))
    h3 = np.tanh(h2 @ get("W3").reshape(NH, NH).T + get("b3"))
    out = h3 @ get("W4") + get("b4")[0]
    d = out - Y
    return float(np.mean(d * d))


def loss_and_grad64(params, X, Y):
    """Unrounded FP64 loss and analytic gradient (for the finite-difference check)."""
    return loss_and_grad(np.asarray(params, dtype=np.float64), X, Y, quantize=False)
