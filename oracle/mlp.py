"""CPU oracle of the learned-correction MLP (test infrastructure only).

The learned correction has no counterpart in the reference; this module restates the
network the CUDA kernels implement, so the kernels' forward pass and gradients can be
checked on the same inputs:

- 4 dense layers 16 -> 128 -> 128 -> 128 -> 1 with SiLU, z * sigmoid(z), after the three
  hidden layers; parameters in one flat float32 vector (``LAYOUT``);
- tensor-core operands rounded to bfloat16 (round to nearest even): inputs, weights,
  hidden activations and, in the backward pass, dL/dZ; sums and biases in float
  (float64 here, float32 on the GPU);
- ``rounding=False`` gives the exact float64 network, used to check ``backward`` against
  finite differences (``tests/test_learned.py``).
"""
import numpy as np

IN, H, OUT = 16, 128, 8
LAYOUT = [('W0', (H, IN)), ('b0', (H,)), ('W1', (H, H)), ('b1', (H,)), ('W2', (H, H)), ('b2', (H,)),
          ('W3', (OUT, H)), ('b3', (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in LAYOUT)


def unflatten(flat):
    out, off = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[off:off + n]).reshape(shape)
        off += n
    return out


def flatten(params):
    return np.concatenate([np.asarray(params[name], dtype='f8').ravel() for name, _ in LAYOUT])


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.asarray(x, dtype='f4').view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype('f8')


def _silu(z):
    return z / (1. + np.exp(-z))


def _silu_grad(z):
    s = 1. / (1. + np.exp(-z))
    return s * (1. + z * (1. - s))


def forward(flat, x, rounding=True):
    """y (batch,) and the cache (inputs, pre-activations, activations) of the backward pass."""
    p = unflatten(np.asarray(flat, dtype='f8'))
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype='f8'))
    a = rnd(x)
    acts, zs = [a], []
    for l in range(3):
        z = a @ rnd(p['W{:d}'.format(l)]).T + p['b{:d}'.format(l)]
        h = _silu(z)
        zs.append(z)
        a = rnd(h)
        acts.append(a)
    y = a @ rnd(p['W3'][0]) + p['b3'][0]
    return y, (acts, zs)


def backward(flat, cache, dy, rounding=True):
    """Gradient of sum_i dy_i y_i with respect to the flat parameters."""
    p = unflatten(np.asarray(flat, dtype='f8'))
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype='f8'))
    acts, zs = cache
    g = {name: np.zeros(shape) for name, shape in LAYOUT}
    g['W3'][0] = dy @ acts[3]
    g['b3'][0] = dy.sum()
    dh = dy[:, None] * rnd(p['W3'][0])[None, :]
    for l in (2, 1, 0):
        dz = dh * _silu_grad(zs[l])
        g['b{:d}'.format(l)] = dz.sum(axis=0)
        g['W{:d}'.format(l)] = rnd(dz).T @ acts[l]
        if l > 0:
            dh = rnd(dz) @ rnd(p['W{:d}'.format(l)])
    return flatten(g)


def mse(y, target, weight=None):
    w = np.ones_like(target) if weight is None else weight
    d = y - target
    return float((w * d * d).mean()), 2. * w * d / len(y)


def adam(w, m, v, g, lr, step, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.):
    """AdamW step (bias-corrected moments, decoupled weight decay); returns new (w, m, v)."""
    m = beta1 * m + (1. - beta1) * g
    v = beta2 * v + (1. - beta2) * g * g
    c1, c2 = 1. - beta1**step, 1. - beta2**step
    w = w - lr * ((m / c1) / (np.sqrt(v / c2) + eps) + weight_decay * w)
    return w, m, v
