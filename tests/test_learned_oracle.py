"""CPU checks of the learned-correction MLP oracle (no GPU): bf16 rounding known answers
and the hand-written backward pass against finite differences of the forward pass."""
import numpy as np

from oracle import mlp as omlp


def test_bf16_round_to_nearest_even():
    one = np.float32(1.)
    ulp = 2.**-7  # bf16 spacing at 1
    cases = {1.: 1., 1. + ulp / 2: 1., 1. + 1.5 * ulp: 1. + 2 * ulp, 1. + ulp / 2 + 2.**-20: 1. + ulp,
             -3.140625: -3.140625, 0.: 0., 65504.: 65536.}
    for x, expected in cases.items():
        assert omlp.bf16(np.float32(x)) == expected, x
    assert omlp.bf16(one) == 1.


def _params(seed):
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in omlp.LAYOUT:
        fan_in = shape[-1]
        p[name] = rng.normal(size=shape) / np.sqrt(fan_in) if name.startswith('W') else 0.1 * rng.normal(size=shape)
    return omlp.flatten(p)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    flat = _params(0)
    x = rng.normal(size=(9, omlp.IN))
    dy = rng.normal(size=9)
    _, cache = omlp.forward(flat, x, rounding=False)
    g = omlp.backward(flat, cache, dy, rounding=False)
    layout = {name: shape for name, shape in omlp.LAYOUT}
    offsets = np.cumsum([0] + [int(np.prod(s)) for _, s in omlp.LAYOUT])
    picks = []
    for (name, shape), off in zip(omlp.LAYOUT, offsets):
        n = int(np.prod(shape))
        if name == 'W3':
            picks += [off + j for j in rng.choice(omlp.H, 4, replace=False)]  # row 0 is the used output row
        elif name == 'b3':
            picks.append(off)
        else:
            picks += list(off + rng.choice(n, 4, replace=False))
    eps = 1e-6
    for i in picks:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += eps
        fm[i] -= eps
        num = (dy @ omlp.forward(fp, x, rounding=False)[0] - dy @ omlp.forward(fm, x, rounding=False)[0]) / (2 * eps)
        assert np.isclose(g[i], num, rtol=1e-5, atol=1e-8), (i, g[i], num)
    # unused output rows / bias entries have zero gradient
    w3 = offsets[[n for n, _ in omlp.LAYOUT].index('W3')]
    assert np.all(g[w3 + omlp.H:w3 + omlp.OUT * omlp.H] == 0.)


def test_adam_matches_closed_form_first_step():
    w, m, v = np.ones(4), np.zeros(4), np.zeros(4)
    g = np.array([1., -2., 0.5, 0.])
    w1, m1, v1 = omlp.adam(w, m, v, g, lr=0.1, step=1)
    # first bias-corrected step is lr * sign(g) (up to eps)
    assert np.allclose(w1, 1. - 0.1 * np.sign(g), atol=1e-6)
