"""The learned preconditioner's oracle (FP64 numpy) on the CPU: its gradient against
finite differences, the BF16 rounding of the host side against torch's, and the start
network being TPA."""
import numpy as np

from baandi_b200 import learned as LP
from oracle import learned_ref as R


def _random_samples(rng, rows=40, cols=3, cplx=True):
    kin = np.sort(rng.uniform(0.0, 6.0, rows))
    x = rng.standard_normal((rows, cols)) + (1j * rng.standard_normal((rows, cols)) if cplx else 0)
    x /= np.linalg.norm(x, axis=0)
    hx = x * (kin[:, None] + 0.3) + 0.05 * (rng.standard_normal((rows, cols)) + (1j if cplx else 0))
    e = 0.1 * (rng.standard_normal((rows, cols)) + (1j * rng.standard_normal((rows, cols)) if cplx else 0))
    lam = np.sum(np.conj(x) * hx, axis=0).real
    return R.samples(x, hx, e, kin, lam)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    s = _random_samples(rng)
    p = LP.init_params(1).astype(np.float64)
    p[R.OW3:R.OB3] = rng.normal(0, 0.3, R.N_HID)   # a live output layer
    p[R.OB3] = 0.1
    loss, g = R.loss_grad(p, *s)
    assert 0.0 < loss < 1.0
    idx = list(rng.choice(R.NPARAMS, 40, replace=False)) + [R.OB3, R.OW3 + 5, R.OW1, R.OB1 + 3, R.OW2 + 100]
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (R.loss_grad(pp, *s)[0] - R.loss_grad(pm, *s)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])


def test_real_samples_have_real_products():
    rng = np.random.default_rng(4)
    feats, base, a, z, col, ecol = _random_samples(rng, cplx=False)
    assert np.all(np.imag(z) == 0.0)
    assert np.all(base <= 0.0) and np.all(base >= -1.0)


def test_start_network_is_tpa():
    rng = np.random.default_rng(5)
    feats = rng.normal(0, 2, (100, R.N_IN))
    m, _ = R.forward(LP.init_params(0), feats)
    assert np.all(m == 0.0)


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(6)
    v = np.concatenate([rng.normal(0, 1, 1000), rng.normal(0, 1e-3, 100), [0.0, -0.0, 1.0, 65504.0]]).astype(np.float32)
    ours = LP.to_bf16_bits(v)
    ref = torch.from_numpy(v).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(ours, ref)
    assert np.array_equal(LP.from_bf16_bits(ours), torch.from_numpy(v).to(torch.bfloat16).float().numpy())
