"""The k-point set's potential install and band density (bg_kset_set_potential_ptr,
bg_kset_band_density_sum) against the per-operator calls they batch."""
import numpy as np
import pytest

from baandi_b200 import _lib as L
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, KPointSet, RealGammaHamiltonian, SolverError
from tests.helpers import colwise_rel

pytestmark = pytest.mark.gpu


def _set(w, kidx, cols, ctx, gamma=False):
    """Operators and their set, all on torch's current stream (as the SCF driver runs
    them), so that grids made by torch are complete before the library reads them."""
    import torch
    s = torch.cuda.current_stream().cuda_stream
    ops = []
    for i in kidx:
        pw = w.plane_waves(w.kpoints[i][0])
        cls = RealGammaHamiltonian if gamma else ComplexHamiltonian
        op = cls.new_owned(pw, w.dims(), w.nonlocal_table(pw), cols, ctx)
        op.set_stream(s)
        ops.append(op)
    ks = KPointSet(ops, ctx)
    ks.set_stream(s)
    return ops, ks


def _blocks(w, ops, cols, gamma=False):
    import torch
    out = []
    for i, op in enumerate(ops):
        x = w.random_block(op.npw, cols, seed_offset=40 + i, real=gamma)
        out.append(torch.from_numpy(np.ascontiguousarray(x.T)).cuda())
    return out


def test_set_potential_matches_per_operator_install(ctx):
    import torch
    w = W.si8_k444()
    ops, ks = _set(w, (0, 5, 17), 8, ctx)
    ref_ops, _ = _set(w, (0, 5, 17), 8, ctx)
    v = torch.from_numpy(w.ionic_potential()).cuda()
    v2 = v + 0.05 * torch.cos(torch.arange(v.numel(), device="cuda", dtype=torch.float64)).reshape(v.shape)
    ks.set_potential_device(v2, 3)
    for op in ref_ops:
        op.set_owned_potential_device(v2, 3)
    xs = _blocks(w, ops, 8)
    for op, r, x in zip(ops, ref_ops, xs):
        assert torch.equal(op.apply_block(x), r.apply_block(x))
    # FP32 after a set install converts the new potential (a stale copy would differ by
    # the 0.05 change; the set and the single apply split the FP64 nonlocal sums
    # differently, so they agree to rounding)
    ks.precision = L.BG_PREC_FP32
    ys = ks.apply_blocks(xs)
    for r, x, y in zip(ref_ops, xs, ys):
        r.precision = L.BG_PREC_FP32
        assert colwise_rel(y.cpu().numpy().T, r.apply_block(x).cpu().numpy().T) < 1e-13


def test_set_potential_rejects_nonfinite_and_stale_epochs(ctx):
    import torch
    w = W.si8_k444()
    ops, ks = _set(w, (1, 2), 4, ctx)
    v = torch.from_numpy(w.ionic_potential()).cuda()
    ks.set_potential_device(v, 5)
    xs = _blocks(w, ops, 4)
    before = [op.apply_block(x) for op, x in zip(ops, xs)]
    bad = v.clone()
    bad[3, 4, 5] = float("nan")
    with pytest.raises(SolverError):
        ks.set_potential_device(bad, 6)
    for op, x, y in zip(ops, xs, before):
        assert torch.equal(op.apply_block(x), y)   # old potential kept everywhere
    with pytest.raises(SolverError):
        ks.set_potential_device(v, 5)   # epoch must increase
    ks.set_potential_device(v, 7)


@pytest.mark.parametrize("name,kidx,gamma", [("si8", (0, 3, 9, 20), False), ("si2", (0,), True)])
def test_set_band_density_equals_per_operator_sum(ctx, name, kidx, gamma):
    import torch
    w = W.WORKLOADS[name]()
    cols = 6
    ops, ks = _set(w, kidx, cols, ctx, gamma)
    xs = _blocks(w, ops, cols, gamma)
    rng = np.random.default_rng(4)
    wts = rng.uniform(0.0, 2.0, (len(ops), cols))
    vol = w.volume
    ref = torch.zeros(w.dims(), dtype=torch.float64, device="cuda")
    for k, (op, x) in enumerate(zip(ops, xs)):
        op.band_density_sum(x, wts[k], vol, out=ref, accumulate=k > 0)
    got = ks.band_density_sum(xs, wts, vol)
    assert float((got - ref).abs().max() / ref.abs().max()) < 1e-13
    # accumulate adds into the given grid
    base = torch.full_like(ref, 0.25)
    acc = ks.band_density_sum(xs, wts, vol, out=base.clone(), accumulate=True)
    assert float((acc - base - got).abs().max() / ref.abs().max()) < 1e-13


def test_set_band_density_checks(ctx):
    w = W.si8_k444()
    ops, ks = _set(w, (0, 1), 4, ctx)
    xs = _blocks(w, ops, 4)
    with pytest.raises(SolverError):
        ks.band_density_sum(xs, np.full((2, 4), -1.0), w.volume)
    with pytest.raises(SolverError):
        ks.band_density_sum(xs, np.ones((2, 4)), 0.0)
    with pytest.raises(SolverError):
        ks.band_density_sum(xs, np.ones((2, 3)), w.volume)
