"""GPU parity of the SCF-map steps beside the apply: band density sum, the kept-HX
potential-change update, the device potential install and the Hartree + LDA-PZ field
step, each against the oracle (oracle/fields_ref.py) or against the operator's own
full apply on the same inputs."""
import numpy as np
import pytest

from baandi_b200 import _lib as L
from baandi_b200 import systems as W
from baandi_b200.fields import FieldGrid
from baandi_b200.hamiltonian import ComplexHamiltonian, RealGammaHamiltonian, SolverError
from oracle import fields_ref as F
from oracle import setup_ref as S

from tests.helpers import colwise_rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _grid_err(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def _operator(w, k, cols, ctx, gamma):
    pw = w.plane_waves(k)
    nl = w.nonlocal_table(pw)
    cls = RealGammaHamiltonian if gamma else ComplexHamiltonian
    return cls.new_owned(pw, w.dims(), nl, cols, ctx), pw


def _oracle_sphere(w, k, dims):
    cell = S.Cell(w.rows)
    b = S.basis_at_k(cell, w.ecut_ha, k)
    idx = S.fft_flat(S.g_to_fft(b, dims), dims)
    if tuple(k) != (0.0, 0.0, 0.0):
        return idx, None, None
    plus, minus, _ = S.half_sphere(b)
    return idx, plus, minus


# ---------------------------------------------------------------- band density
@pytest.mark.parametrize("name,kidx,cols", [("si8", 5, 24), ("al32", 3, 9)])
def test_band_density_complex(ctx, name, kidx, cols):
    w = W.WORKLOADS[name]()
    k = w.kpoints[kidx][0]
    dims = w.dims()
    op, pw = _operator(w, k, cols, ctx, False)
    x = w.random_block(pw.npw, cols, seed_offset=3)
    weights = np.linspace(2.0, 0.0, cols) * w.kpoints[kidx][1]
    rho = op.band_density_sum(x, weights, w.volume)
    idx, _, _ = _oracle_sphere(w, k, dims)
    ref = F.band_density_sum(dims, idx, x, weights, w.volume)
    assert _grid_err(rho, ref) <= TOL
    # device pointers give the same grid
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    rd = op.band_density_sum(xd, weights, w.volume)
    op.sync()
    assert np.array_equal(rd.cpu().numpy(), rho)
    # k-point sum: accumulate adds onto the caller's grid
    acc = op.band_density_sum(x[:, : cols // 2].copy(order="F"), weights[: cols // 2], w.volume)
    op.band_density_sum(x[:, cols // 2:].copy(order="F"), weights[cols // 2:], w.volume, out=acc, accumulate=True)
    assert _grid_err(acc, ref) <= TOL


@pytest.mark.parametrize("cols", [7, 8])
def test_band_density_gamma(ctx, cols):
    w = W.WORKLOADS["si2"]()
    dims = w.dims()
    op, pw = _operator(w, (0.0, 0.0, 0.0), cols, ctx, True)
    x = w.random_block(pw.npw, cols, seed_offset=4, real=True)
    weights = np.array([2.0, 2.0, 1.5, 1.0, 0.5, 0.25, 0.0, 2.0])[:cols]
    rho = op.band_density_sum(x, weights, w.volume)
    idx, plus, minus = _oracle_sphere(w, (0.0, 0.0, 0.0), dims)
    ref = F.band_density_sum(dims, idx, F.expand_orc(x, plus, minus), weights, w.volume)
    assert _grid_err(rho, ref) <= TOL
    # a normalised band carries its weight of electrons
    n = int(np.prod(dims))
    assert abs(rho.sum() * w.volume / n - weights.sum()) < 1e-10


def test_band_density_rejects(ctx):
    w = W.WORKLOADS["si2"]()
    op, pw = _operator(w, (0.0, 0.0, 0.0), 4, ctx, True)
    x = w.random_block(pw.npw, 4, real=True)
    with pytest.raises(SolverError) as e:
        op.band_density_sum(x, [1.0, -1.0, 1.0, 1.0], w.volume)
    assert e.value.args[0].startswith("BG_ESHAPE")
    with pytest.raises(SolverError):
        op.band_density_sum(x, [1.0] * 4, 0.0)
    bad = x.copy(order="F")
    bad[3, 2] = np.nan
    with pytest.raises(SolverError) as e:
        op.band_density_sum(bad, [1.0] * 4, w.volume)
    assert "BG_ENONFINITE" in str(e.value)
    rho = op.band_density_sum(x, [1.0] * 4, w.volume)  # the operator stays usable
    assert np.all(np.isfinite(rho))


# ---------------------------------------------------------------- kept HX
def _change(w, seed):
    rng = np.random.default_rng(seed)
    return 0.05 * rng.standard_normal(w.dims())


@pytest.mark.parametrize("name,kidx,cols,gamma", [("si8", 7, 10, False), ("si2", 0, 7, True)])
def test_add_local_change_equals_full_apply(ctx, name, kidx, cols, gamma):
    """H_new x = H_old x + (V_new - V_old) x (crates/dft-engine/src/refscf/kept_hx.rs:
    98-160): the kept update matches a fresh apply with the new potential."""
    w = W.WORKLOADS[name]()
    k = w.kpoints[kidx][0]
    op, pw = _operator(w, k, cols, ctx, gamma)
    v0 = w.ionic_potential()
    dv = _change(w, 17)
    x = w.random_block(pw.npw, cols, seed_offset=5, real=gamma)
    op.set_owned_potential(v0, 1)
    hx = op.apply_block(x)
    op.add_local_change(x, dv, hx)
    op.set_owned_potential(v0 + dv, 2)
    fresh = op.apply_block(x)
    assert colwise_rel(hx, fresh) <= TOL
    if not gamma:
        idx, _, _ = _oracle_sphere(w, k, w.dims())
        h0 = np.zeros_like(x)
        ref = F.add_local_change(w.dims(), idx, x, dv, h0)
        got = op.add_local_change(x, dv, np.zeros_like(x, order="F"))
        assert colwise_rel(got, ref) <= TOL


def test_add_local_change_device_and_errors(ctx):
    import torch
    w = W.WORKLOADS["si8"]()
    k = w.kpoints[2][0]
    op, pw = _operator(w, k, 6, ctx, False)
    op.set_owned_potential(w.ionic_potential(), 1)
    x = w.random_block(pw.npw, 6, seed_offset=6)
    dv = _change(w, 18)
    hx = op.apply_block(x)
    want = op.add_local_change(x, dv, hx.copy(order="F"))
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    hd = torch.from_numpy(np.ascontiguousarray(hx.T)).cuda()
    op.add_local_change(xd, torch.from_numpy(dv).cuda(), hd)
    op.sync()
    assert np.array_equal(hd.cpu().numpy().T, want)
    bad = dv.copy()
    bad[1, 2, 3] = np.inf
    keep = hx.copy(order="F")
    with pytest.raises(SolverError) as e:
        op.add_local_change(x, bad, keep)
    assert "BG_ENONFINITE" in str(e.value)
    assert np.array_equal(keep, hx)


def test_set_potential_device_matches_host(ctx):
    import torch
    w = W.WORKLOADS["si8"]()
    k = w.kpoints[1][0]
    op, pw = _operator(w, k, 5, ctx, False)
    v = w.ionic_potential()
    x = w.random_block(pw.npw, 5, seed_offset=7)
    op.set_owned_potential(v, 1)
    a = op.apply_block(x)
    op.set_owned_potential_device(torch.from_numpy(v + 0.0).cuda(), 2)
    b = op.apply_block(x)
    assert np.array_equal(a, b)
    bad = torch.from_numpy(v + 0.0).cuda()
    bad[0, 0, 0] = float("nan")
    with pytest.raises(SolverError):
        op.set_owned_potential_device(bad, 3)
    assert op.owned_epoch() == 2
    assert np.array_equal(op.apply_block(x), a)  # the rejected grid left the old potential


# ---------------------------------------------------------------- fields
def _density(w, seed, signed=False):
    """A smooth positive density (low-pass filtered noise) on the workload's grid;
    `signed` shifts it so that part of the grid is negative (mixed densities can be)."""
    rng = np.random.default_rng(seed)
    dims = w.dims()
    freq = np.meshgrid(*(np.fft.fftfreq(n) * n for n in dims), indexing="ij")
    filt = np.exp(-0.05 * sum(f * f for f in freq))
    smooth = np.fft.ifftn(np.fft.fftn(rng.standard_normal(dims)) * filt).real
    base = 0.02 + 0.01 * np.abs(smooth) / np.max(np.abs(smooth))
    if signed:
        base = base - 0.8 * base.max()
    return np.ascontiguousarray(base)


@pytest.mark.parametrize("name,signed", [("si2", False), ("si8", False), ("al32", True), ("si216", False)])
def test_fields_match_oracle(ctx, name, signed):
    w = W.WORKLOADS[name]()
    rho = _density(w, 11, signed)
    fg = FieldGrid(w.rows, w.dims(), ctx)
    got = fg.lda_hartree(rho)
    hxc, vh, eh, ex, vx = F.fields(w.rows, rho)
    assert _grid_err(got.vh, vh) <= TOL
    assert _grid_err(got.hxc, hxc) <= TOL
    for a, b in ((got.hartree, eh), (got.xc, ex), (got.xc_integral, vx)):
        assert abs(a - b) <= TOL * abs(b)
    import torch
    dev = fg.lda_hartree(torch.from_numpy(rho).cuda())
    assert np.array_equal(dev.hxc.cpu().numpy(), got.hxc)
    assert dev.hartree == got.hartree and dev.xc == got.xc


def test_fields_hartree_analytic(ctx):
    """crates/dft-physics/src/tests.rs:80-150 on the GPU: E_H = 4 pi V A^2/|G|^2 and
    V_H = 8 pi A/|G|^2 cos on the skew Si cell, 12 x 10 x 9 grid."""
    a = 5.43 / 0.529177210903
    rows = np.array([[0, a / 2, a / 2], [a / 2, 0, a / 2], [a / 2, a / 2, 0]])
    dims = (12, 10, 9)
    fg = FieldGrid(rows, dims, ctx)
    i, j, _ = np.meshgrid(*(np.arange(n) for n in dims), indexing="ij")
    cosine = np.cos(2 * np.pi * (i / dims[0] - j / dims[1]))
    amp = 0.02
    got = fg.lda_hartree(np.ascontiguousarray(0.3 + 2 * amp * cosine))
    g2 = F.squared_frequencies(rows, dims)[1, dims[1] - 1, 0]
    vol = fg.volume()
    assert abs(got.hartree - 4 * np.pi * vol * amp * amp / g2) <= 1e-12 * (4 * np.pi * vol * amp * amp / g2)
    vscale = 8 * np.pi * amp / g2
    assert np.max(np.abs(got.vh - vscale * cosine)) / vscale <= 1e-12
    flat = fg.lda_hartree(np.full(dims, 0.3))
    assert abs(flat.hartree) < 1e-14 and np.max(np.abs(flat.vh)) < 1e-14


def test_fields_rejects_nonfinite(ctx):
    w = W.WORKLOADS["si2"]()
    fg = FieldGrid(w.rows, w.dims(), ctx)
    rho = _density(w, 12)
    rho[2, 3, 4] = np.nan
    with pytest.raises(SolverError) as e:
        fg.lda_hartree(rho)
    assert "BG_ENONFINITE" in str(e.value)
    ok = fg.lda_hartree(_density(w, 12))  # usable after the error
    assert np.isfinite(ok.hartree)
    with pytest.raises(SolverError):
        FieldGrid(w.rows, (7, 25, 25), ctx)  # 7 is not 2,3,5-smooth
