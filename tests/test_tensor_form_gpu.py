"""The precision form on the tensor cores (BG_PREC_TENSOR): the H apply with its local
part in FP32 and P^H x, P W as BF16x3 products; the batched Davidson whose first phase
uses those applies plus BF16x3 H Grams and rotations and hands over to FP64 once every
active residual is below 1e-4; and the SCF built on it.  Errors are stated against the
FP64 forms: the apply within 2e-5 relative per column, Davidson eigenvalues within 1e-8
Ha of the FP64 solve (convergence is judged in FP64), SCF energy within 1e-6 Ha/atom."""
import numpy as np
import pytest

from baandi_b200 import _lib as L
from baandi_b200 import davidson as DV
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, KPointSet
from tests.helpers import colwise_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,cols", [("si64", 12), ("si216", 6), ("al32", 5)])
def test_tensor_apply_error(ctx, name, cols):
    w = W.WORKLOADS[name]()
    k = w.kpoints[-1][0]
    pw = w.plane_waves(k)
    op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 16, ctx)
    op.set_owned_potential(w.ionic_potential(), 1)
    x = w.random_block(pw.npw, cols, seed_offset=3)
    ref = op.apply_block(x)
    op.precision = L.BG_PREC_TENSOR
    y = op.apply_block(x)
    op.precision = L.BG_PREC_FP64
    err = colwise_rel(y, ref)
    assert 0.0 < err <= 2e-5, err


def test_tensor_kset_apply_matches_operator(ctx):
    """Batched tensor applies over several k points agree with the per-operator ones (their
    split-K depths differ, so to the FP32 accumulation's rounding)."""
    import torch
    w = W.al32_k222()
    v = w.ionic_potential()
    ops, xs = [], []
    for i, (k, _) in enumerate(w.kpoints[:3]):
        pw = w.plane_waves(k)
        op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 8, ctx)
        op.set_owned_potential(v, 1)
        ops.append(op)
        xs.append(torch.from_numpy(np.ascontiguousarray(w.random_block(pw.npw, 8, seed_offset=i).T)).cuda())
    ks = KPointSet(ops, ctx)
    ks.precision = L.BG_PREC_TENSOR
    ys = ks.apply_blocks(xs)
    ks.sync()
    for op, x, y in zip(ops, xs, ys):
        op.precision = L.BG_PREC_TENSOR
        ref = op.apply_block(x)
        op.sync()
        assert float(((y - ref).norm(dim=1) / ref.norm(dim=1)).max()) <= 2e-5


def test_tensor_davidson_hands_over_to_fp64(ctx):
    """Si64, 160 bands at capacity 320: the precision form reaches the FP64 solve's
    eigenvalues within 1e-8 Ha (occupied) after a tensor-core phase of at least one
    iteration."""
    w = W.si64_gamma()
    pw = w.plane_waves()
    v = w.ionic_potential()
    op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 320, ctx)
    op.set_owned_potential(v, 1)
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, 160, seed_offset=5)
    ks = KPointSet([op], ctx)
    base = dict(bands=160, threshold=1e-9, occupied=128, first_step=False, max_iterations=60)
    (ref,) = DV.solve_kset(ks, [start], [diag], DV.Options(**base))
    (ten,) = DV.solve_kset(ks, [start], [diag], DV.Options(**base, apply_precision="tensor"))
    assert ten.tensor_iterations >= 1
    assert ten.converged[:128].sum() >= ref.converged[:128].sum() - 4
    conv = ten.converged[:128] & ref.converged[:128]
    assert conv.sum() >= 64
    assert np.max(np.abs(ten.eigenvalues[:128][conv] - ref.eigenvalues[:128][conv])) < 1e-8


def test_tensor_scf_energy_matches_fp64(ctx):
    """Si64 SCF (Thomas-Fermi mixing, Fermi-Dirac 0.01 Ha): the precision form's total
    energy within 1e-6 Ha/atom of the FP64 SCF.  Both run to 1e-7 Ha/atom, so that the two
    trajectories' own convergence error (up to the SCF threshold each) stays well below
    the bound and the comparison measures the precision form."""
    from baandi_b200.scf import GpuScf, ScfOptions
    w = W.si64_gamma()
    o = dict(threshold_ha=1e-7 * w.natoms, smearing_ha=0.01, thomas_fermi=True)
    plain = GpuScf(w, ctx, ScfOptions(**o)).run()
    tensor = GpuScf(w, ctx, ScfOptions(**o, tensor=True)).run()
    assert plain.converged and tensor.converged
    assert abs(tensor.energy_ha - plain.energy_ha) <= 1e-6 * w.natoms
    assert any(r.tensor_iterations > 0 for r in tensor.records)


def test_autotuner_times_the_projection_split(ctx):
    """A tensor-form apply tunes the split-K count of its projection once per shape: the
    report lists the timed counts (each at least the accuracy bound's minimum of one split
    per 4,096 complex K) and the fastest one is kept."""
    w = W.si8_k444()
    pw = w.plane_waves(w.kpoints[2][0])
    nl = w.nonlocal_table(pw)
    nproj = int(nl.table.shape[1])   # the table is (npw, nproj)
    op = ComplexHamiltonian.new_owned(pw, w.dims(), nl, 24, ctx)
    op.set_owned_potential(w.ionic_potential(), 1)
    x = w.random_block(pw.npw, 24, seed_offset=4)
    op.precision = L.BG_PREC_TENSOR
    y = op.apply_block(x)
    op.precision = L.BG_PREC_FP64
    ref = op.apply_block(x)
    assert np.max(np.linalg.norm(y - ref, axis=0) / np.linalg.norm(ref, axis=0)) < 2e-5
    entries = [e for e in L.autotune_report() if e["m"] == nproj and e["k"] == pw.npw and e["n"] == 24]
    assert len(entries) == 1
    e = entries[0]
    timed = {int(k): v for k, v in e["timed_ms"].items()}
    assert timed and e["ksplit"] in timed
    assert timed[e["ksplit"]] == min(timed.values())
    assert min(timed) >= -(-2 * pw.npw // 32) // 256
