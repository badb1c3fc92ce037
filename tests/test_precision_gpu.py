"""The precision form of the apply (BG_PREC_FP32: scatter, 3D transforms, x V(r) and
gather in FP32; kinetic and nonlocal parts in FP64) against the FP64 apply, and the
Davidson with FP32 applies against the FP64 one."""
import numpy as np
import pytest

from baandi_b200 import _lib as L
from baandi_b200 import davidson as DV
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, KPointSet, RealGammaHamiltonian, SolverError
from tests.helpers import colwise_rel

pytestmark = pytest.mark.gpu

TOL32 = 2e-5   # relative |H x|: FP32 element error growing over the 3D transform stages


def _op(w, kidx, cols, ctx, gamma=False):
    k = w.kpoints[kidx][0]
    pw = w.plane_waves(k)
    cls = RealGammaHamiltonian if gamma else ComplexHamiltonian
    op = cls.new_owned(pw, w.dims(), w.nonlocal_table(pw), cols, ctx)
    op.set_owned_potential(w.ionic_potential(), 1)
    return op, pw


@pytest.mark.parametrize("name,kidx,cols,gamma", [("si8", 4, 12, False), ("si2", 0, 7, True), ("al32", 2, 6, False)])
def test_fp32_apply_close_to_fp64(ctx, name, kidx, cols, gamma):
    w = W.WORKLOADS[name]()
    op, pw = _op(w, kidx, cols, ctx, gamma)
    x = w.random_block(pw.npw, cols, seed_offset=9, real=gamma)
    y64 = op.apply_block(x)
    op.precision = L.BG_PREC_FP32
    y32 = op.apply_block(x)
    err = colwise_rel(y32, y64)
    assert 1e-9 < err <= TOL32, err   # really FP32, and close


def test_fp32_kset_equals_single_applies(ctx):
    w = W.si8_k444()
    ops, xs = [], []
    for i in (0, 9, 30):
        op, pw = _op(w, i, 8, ctx)
        op.precision = L.BG_PREC_FP32
        ops.append(op)
        xs.append(w.random_block(pw.npw, 8, seed_offset=i))
    ks = KPointSet(ops, ctx)
    ks.precision = L.BG_PREC_FP32
    ys = ks.apply_blocks(xs)
    for op, x, y in zip(ops, xs, ys):
        assert colwise_rel(y, op.apply_block(x)) < 1e-13


def test_fp32_davidson_close_to_fp64(ctx):
    """Eigenvalues of a Si8 k point with FP32 applies agree with the FP64 solve to the
    FP32 level (1e-5 Ha)."""
    w = W.si8_k444()
    op, pw = _op(w, 6, 48, ctx)
    v = w.ionic_potential()
    diag = op.diagonal_static() + v.mean()
    start = w.random_block(pw.npw, 24, seed_offset=3)
    ref = DV.solve(op, start, diag, DV.Options(24, 1e-8, 16, first_step=True, max_iterations=60))
    ks = KPointSet([op], ctx)
    (sol,) = DV.solve_kset(ks, [start], [diag], DV.Options(24, 1e-6, 16, first_step=True, max_iterations=60,
                                                            apply_precision="fp32"))
    assert np.max(np.abs(sol.eigenvalues - ref.eigenvalues)) < 1e-5
    single = DV.solve(op, start, diag, DV.Options(24, 1e-6, 16, first_step=True, max_iterations=60,
                                                   apply_precision="fp32"))
    assert np.max(np.abs(single.eigenvalues - ref.eigenvalues)) < 1e-5


def test_fp32_needs_a_compile_time_grid(ctx):
    import dataclasses
    w = dataclasses.replace(W.si8_k444(), dims_override=[48, 48, 48])
    op, pw = _op(w, 0, 4, ctx)
    op.precision = L.BG_PREC_FP32
    with pytest.raises(SolverError):
        op.apply_block(w.random_block(pw.npw, 4))


def test_scf_with_fp32_early_maps_reaches_the_fp64_energy(ctx):
    """Si2 Gamma SCF to 1e-8 Ha with FP32 applies in the maps whose ethr is at least
    1e-5 Ry: the converged energy equals the FP64 run's within 1e-7 Ha/atom, and the
    early maps did run in FP32."""
    from baandi_b200.scf import GpuScf, ScfOptions
    w = W.si2_gamma()
    plain = GpuScf(w, ctx, ScfOptions(threshold_ha=1e-8, smearing_ha=0.01)).run()
    tuned = GpuScf(w, ctx, ScfOptions(threshold_ha=1e-8, smearing_ha=0.01, fp32_ethr_ry=1e-5)).run()
    assert plain.converged and tuned.converged
    assert any(r.precision == "fp32" for r in tuned.records)
    assert tuned.records[-1].precision == "fp64"
    assert abs(tuned.energy_ha - plain.energy_ha) <= 1e-7 * w.natoms
    assert abs(tuned.iterations - plain.iterations) <= 2
