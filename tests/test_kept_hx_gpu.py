"""Kept H X (crates/dft-engine/src/refscf/kept_hx.rs:98-160): the batched Davidson started
from a supplied H of its start block (bg_kset_davidson_solve_hx) against the same solve
that applies H itself, the H X it returns against a fresh apply of its eigenvectors, and
the SCF with kept H X against the SCF without (the same energy, one start apply fewer
per map after the first)."""
import dataclasses

import numpy as np
import pytest

from baandi_b200 import davidson as DV
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian, KPointSet
from baandi_b200.scf import GpuScf, ScfOptions

pytestmark = pytest.mark.gpu


def _si8_set(ctx, kpts=(0, 5)):
    import torch
    w = W.si8_k444()
    v = w.ionic_potential()
    ops, starts, diags = [], [], []
    for i, kk in enumerate(kpts):
        k = w.kpoints[kk][0]
        pw = w.plane_waves(k)
        op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), 48, ctx)
        op.set_owned_potential(v, 1)
        ops.append(op)
        x = w.random_block(pw.npw, 24, seed_offset=40 + i)
        starts.append(torch.from_numpy(np.ascontiguousarray(x.T)).cuda())
        diags.append(torch.from_numpy(op.diagonal_static() + v.mean()).cuda())
    return KPointSet(ops, ctx), ops, starts, diags


def test_start_hx_and_returned_hx(ctx):
    import torch
    ks, ops, starts, diags = _si8_set(ctx)
    opts = DV.Options(24, 1e-10, 16, first_step=True, max_iterations=60)
    ref = DV.solve_kset(ks, starts, diags, opts)
    torch.cuda.synchronize()
    hx0 = [op.apply_block(x) for op, x in zip(ops, starts)]   # on the operators' own streams
    torch.cuda.synchronize()
    kept = DV.solve_kset(ks, starts, diags, opts, start_hx=hx0, want_hx=True)
    for op, a, b in zip(ops, ref, kept):
        assert a.iterations == b.iterations
        assert np.max(np.abs(a.eigenvalues - b.eigenvalues)) < 1e-12
        assert b.h_columns == a.h_columns - 24          # the start block was not applied
        fresh = op.apply_block(b.eigenvectors)
        torch.cuda.synchronize()
        rel = float(torch.linalg.norm(b.hx - fresh) / torch.linalg.norm(fresh))
        assert rel < 1e-12


def test_kept_hx_rejects_host_blocks(ctx):
    from baandi_b200.hamiltonian import SolverError
    ks, ops, starts, diags = _si8_set(ctx, kpts=(0,))
    opts = DV.Options(24, 1e-8, 16, first_step=True, max_iterations=5)
    with pytest.raises(SolverError):
        DV.solve_kset(ks, [starts[0].cpu().numpy().T.copy()], [diags[0].cpu().numpy()], opts, want_hx=True)


def test_scf_with_kept_hx_matches_fresh_applies(ctx):
    """Si8 on two k points to 1e-8 Ha (Fermi-Dirac 0.01 Ha): the same energy within
    1e-9 Ha/atom and the same maps; every map after the first applies H to one start
    block fewer per k point."""
    w = W.si8_k444()
    ks = w.kpoints[:2]
    total = sum(x for _, x in ks)
    w = dataclasses.replace(w, kpoints=[(k, x / total) for k, x in ks])
    o = dict(threshold_ha=1e-8, smearing_ha=0.01)
    fresh = GpuScf(w, ctx, ScfOptions(**o, kept_hx=False)).run()
    kept = GpuScf(w, ctx, ScfOptions(**o)).run()
    assert fresh.converged and kept.converged
    assert abs(kept.energy_ha - fresh.energy_ha) <= 1e-9 * w.natoms
    assert len(kept.records) == len(fresh.records)
    saved = sum(a.h_columns - b.h_columns for a, b in zip(fresh.records, kept.records))
    assert saved >= (len(kept.records) - 2) * w.bands * len(w.kpoints)
