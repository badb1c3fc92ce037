"""The learned preconditioner trained on 200 seeded Al32 geometries (tests/golden/
learned_al32.npz, written by tests/golden/train_learned_al32.py) on the held-out geometry:
the network lowers the correction loss against TPA's; the batched solver with it reaches
TPA's occupied eigenvalues on all 8 k points; the SCF with it reaches the TPA SCF's energy.
It needs more H columns than TPA on this cell (the recorded figures below), so the solver
runs are checked for their results, not for a gain."""
import os

import numpy as np
import pytest

from baandi_b200 import davidson as DV
from baandi_b200 import learned as LP
from baandi_b200 import systems as W

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "learned_al32.npz")
HELD_OUT = 4999
BANDS, CAPACITY = 64, 160


def _fixture():
    return np.load(FIXTURE)


def test_fixture_records_the_training():
    """CPU: the committed network and the figures measured when it was made."""
    f = _fixture()
    assert int(f["geometries"]) == 200 and int(f["steps"]) == 600 and int(f["held_out"]) == HELD_OUT
    p = f["params"]
    assert p.shape == (LP.NPARAMS,) and np.all(np.isfinite(p))
    assert float(f["held_after"]) < 0.85 * float(f["held_before"])
    trace = f["trace"]
    assert trace[-1, 1] < trace[0, 1]
    # recorded: the network needs more H columns than TPA on the held-out geometry
    assert int(f["cols_learned"]) > int(f["cols_tpa"])


@pytest.mark.gpu
def test_held_out_loss_falls(ctx):
    """k point 0 of the held-out geometry, Davidson states after 1, 3, 8 and 20 TPA
    iterations: the trained network's correction loss is below TPA's (the start network)."""
    w = W.al32_k222(HELD_OUT)
    p = LP.converged_problem(w, ctx, BANDS, CAPACITY, k_index=0, threshold=1e-12)
    s = LP.build_samples(ctx, [p], iterations=(1, 3, 8, 20), min_error=1e-10)
    t = LP.Trainer(ctx, LP.init_params(0))
    tpa = t.loss_grad(s)
    trained = LP.Trainer(ctx, _fixture()["params"])
    loss = trained.loss_grad(s)
    print(f"held-out loss at k 0: tpa {tpa:.4f} trained {loss:.4f}")
    assert loss < 0.9 * tpa


@pytest.mark.gpu
def test_batched_solver_reaches_tpa_eigenvalues(ctx):
    """All 8 k points of the held-out geometry, one seeded start, occupied bands (48) to
    1e-8 Ha: the network's solve converges to TPA's occupied eigenvalues within 1e-7 Ha."""
    import torch
    from baandi_b200.hamiltonian import ComplexHamiltonian, KPointSet
    w = W.al32_k222(HELD_OUT)
    v = w.ionic_potential()
    ops, kins = [], []
    for k, _ in w.kpoints:
        pw = w.plane_waves(k)
        op = ComplexHamiltonian.new_owned(pw, w.dims(), w.nonlocal_table(pw), CAPACITY, ctx)
        op.set_owned_potential(v, 1)
        ops.append(op)
        kins.append(torch.from_numpy(op.kinetic_diagonal()).cuda())
    ks = KPointSet(ops, ctx)
    LP.install(ctx, _fixture()["params"])
    x0 = [torch.from_numpy(np.ascontiguousarray(w.random_block(op.global_len(), BANDS, seed_offset=7).T)).cuda()
          for op in ops]
    res = {}
    for name in ("tpa", "learned"):
        o = DV.Options(BANDS, 1e-8, w.occupied, first_step=True, max_iterations=200, preconditioner=name)
        res[name] = DV.solve_kset(ks, x0, kins, o)
    for a, b in zip(res["tpa"], res["learned"]):
        assert np.all(a.converged[:w.occupied]) and np.all(b.converged[:w.occupied])
        assert np.max(np.abs(a.eigenvalues[:w.occupied] - b.eigenvalues[:w.occupied])) < 1e-7
    cols = {n: sum(s.h_columns for s in r) for n, r in res.items()}
    print(f"held-out H columns: tpa {cols['tpa']} learned {cols['learned']}; "
          f"fallbacks {sum(s.fallbacks for s in res['learned'])}")


@pytest.mark.gpu
def test_scf_with_the_network_reaches_the_tpa_energy(ctx):
    """The held-out geometry's SCF (Fermi-Dirac 0.01 Ha, Thomas-Fermi mixing) to 1e-8
    Ha/atom with TPA and with the network, each map's Davidson allowed 80 iterations (the
    network's solves need more than the default 20 to reach their threshold): energies
    within 1e-6 Ha/atom."""
    from baandi_b200.scf import GpuScf, ScfOptions
    w = W.al32_k222(HELD_OUT)
    LP.install(ctx, _fixture()["params"])
    e = {}
    for name in ("tpa", "learned"):
        o = ScfOptions(threshold_ha=1e-8 * w.natoms, smearing_ha=0.01, thomas_fermi=True, preconditioner=name,
                       davidson_max_iterations=80)
        r = GpuScf(w, ctx, o).run()
        assert r.converged
        e[name] = r.energy_ha
        print(f"SCF {name}: {r.iterations} maps, {sum(m.h_columns for m in r.records)} H columns, "
              f"{r.seconds:.3f} s, E = {r.energy_ha:.9f} Ha, Davidson iterations per map "
              f"{[m.davidson_iterations for m in r.records]}")
    assert abs(e["learned"] - e["tpa"]) <= 1e-6 * w.natoms
