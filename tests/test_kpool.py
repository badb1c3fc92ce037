"""k points split over ranks (baandi_b200.kpool, the reference's k-point pools with one
rank per pool: crates/dft-engine/src/refscf/k_pool.rs:76-330), on CPU: the block layout,
the fixed-order sum, and two gloo ranks each running the oracle SCF on its own k points
(Si2, 2x2x2 Monkhorst-Pack, 8 k points, Fermi-Dirac 0.01 Ha) with the pool's eigenvalue
gather and density sum, against the single-process SCF: the same maps, energies within
1e-12 Ha, and the same energy, eigenvalues and density bits on both ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from baandi_b200.kpool import KPool, block_counts, block_first, tree_sum


def test_block_layout_follows_the_reference():
    # crates/dft-mpi/src/lib.rs:207-223: the first total % parts blocks one larger
    assert block_counts(8, 3) == [3, 3, 2]
    assert block_first([3, 3, 2]) == [0, 3, 6]
    assert block_counts(36, 8) == [5, 5, 5, 5, 4, 4, 4, 4]
    p = KPool(8, rank=1, world=3)
    assert list(p.local) == [3, 4, 5]
    assert [p.owner(k) for k in range(8)] == [0, 0, 0, 1, 1, 1, 2, 2]
    with pytest.raises(ValueError):
        KPool(2, rank=0, world=3)


def test_tree_sum_order_is_fixed():
    rng = np.random.default_rng(3)
    parts = [rng.standard_normal(1000) * 10.0 ** rng.integers(-8, 8) for _ in range(5)]
    expect = ((parts[0] + parts[1]) + (parts[2] + parts[3])) + parts[4]
    assert np.array_equal(tree_sum(parts), expect)


def test_single_rank_pool_is_the_identity():
    p = KPool(4)
    vals = [np.arange(3.0) + k for k in range(4)]
    assert p.gather_eigenvalues(vals) is not None and all(
        np.array_equal(a, b) for a, b in zip(p.gather_eigenvalues(vals), vals))
    x = np.ones(7)
    assert p.sum_partials(x) is x


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    from oracle import setup_ref as S
    from oracle import workloads_ref as WR
    c = WR.si2()
    ks = S.reduce_time_reversal(S.monkhorst_pack((2, 2, 2)))
    starts = [c.random_block(S.basis_at_k(c.cell, c.ecut_ha, k).npw, c.bands, seed_offset=100 + i)
              for i, (k, _) in enumerate(ks)]
    return c, ks, starts


def _run(pool, kept=True):
    from oracle import scf_ref
    c, ks, starts = _case()
    local = pool.local if pool is not None else range(len(ks))
    return scf_ref.run(c.rows, c.species(), c.ecut_ha, c.dims(), ks, False, c.bands, c.ionic_potential(),
                       [starts[i] for i in local], 0.0, threshold_ha=1e-9, smearing_ha=0.01, kept_hx=kept,
                       pool=pool)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, ks, _ = _case()
        pool = KPool(len(ks), rank, world, dist)
        r = _run(pool)
        q.put((rank, r.converged, r.iterations, r.energy, r.energies, [np.asarray(v) for v in r.eigenvalues]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_split_the_k_points():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict()
    for _ in range(world):
        rank, *rest = q.get(timeout=280)
        got[rank] = rest
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = _run(None)
    conv0, its0, e0, energies0, vals0 = got[0]
    conv1, its1, e1, energies1, vals1 = got[1]
    # every rank holds the same bits: the density sum has one order
    assert e0 == e1 and energies0 == energies1
    assert all(np.array_equal(a, b) for a, b in zip(vals0, vals1))
    # and the split map is the single-process map to rounding
    assert conv0 and single.converged and its0 == single.iterations
    assert abs(e0 - single.energy) < 1e-12
    assert max(abs(a - b) for a, b in zip(energies0, single.energies)) < 1e-11
    assert max(float(np.max(np.abs(a - b))) for a, b in zip(vals0, single.eigenvalues)) < 1e-10
