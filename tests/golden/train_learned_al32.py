"""Train the learned preconditioner on seeded Al32 geometries and write the network.

    python tests/golden/train_learned_al32.py [--geometries 200] [--steps 600] [--scf]

Needs one GPU.  Geometries: the Al32 cell (fcc 2x2x2 conventional, a = 15.30 Bohr, 30 Ry,
60^3 grid, 2x2x2 k mesh, 64 bands) with every atom displaced by seeded uniform noise of
+-0.08 Bohr, seeds TRAIN_BASE + 0 .. TRAIN_BASE + geometries - 1.  Geometry g contributes
its k point g % 8: the eigenpairs of the lowest 64 + 16 bands from a tight FP64 Davidson
(REF_THRESHOLD Ha) stand in for the exact spectrum, and two TPA Davidson states of it
(after its[g % n] and its[(g + n // 2) % n] iterations; its = TRAIN_ITERATIONS, n = 13,
unless --iterations names others) give 8 seeded bands each with |e|^2 above MIN_ERROR,
paired with their ideal corrections e.  600 full-batch Adam steps from TPA (zero output
layer).  The held-out geometry (seed HELD_OUT, k points 0 and 5) scores the correction
loss before and after; then the batched solver on all 8 of its k points
counts H columns for TPA and the trained network (occupied bands to 1e-8 Ha), and with
--scf both SCFs (Fermi-Dirac 0.01 Ha, to 1e-6 Ha/atom) are timed.

Writes tests/golden/learned_al32.npz: params (FP32 master), the seeds, the loss trace
and the held-out figures.
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from baandi_b200 import davidson as DV  # noqa: E402
from baandi_b200 import learned as LP  # noqa: E402
from baandi_b200 import systems as W  # noqa: E402

TRAIN_BASE = 5000
HELD_OUT = 4999
BANDS, BUFFER, CAPACITY = 64, 16, 160
HELD_K = (0, 5)
REF_THRESHOLD = 1e-12
MIN_ERROR = 1e-10


def held_out_columns(ctx, params, starts=(7, 11)):
    """H columns of the batched solver over every k point of the held-out geometry, TPA
    against the network (occupied bands to 1e-8 Ha), and the largest occupied eigenvalue
    difference between the two."""
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
    LP.install(ctx, params)
    cols, dev = {"tpa": 0, "learned": 0}, 0.0
    for so in starts:
        x0 = [torch.from_numpy(np.ascontiguousarray(w.random_block(op.global_len(), BANDS, seed_offset=so).T)).cuda()
              for op in ops]
        vals = {}
        for name in cols:
            o = DV.Options(BANDS, 1e-8, w.occupied, first_step=True, max_iterations=200, preconditioner=name)
            sols = DV.solve_kset(ks, x0, kins, o)
            cols[name] += sum(s.h_columns for s in sols)
            vals[name] = [s.eigenvalues[:w.occupied] for s in sols]
        dev = max(dev, max(float(np.max(np.abs(a - b))) for a, b in zip(vals["tpa"], vals["learned"])))
    return cols, dev


def scf_times(ctx, params):
    from baandi_b200.scf import GpuScf, ScfOptions
    w = W.al32_k222(HELD_OUT)
    LP.install(ctx, params)
    out = {}
    for name in ("tpa", "learned"):
        o = ScfOptions(threshold_ha=1e-6 * w.natoms, smearing_ha=0.01, thomas_fermi=True, preconditioner=name)
        s = GpuScf(w, ctx, o)
        s.warm_up()
        r = s.run()
        out[name] = (r.seconds, r.iterations, sum(m.h_columns for m in r.records), r.energy_ha)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--geometries", type=int, default=200)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--scf", action="store_true")
    ap.add_argument("--iterations", default=None,
                    help="comma-separated Davidson iteration counts the states are drawn from "
                         "(default: TRAIN_ITERATIONS)")
    ap.add_argument("--out", default=os.path.join(HERE, "learned_al32.npz"))
    a = ap.parse_args()
    from baandi_b200.hamiltonian import default_context
    ctx = default_context()
    its = LP.TRAIN_ITERATIONS if a.iterations is None else tuple(int(x) for x in a.iterations.split(","))
    half = len(its) // 2

    def problems():
        for g in range(a.geometries):
            w = W.al32_k222(TRAIN_BASE + g)
            yield LP.converged_problem(w, ctx, BANDS, CAPACITY, k_index=g % len(w.kpoints), buffer=BUFFER,
                                       threshold=REF_THRESHOLD)

    t0 = time.perf_counter()
    samples = LP.build_samples(ctx, problems(), iterations=lambda g: (its[g % len(its)], its[(g + half) % len(its)]),
                               min_error=MIN_ERROR, bands_per_state=8, seed=1)
    t_data = time.perf_counter() - t0
    hw = W.al32_k222(HELD_OUT)
    held = LP.build_samples(ctx, (LP.converged_problem(hw, ctx, BANDS, CAPACITY, k_index=k, buffer=BUFFER,
                                                       threshold=REF_THRESHOLD)
                                  for k in HELD_K), iterations=(1, 3, 8, 20), min_error=MIN_ERROR)
    t = LP.Trainer(ctx, LP.init_params(0), lr=a.lr)
    before = t.loss_grad(held)
    trace = []
    t1 = time.perf_counter()
    for i in range(a.steps):
        loss = t.step(samples)
        if i % 10 == 0 or i == a.steps - 1:
            trace.append((i, loss))
    t_train = time.perf_counter() - t1
    params = t.params()
    after = t.loss_grad(held)
    print(f"samples {samples.used} over {samples.cols_used} bands, data {t_data:.1f} s, "
          f"training {t_train:.1f} s; train loss {trace[0][1]:.4f} -> {trace[-1][1]:.4f}; "
          f"held-out loss {before:.4f} -> {after:.4f}", flush=True)
    cols, dev = held_out_columns(ctx, params)
    print(f"held-out H columns: tpa {cols['tpa']} learned {cols['learned']} "
          f"({100.0 * (cols['learned'] / cols['tpa'] - 1.0):+.1f} %), occupied eigenvalues within {dev:.1e} Ha",
          flush=True)
    extra = {}
    if a.scf:
        st = scf_times(ctx, params)
        for name, (sec, maps, hcols, e) in st.items():
            print(f"held-out SCF {name}: {sec:.3f} s, {maps} maps, {hcols} H columns, E = {e:.9f} Ha", flush=True)
        extra = {"scf_" + k: np.array(v) for k, v in st.items()}
    np.savez(a.out, params=params.astype(np.float32), train_base=TRAIN_BASE, geometries=a.geometries,
             held_out=HELD_OUT, steps=a.steps, lr=a.lr, trace=np.array(trace), held_before=before,
             held_after=after, cols_tpa=cols["tpa"], cols_learned=cols["learned"], samples=samples.used, **extra)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
