"""Learned preconditioner for the Davidson corrections (BG_PRECOND_LEARNED).

A per-G-vector network 5 -> 64 -> 64 -> 1 (GELU, BF16 parameters, FP32 accumulation)
outputs a log-multiplier on the TPA factor (crates/dft-solvers/src/lib.rs:176-207):
c_g = -tpa(t_g, s_j) exp(clamp(m(f), -3, 3)) r_g.  Its inputs per row g of band j are the
TPA ratio t_g/s_j, |k+G|^2/2, the band kinetic energy s_j, the Ritz value and the local
residual magnitude |r_g|/rms_j(r) (baandi_b200/csrc/learned.cuh).  A network whose last
layer is zero is TPA exactly, so training starts from TPA.

Training pairs come from the solver itself: Davidson states (Ritz vectors X, values,
H X) taken after 1, 2, 3, ... iterations on seeded displaced geometries, each band paired
with its ideal correction, the part of its Ritz vector outside the exact eigenspace it
converges to (exact eigenpairs of the dense H built by applying the operator to the unit
vectors; for cells too large for a dense H, the eigenpairs of a tight FP64 Davidson over
the tracked bands and a buffer of higher ones).  The loss scores each band's correction by its squared cosine with the ideal
one (the Davidson ignores the scale of a correction); the loss, its gradient and the Adam
step are device kernels (csrc/learned.cu).  The solver falls back to TPA when a solve
stalls (stats.fallbacks).
"""
from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import operands as O
from .hamiltonian import SolverError

NPARAMS = L.BG_LEARNED_PARAMS
N_IN, N_HID = 5, 64
OW1 = 0
OB1 = OW1 + N_HID * N_IN
OW2 = OB1 + N_HID
OB2 = OW2 + N_HID * N_HID
OW3 = OB2 + N_HID
OB3 = OW3 + N_HID


def init_params(seed: int = 0) -> np.ndarray:
    """Seeded start: hidden layers with variance-preserving normal weights, the output
    layer zero (the network starts as TPA)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, np.float32)
    p[OW1:OB1] = rng.normal(0.0, np.sqrt(1.0 / N_IN), N_HID * N_IN)
    p[OW2:OB2] = rng.normal(0.0, np.sqrt(1.0 / N_HID), N_HID * N_HID)
    return p


def to_bf16_bits(p: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 bit patterns, round to nearest even (the library's rounding)."""
    u = np.ascontiguousarray(p, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def install(ctx, params: np.ndarray) -> None:
    """Make `params` the context's network for BG_PRECOND_LEARNED."""
    p = np.ascontiguousarray(params, np.float32)
    if p.shape != (NPARAMS,):
        raise SolverError(L.BG_ESHAPE, f"learned parameters must be {NPARAMS} floats")
    rc = L.load().bg_learned_set(ctx.handle, p.ctypes.data_as(ctypes.c_void_p))
    if rc:
        raise SolverError(rc, L.last_error(ctx.handle))


def clear(ctx) -> None:
    L.load().bg_learned_clear(ctx.handle)


class Samples:
    """Device sample arrays (torch) for n (row, band) samples over ncols bands."""

    def __init__(self, n: int, ncols: int):
        import torch
        dev = "cuda"
        self.n, self.ncols = int(n), int(ncols)
        self.feats = torch.zeros((n, N_IN), dtype=torch.float32, device=dev)
        self.base = torch.zeros(n, dtype=torch.float32, device=dev)
        self.a = torch.zeros(n, dtype=torch.float32, device=dev)
        self.z = torch.zeros((n, 2), dtype=torch.float32, device=dev)
        self.col = torch.zeros(n, dtype=torch.int32, device=dev)
        self.ecol = torch.zeros(ncols, dtype=torch.float64, device=dev)
        self.used, self.cols_used = 0, 0

    def desc(self, n=None, ncols=None):
        return L.LearnedSamples(self.used if n is None else n, self.cols_used if ncols is None else ncols,
                                self.feats.data_ptr(), self.base.data_ptr(), self.a.data_ptr(), self.z.data_ptr(),
                                self.col.data_ptr(), self.ecol.data_ptr())

    def add_state(self, ctx, x, hx, target, kinetic, lam):
        """Append the samples of one Davidson state: x, hx, target (rows x cols numpy,
        real or complex), kinetic (rows), lam (cols)."""
        import torch
        rows, cols = x.shape
        if self.used + rows * cols > self.n or self.cols_used + cols > self.ncols:
            raise SolverError(L.BG_ESHAPE, "sample arrays full")
        cplx = np.iscomplexobj(x) or np.iscomplexobj(hx) or np.iscomplexobj(target)

        def dev(m):
            m = np.asarray(m)
            if cplx:
                m = np.ascontiguousarray(np.asarray(m, np.complex128).T)
                return torch.from_numpy(m.view(np.float64)).cuda()
            return torch.from_numpy(np.ascontiguousarray(np.asarray(m, np.float64).T)).cuda()

        tx, thx, te = dev(x), dev(hx), dev(target)
        tk = torch.from_numpy(np.ascontiguousarray(kinetic, np.float64)).cuda()
        tl = torch.from_numpy(np.ascontiguousarray(lam, np.float64)).cuda()
        d = self.desc(self.n, self.ncols)
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.load().bg_learned_samples_build(ctx.handle, rows, cols, 1 if cplx else 0, tx.data_ptr(), thx.data_ptr(),
                                               te.data_ptr(), tk.data_ptr(), tl.data_ptr(), self.cols_used,
                                               self.used, ctypes.byref(d), ctypes.c_void_p(stream))
        if rc:
            raise SolverError(rc, L.last_error(ctx.handle))
        torch.cuda.current_stream().synchronize()
        self.used += rows * cols
        self.cols_used += cols


class Trainer:
    """Adam on the FP32 master parameters; the network runs with their BF16 rounding."""

    def __init__(self, ctx, params: np.ndarray, lr: float = 3e-3):
        import torch
        self.ctx, self.lr, self.step_count = ctx, float(lr), 0
        self.master = torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
        self.m1 = torch.zeros_like(self.master)
        self.m2 = torch.zeros_like(self.master)
        self.grad = torch.zeros_like(self.master)
        self.net = torch.from_numpy(to_bf16_bits(params).view(np.int16)).cuda()
        self._work = None

    def _work_for(self, s: Samples):
        import torch
        need = 6 * s.cols_used + 1 + (s.used + 1) // 2
        if self._work is None or self._work.numel() < need:
            self._work = torch.zeros(need, dtype=torch.float64, device="cuda")
        return self._work

    def loss_grad(self, s: Samples, net=None) -> float:
        """Loss of the samples under `net` (device BF16 bits; default the current
        network) with its gradient left in self.grad."""
        import torch
        net = self.net if net is None else net
        d = s.desc()
        loss = ctypes.c_double(0.0)
        rc = L.load().bg_learned_loss_grad(self.ctx.handle, ctypes.byref(d), net.data_ptr(), self.grad.data_ptr(),
                                           self._work_for(s).data_ptr(), ctypes.byref(loss),
                                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc:
            raise SolverError(rc, L.last_error(self.ctx.handle))
        return loss.value

    def step(self, s: Samples) -> float:
        import torch
        loss = self.loss_grad(s)
        self.step_count += 1
        rc = L.load().bg_learned_adam(self.ctx.handle, self.master.data_ptr(), self.m1.data_ptr(),
                                      self.m2.data_ptr(), self.grad.data_ptr(), self.net.data_ptr(),
                                      self.step_count, ctypes.c_float(self.lr),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc:
            raise SolverError(rc, L.last_error(self.ctx.handle))
        return loss

    def params(self) -> np.ndarray:
        return self.master.cpu().numpy().copy()


# ------------------------------------------------------------------ training data
def displaced(w, seed: int, amp: float):
    """The workload with every atom moved by seeded uniform noise in [-amp, amp] Bohr."""
    rng = np.random.default_rng(seed)
    species = [O.Species(s.pseudo, np.atleast_2d(s.positions) + rng.uniform(-amp, amp, np.shape(np.atleast_2d(s.positions))))
               for s in w.species]
    return dataclasses.replace(w, species=species, seed=w.seed + 1000 + seed, _dims=None)


@dataclass
class Problem:
    """One geometry's operator with its exact spectrum (dense H)."""
    op: object
    kinetic: np.ndarray
    evals: np.ndarray
    evecs: np.ndarray
    start: np.ndarray
    bands: int


def exact_problem(w, ctx, bands: int, capacity: int) -> Problem:
    """Operator of the workload's first k point and the exact eigenpairs of its dense H
    (H applied to the unit vectors on the GPU, then a dense symmetric eigensolve)."""
    import torch
    from .hamiltonian import ComplexHamiltonian, RealGammaHamiltonian
    k = w.kpoints[0][0]
    pw = w.plane_waves(k)
    cls = RealGammaHamiltonian if w.gamma_real else ComplexHamiltonian
    op = cls.new_owned(pw, w.dims(), w.nonlocal_table(pw), capacity, ctx)
    op.set_owned_potential(w.ionic_potential(), 1)
    rows = op.global_len()
    dt = np.float64 if w.gamma_real else np.complex128
    h = np.zeros((rows, rows), dt, order="F")
    for c0 in range(0, rows, capacity):
        c1 = min(rows, c0 + capacity)
        e = np.zeros((rows, c1 - c0), dt, order="F")
        e[np.arange(c0, c1), np.arange(c1 - c0)] = 1.0
        h[:, c0:c1] = op.apply_block(e)
    ht = torch.from_numpy(np.ascontiguousarray(h)).cuda()
    ht = 0.5 * (ht + ht.conj().T)
    ev, vec = torch.linalg.eigh(ht)
    kin = op.kinetic_diagonal()
    start = w.random_block(rows, bands, seed_offset=7, real=w.gamma_real)
    return Problem(op, kin, ev.cpu().numpy(), vec.cpu().numpy(), start, bands)


def converged_problem(w, ctx, bands: int, capacity: int, k_index: int = 0, buffer: int = 16,
                      threshold: float = 1e-11, start_offset: int = 7) -> Problem:
    """Operator of the workload's k point `k_index` (ionic potential) with the eigenpairs of
    its lowest bands + buffer from the FP64 Davidson (smooth preconditioner) converged to
    `threshold` Ha, in place of a dense H's.  The buffer keeps every tracked band's
    eigenspace (and a cluster that reaches past the last band) inside the solved set."""
    from . import davidson as DV
    from .hamiltonian import ComplexHamiltonian, RealGammaHamiltonian
    k = w.kpoints[k_index][0]
    pw = w.plane_waves(k)
    real = w.gamma_real and pw.gamma
    cls = RealGammaHamiltonian if real else ComplexHamiltonian
    nb = bands + buffer
    op = cls.new_owned(pw, w.dims(), w.nonlocal_table(pw), max(capacity, 2 * nb), ctx)
    v = w.ionic_potential()
    op.set_owned_potential(v, 1)
    rows = op.global_len()
    x0 = w.random_block(rows, nb, seed_offset=3, real=real)
    o = DV.Options(nb, threshold, nb, first_step=True, max_iterations=400)
    sol = DV.solve(op, x0, op.diagonal_static() + float(np.mean(v)), o)
    if not bool(np.all(sol.converged)):
        raise RuntimeError("reference eigenpairs did not converge")
    kin = op.kinetic_diagonal()
    start = w.random_block(rows, bands, seed_offset=start_offset, real=real)
    return Problem(op, kin, np.asarray(sol.eigenvalues), np.asarray(sol.eigenvectors), start, bands)


def ideal_corrections(p: Problem, x: np.ndarray, tol: float = 1e-6) -> np.ndarray:
    """e_j = -(x_j - P_j x_j), P_j the projector on the exact eigenspace of eigenvalue j
    (eigenvalues within tol of it)."""
    out = np.empty_like(x)
    for j in range(x.shape[1]):
        cl = np.nonzero(np.abs(p.evals - p.evals[j]) <= tol)[0]
        u = p.evecs[:, cl]
        out[:, j] = -(x[:, j] - u @ (u.conj().T @ x[:, j]))
    return out


def davidson_states(p: Problem, iterations, threshold=1e-10):
    """(x, hx, lam) after each iteration count in `iterations` (TPA corrections)."""
    from . import davidson as DV
    out = []
    for it in iterations:
        o = DV.Options(p.bands, threshold, p.bands, first_step=True, max_iterations=it, preconditioner="tpa")
        sol = DV.solve(p.op, p.start, p.kinetic, o)
        x = sol.eigenvectors
        out.append((x, p.op.apply_block(x), sol.eigenvalues))
    return out


TRAIN_ITERATIONS = (1, 2, 3, 4, 5, 6, 8, 10, 13, 16, 20, 25, 30)


def build_samples(ctx, problems, iterations=TRAIN_ITERATIONS, min_error=1e-12, bands_per_state=None,
                  seed=0) -> Samples:
    """Samples of every problem's Davidson states; bands already exact (|e|^2 below
    min_error) are left out.  problems: any iterable (a generator frees each problem's
    operator once its states are taken).  iterations: one tuple for every problem, or a
    callable problem index -> tuple.  bands_per_state: keep a seeded random subset of that many of
    each state's remaining bands (None: all)."""
    states = []
    rng = np.random.default_rng(seed)
    for i, p in enumerate(problems):
        its = iterations(i) if callable(iterations) else iterations
        for x, hx, lam in davidson_states(p, its):
            e = ideal_corrections(p, x)
            keep = np.nonzero(np.sum(np.abs(e) ** 2, axis=0) > min_error)[0]
            if bands_per_state is not None and len(keep) > bands_per_state:
                keep = np.sort(rng.choice(keep, bands_per_state, replace=False))
            if len(keep):
                states.append((p.kinetic, x[:, keep], hx[:, keep], e[:, keep], lam[keep]))
    n = sum(x.shape[0] * x.shape[1] for _, x, _, _, _ in states)
    ncols = sum(x.shape[1] for _, x, _, _, _ in states)
    s = Samples(n, ncols)
    for kin, x, hx, e, lam in states:
        s.add_state(ctx, x, hx, e, kin, lam)
    return s


def train(ctx, samples: Samples, steps: int = 300, lr: float = 3e-3, seed: int = 0, params=None):
    """Adam from init_params(seed) (or `params`); returns (params, losses)."""
    t = Trainer(ctx, init_params(seed) if params is None else params, lr)
    losses = [t.step(samples) for _ in range(steps)]
    return t.params(), losses
