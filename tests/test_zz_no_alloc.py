"""bg_local_apply_noalloc: the local + kinetic apply for callers that cannot allocate
device memory (their memory belongs to another runtime's pool, or allocation is
forbidden after start-up because cudaMalloc/cudaFree can synchronise the device).

The entry point takes only caller-owned buffers and keeps its intermediates in the
library's fixed 32 MiB device scratch.  Its result must match the oracle's local +
kinetic apply (the C++ FP64 restatement with no projectors) and the operator entry
point (bg_op_apply_block of an operator without projectors) within the FP64 tolerance
of the parity tests, on two calls in a row (the scratch keeps the previous call's
contents, so the second call checks that nothing stale leaks through).  A grid index
out of range is skipped and reported, never accessed.  This file is collected last on
purpose."""
import ctypes

import numpy as np
import pytest

from baandi_b200 import _lib
from baandi_b200 import operands as O
from baandi_b200 import systems as W
from baandi_b200.hamiltonian import ComplexHamiltonian
from oracle import oracle as OR
from tests.helpers import oracle_inputs
from oracle import setup_ref as S

TOL = 1e-12

pytestmark = pytest.mark.gpu


def _noalloc(dims, idx, v, kin, x, y, stream):
    lib = _lib.load()
    d = (ctypes.c_int32 * 3)(*dims)
    cols = x.shape[0]
    return lib.bg_local_apply_noalloc(ctypes.cast(d, ctypes.c_void_p), idx.numel(), idx.data_ptr(), v.data_ptr(),
                                      kin.data_ptr(), x.data_ptr(), y.data_ptr(), cols, stream)


@pytest.mark.parametrize("name,kidx,cols", [("si8", 5, 8), ("si2", 0, 12)])
def test_noalloc_matches_operator_twice(ctx, name, kidx, cols):
    import torch
    w = W.WORKLOADS[name]()
    k = w.kpoints[kidx][0]
    dims = w.dims()
    pw = w.plane_waves(k)
    op = ComplexHamiltonian.new_owned(pw, dims, None, cols, ctx)
    v = w.ionic_potential()
    op.set_owned_potential(v, 1)
    dev = torch.device("cuda")
    idx = torch.from_numpy(O.fft_index(pw.miller, dims, pw.gamma).astype(np.int32)).to(dev)
    vd = torch.from_numpy(np.ascontiguousarray(v).reshape(-1)).to(dev)
    kin = torch.from_numpy(0.5 * pw.kpg2).to(dev)
    stream = torch.cuda.current_stream()
    for call, (ncols, seed) in enumerate([(cols, 11), (cols - 3, 12)]):
        x = torch.from_numpy(np.ascontiguousarray(w.random_block(pw.npw, ncols, seed_offset=seed).T)).to(dev)
        y = torch.full_like(x, complex(float("nan"), float("nan")))
        rc = _noalloc(dims, idx, vd, kin, x, y, stream.cuda_stream)
        assert rc == _lib.BG_OK, _lib.last_error(None)
        torch.cuda.synchronize()
        ref = op.apply_block(x)
        op.sync()
        a, b = y.cpu().numpy().T, ref.cpu().numpy().T
        err = float(np.max(np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)))
        assert err <= TOL, f"call {call}: relative error {err:.3e} against the operator"
        _, ob, _ = oracle_inputs(w, k)
        oref = OR.apply_complex(dims, S.fft_flat(S.g_to_fft(ob, dims), dims), v, 0.5 * ob.kpg2, None,
                                x.cpu().numpy().T)
        err = float(np.max(np.linalg.norm(a - oref, axis=0) / np.linalg.norm(oref, axis=0)))
        assert err <= TOL, f"call {call}: relative error {err:.3e} against the oracle"


def test_noalloc_skips_and_reports_bad_index(ctx):
    """One fft_index entry past the grid: that row is skipped (never accessed), the call
    reports BG_ESHAPE, and every other row still equals the oracle's answer (the bad
    row's coefficient is zero, so it contributes nothing to the others)."""
    import torch
    w = W.WORKLOADS["si2"]()
    dims = w.dims()
    pw = w.plane_waves()
    _, ob, _ = oracle_inputs(w, (0.0, 0.0, 0.0))
    v = w.ionic_potential()
    dev = torch.device("cuda")
    idx_h = O.fft_index(pw.miller, dims, pw.gamma).astype(np.int32)
    bad = 17
    idx_h[bad] = int(np.prod(dims)) + 5
    x_h = w.random_block(pw.npw, 3, seed_offset=21)
    x_h[bad, :] = 0.0
    idx = torch.from_numpy(idx_h).to(dev)
    vd = torch.from_numpy(np.ascontiguousarray(v).reshape(-1)).to(dev)
    kin = torch.from_numpy(0.5 * pw.kpg2).to(dev)
    x = torch.from_numpy(np.ascontiguousarray(x_h.T)).to(dev)
    y = torch.zeros_like(x)
    rc = _noalloc(dims, idx, vd, kin, x, y, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.BG_ESHAPE
    assert "outside" in _lib.last_error(None)
    oref = OR.apply_complex(dims, S.fft_flat(S.g_to_fft(ob, dims), dims), v, 0.5 * ob.kpg2, None, x_h)
    a = y.cpu().numpy().T
    keep = np.ones(pw.npw, bool)
    keep[bad] = False
    err = float(np.max(np.linalg.norm(a[keep] - oref[keep], axis=0) / np.linalg.norm(oref[keep], axis=0)))
    assert err <= TOL
    # a non-finite coefficient is reported as well
    x_h[3, 1] = np.nan
    x = torch.from_numpy(np.ascontiguousarray(x_h.T)).to(dev)
    idx_h[bad] = O.fft_index(pw.miller, dims, pw.gamma).astype(np.int32)[bad]
    rc = _noalloc(dims, torch.from_numpy(idx_h).to(dev), vd, kin, x, y, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.BG_ENONFINITE


def test_noalloc_rejects_oversize(ctx):
    import torch
    dims = [45, 45, 45]
    dev = torch.device("cuda")
    idx = torch.zeros(10, dtype=torch.int32, device=dev)
    v = torch.zeros(45 ** 3, dtype=torch.float64, device=dev)
    kin = torch.zeros(10, dtype=torch.float64, device=dev)
    x = torch.zeros((24, 10), dtype=torch.complex128, device=dev)  # 24 * 45^3 > 2,097,152
    y = torch.zeros_like(x)
    rc = _noalloc(dims, idx, v, kin, x, y, 0)
    assert rc == _lib.BG_ESHAPE
    assert "32 MiB" in _lib.last_error(None)
