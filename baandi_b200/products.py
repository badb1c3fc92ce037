"""Complex products on the tcgen05 tensor cores with BF16x3 split operands
(bg_zgemm_bf16x3): the precision form of the projector and subspace products."""
from __future__ import annotations

from . import _lib as L
from .hamiltonian import SolverError, default_context

OPS = {"store": 0, "add": 1, "sub": 2}


def zgemm_bf16x3(a, b, c=None, adjoint_a=True, op="store", ctx=None):
    """C (op)= A^H B (adjoint_a) or A B for complex128 CUDA tensors in column-major
    storage, i.e. torch tensors whose transpose is contiguous: pass the matrices as
    `x.T` views of row-major (cols, rows) tensors, the layout of apply_block's device
    blocks.  Returns C (shape (m, n), column-major)."""
    import torch
    ctx = ctx or default_context()
    for t in (a, b):
        if t.dtype != torch.complex128 or not t.is_cuda or not t.T.is_contiguous():
            raise SolverError(L.BG_ESHAPE, "column-major complex128 CUDA matrices expected")
    if adjoint_a:
        k, m = a.shape
    else:
        m, k = a.shape
    if b.shape[0] != k:
        raise SolverError(L.BG_ESHAPE, "inner dimensions differ")
    n = b.shape[1]
    if c is None:
        c = torch.zeros((n, m), dtype=torch.complex128, device=a.device).T
    if c.shape != (m, n) or not c.T.is_contiguous():
        raise SolverError(L.BG_ESHAPE, "C must be a column-major (m, n) complex128 CUDA matrix")
    stream = torch.cuda.current_stream(a.device).cuda_stream
    rc = L.load().bg_zgemm_bf16x3(ctx.handle, 0 if adjoint_a else 1, m, n, k, a.data_ptr(), a.stride(1),
                                  b.data_ptr(), b.stride(1), c.data_ptr(), c.stride(1), OPS[op], stream)
    if rc != L.BG_OK:
        raise SolverError(rc, f"{L.CODE_NAMES.get(rc, rc)}: {L.last_error(ctx.handle)}")
    return c
