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


def main(argv=None) -> int:
    """One BF16x3 product of seeded random operands on cuda:0, repeated: wall time of each
    call (CUDA events; the call allocates its workspace) and the normwise error against the
    FP64 product.  kernels > 0 also runs the calls once more under torch.profiler's CUDA
    activity tracer and prints the device time of each kernel per call."""
    import argparse

    import torch
    p = argparse.ArgumentParser(description="BF16x3 tensor-core complex product")
    p.add_argument("--mode", choices=("tn", "nn"), default="tn", help="tn: C = A^H B; nn: C = A B")
    p.add_argument("--m", type=int, default=864)
    p.add_argument("--n", type=int, default=480)
    p.add_argument("--k", type=int, default=80725)
    p.add_argument("--reps", type=int, default=4)
    p.add_argument("--kernels", action="store_true")
    a = p.parse_args(argv)
    g = torch.Generator(device="cuda").manual_seed(1)

    def cm(r, c):
        return torch.randn((c, r), dtype=torch.complex128, device="cuda", generator=g).T

    adj = a.mode == "tn"
    A = cm(a.k, a.m) if adj else cm(a.m, a.k)
    B = cm(a.k, a.n)
    C = torch.zeros((a.n, a.m), dtype=torch.complex128, device="cuda").T
    for _ in range(a.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        zgemm_bf16x3(A, B, C, adjoint_a=adj)
        e1.record()
        torch.cuda.synchronize()
        print(f"{a.mode} {a.m}x{a.n}x{a.k}: {e0.elapsed_time(e1):.3f} ms per call")
    ref = (A.conj().T @ B) if adj else (A @ B)
    print(f"normwise relative error vs FP64: {float(torch.linalg.norm(C - ref) / torch.linalg.norm(ref)):.3e}")
    if a.kernels:
        import collections
        import json
        import os
        import tempfile

        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            for _ in range(a.reps):
                zgemm_bf16x3(A, B, C, adjoint_a=adj)
            torch.cuda.synchronize()
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "trace.json")
            prof.export_chrome_trace(path)
            with open(path) as f:
                events = json.load(f)["traceEvents"]
        total, count = collections.defaultdict(float), collections.Counter()
        for e in events:
            if e.get("cat") == "kernel":
                name = e["name"].replace("(anonymous namespace)::", "").replace("void ", "").split("(")[0]
                total[name] += e["dur"]
                count[name] += 1
        per_call = sum(total.values()) / a.reps
        for name, us in sorted(total.items(), key=lambda kv: -kv[1]):
            print(f"  {name[:60]:60s} {us / count[name] / 1e3:8.3f} ms x{count[name] // a.reps} per call")
        flops = 24.0 * a.m * a.n * a.k  # three real products of 2M x 2N x 2K on the stacked operands
        print(f"kernels {per_call / 1e3:.3f} ms per call: {flops / (per_call * 1e-6) / 1e12:.0f} TFLOP/s of BF16 "
              f"products, {8.0 * a.m * a.n * a.k / (per_call * 1e-6) / 1e12:.1f} TFLOP/s of complex FP64 work")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
