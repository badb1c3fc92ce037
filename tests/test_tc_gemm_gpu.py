"""BF16x3 complex products on the tcgen05 tensor cores (bg_zgemm_bf16x3) against the
FP64 product, at the shapes of the Si216 cell's projector products (80,725 plane waves,
864 projectors, 480 columns) and Davidson subspace products (basis of 960 columns), and
at small ragged shapes.  Bound: every entry within 1e-4 of sum_r |a_r| |b_r| (the BF16x3
split keeps about 16 significant bits per term, then FP32 accumulation), and the
normwise relative error below 1e-4 (random operands cancel, so at depth 80,725 the
FP32 accumulation shows at a few 1e-5 of the result's norm)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand(shape, seed, dev):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    re = torch.randn(shape[1], shape[0], generator=g, dtype=torch.float64)
    im = torch.randn(shape[1], shape[0], generator=g, dtype=torch.float64)
    return torch.complex(re, im).to(dev).T   # column-major (rows, cols)


@pytest.mark.parametrize("adj,m,n,k", [
    (True, 37, 23, 1000), (True, 5, 1, 7), (True, 128, 128, 64), (True, 864, 480, 80725), (True, 960, 480, 80725),
    (False, 1000, 37, 23), (False, 131, 3, 5), (False, 80725, 480, 960), (False, 80725, 480, 864),
])
def test_bf16x3_product_matches_fp64(ctx, adj, m, n, k):
    import torch
    from baandi_b200.products import zgemm_bf16x3
    dev = torch.device("cuda")
    a = _rand((k, m) if adj else (m, k), 11 + m, dev)
    b = _rand((k, n), 17 + n, dev)
    c = zgemm_bf16x3(a, b, adjoint_a=adj, ctx=ctx)
    ref = (a.conj().T @ b) if adj else (a @ b)
    bound = ((a.abs().T @ b.abs()) if adj else (a.abs() @ b.abs()))
    err = (c - ref).abs()
    assert bool(torch.isfinite(c).all())
    assert float((err / bound).max()) <= 1e-4
    assert float(torch.linalg.norm(c - ref) / torch.linalg.norm(ref)) <= 1e-4


def test_bf16x3_accumulate_modes(ctx):
    import torch
    from baandi_b200.products import zgemm_bf16x3
    dev = torch.device("cuda")
    a = _rand((300, 70), 3, dev)
    b = _rand((300, 40), 4, dev)
    base = _rand((70, 40), 5, dev)
    ref = a.conj().T @ b
    c = base.clone()
    zgemm_bf16x3(a, b, c, op="add", ctx=ctx)
    assert float(torch.linalg.norm(c - (base + ref)) / torch.linalg.norm(ref)) <= 3e-5
    c = base.clone()
    zgemm_bf16x3(a, b, c, op="sub", ctx=ctx)
    assert float(torch.linalg.norm(c - (base - ref)) / torch.linalg.norm(ref)) <= 3e-5
