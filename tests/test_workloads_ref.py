"""The oracle's restatement of the benchmark cells (oracle/workloads_ref.py, which the
CPU baseline and the reference arm of bench.py use) describes the same systems as the
product's workload builders: atom positions, grid, plane-wave counts, k points and the
ionic potential agree."""
import numpy as np
import pytest

from baandi_b200 import systems as W
from oracle import workloads_ref as R


@pytest.mark.parametrize("name", ["si2", "si8", "si64", "al32"])
def test_cells_agree(name):
    w = W.WORKLOADS[name]()
    c = R.CELLS[name]()
    assert c.natoms == w.natoms and c.bands == w.bands
    pos = np.concatenate([np.atleast_2d(s.positions) for s in w.species])
    assert np.array_equal(c.positions, pos)
    assert c.dims() == list(w.dims())
    assert len(c.kpoints) == len(w.kpoints)
    for (ka, wa), (kb, wb) in zip(c.kpoints, w.kpoints):
        assert np.allclose(ka, kb, atol=0, rtol=0) and wa == wb
    k = c.kpoints[-1][0]
    assert c.basis(k).npw == w.plane_waves(k).npw


@pytest.mark.parametrize("name", ["si2", "al32"])
def test_potential_agrees(name):
    w = W.WORKLOADS[name]()
    c = R.CELLS[name]()
    a, b = c.ionic_potential(), w.ionic_potential()
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
