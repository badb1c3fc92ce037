"""The library's operand builders (bg_setup_*) against the oracle's restatement of the
reference setup: Miller lists and grid indices bit for bit, projector tables and form
factors to rounding (CPU only)."""
import numpy as np
import pytest

from baandi_b200 import operands as P
from baandi_b200 import systems as W
from oracle import setup_ref as S


@pytest.mark.parametrize("name", ["si2", "si8", "al32", "si64"])
def test_sphere_grid_and_projectors(name):
    w = W.WORKLOADS[name]()
    cell = S.Cell(w.rows)
    assert abs(w.volume - cell.volume) <= 1e-12 * cell.volume
    dims, req = P.grid(w.rows, w.ecut_ha)
    odims, oreq = S.grid_dims(cell, w.ecut_ha)
    assert dims == odims and req == oreq
    for kidx in sorted({0, len(w.kpoints) // 2, len(w.kpoints) - 1}):
        k = w.kpoints[kidx][0]
        pw = w.plane_waves(k)
        b = S.basis_at_k(cell, w.ecut_ha, k)
        assert np.array_equal(pw.miller, b.miller)
        assert np.array_equal(pw.kpg2, b.kpg2)
        d = w.dims()
        assert np.array_equal(P.fft_index(pw.miller, d, pw.gamma), S.fft_flat(S.g_to_fft(b, d), d))
        if name in ("si2", "si8"):
            nl = w.nonlocal_table(pw)
            p = w.species[0].pseudo
            ps = S.Pseudo(p.z, p.r, p.rab, p.local, [S.Projector(l, u) for l, u in zip(p.l, p.beta)], p.dij)
            onl = S.nonlocal_table(b, cell.volume, [S.Species(ps, w.species[0].positions)])
            assert np.max(np.abs(nl.table - onl.table)) <= 1e-13 * np.max(np.abs(onl.table))
            assert list(nl.channels) == list(onl.channels)
            assert np.array_equal(np.concatenate(onl.couplings), nl.couplings)


def test_half_sphere_and_form_factor():
    w = W.si2_gamma()
    pw = w.plane_waves()
    plus, minus = P.half_sphere(pw.miller)
    b = S.basis_at_k(S.Cell(w.rows), w.ecut_ha)
    oplus, ominus, _ = S.half_sphere(b)
    assert np.array_equal(plus, oplus) and np.array_equal(minus, ominus)
    p = w.species[0].pseudo
    ps = S.Pseudo(p.z, p.r, p.rab, p.local, [], p.dij)
    g = np.array([0.0, 0.3, 1.0, 2.5, 7.0])
    ours = P.local_form_factor(w.species[0], w.volume, g)
    ref = S.local_form_factor(ps, w.volume, g)
    assert np.max(np.abs(ours - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_kpoint_meshes():
    assert len(W.si8_k444().kpoints) == 36
    assert len(W.al32_k222().kpoints) == 8
    ks = W.si8_k444().kpoints
    oks = S.reduce_time_reversal(S.monkhorst_pack((4, 4, 4)))
    assert [tuple(k) for k, _ in ks] == [tuple(k) for k, _ in oks]
    assert np.allclose([w for _, w in ks], [w for _, w in oks], rtol=0, atol=1e-15)


def test_operand_errors():
    with pytest.raises(Exception):
        P.volume(np.zeros((3, 3)))
    with pytest.raises(Exception):
        P.plane_waves(np.eye(3) * 10.0, -1.0)
    with pytest.raises(Exception):
        P.half_sphere(np.array([[1, 0, 0], [0, 0, 0]], np.int32))
