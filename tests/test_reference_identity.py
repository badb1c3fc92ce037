"""The SCF against a number the reference itself produced: its R0 identity case
(crates/dft-cli/tests/reference_identity.rs:15-160) runs its SCF driver on a synthetic
Si2 fcc cell (a = 10.26 Bohr, atoms at 0 and a/4 (1,1,1)), ecutwfc 8 Ry, Γ only, LDA-PZ,
with the pseudopotential of crates/dft-cli/tests/common/mod.rs:47-90 (Z = 4, local
-2 Z erf(r)/r Ry, projectors r^(l+1) exp(-r^2/(i+1)) for l = 0, 0, 1, DIJ
'2 0.4 0 0.4 4 0 0 0 6' Ry, 161 mesh points) and pins the converged total energy's bits:
0xc012bb05409e658e (reference driver) and 0xc012bb05409f01ad (its strict oracle), i.e.
-4.682637223880546 and -4.682637223916044 Ha, 3.5e-11 Ha apart.  Here the oracle SCF and
the GPU SCF (8 bands, fixed occupations, converged to 5e-12 Ha) must land within 1e-9 Ha
of both.  The path differs where it cannot matter at convergence: uniform start density
and Broyden mixing here, the atomic start and Pulay mixing there."""
import math

import numpy as np
import pytest

from oracle import ewald_ref as E
from oracle import scf_ref
from oracle import setup_ref as S

REFERENCE_HA = -4.682637223880546   # bits 0xc012bb05409e658e
STRICT_HA = -4.682637223916044      # bits 0xc012bb05409f01ad
ROWS = np.array([[0.0, 5.13, 5.13], [5.13, 0.0, 5.13], [5.13, 5.13, 0.0]])
POS = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]]) @ ROWS
ECUT_HA = 4.0
BANDS = 8


def test_golden_bits_decode():
    import struct
    assert struct.unpack("<d", struct.pack("<Q", 0xc012bb05409e658e))[0] == REFERENCE_HA
    assert struct.unpack("<d", struct.pack("<Q", 0xc012bb05409f01ad))[0] == STRICT_HA


def _oracle_case():
    ps = S.reference_test_pseudo(161)
    species = [S.Species(ps, POS)]
    cell = S.Cell(ROWS)
    dims, _ = S.grid_dims(cell, ECUT_HA, None)
    dens = S.basis_at_k(cell, 4.0 * ECUT_HA)
    box = np.zeros(dims, np.complex128)
    idx = S.g_to_fft(dens, dims)
    box[idx[:, 0], idx[:, 1], idx[:, 2]] = S.ionic_local(dens, cell.volume, species)
    v_ion = np.ascontiguousarray((np.fft.ifftn(box) * box.size).real)
    return ps, species, cell, dims, v_ion


def test_oracle_scf_reproduces_the_reference_energy():
    ps, species, cell, dims, v_ion = _oracle_case()
    assert list(dims) == [15, 15, 15]
    b = S.basis_at_k(cell, ECUT_HA)
    plus, minus, _ = S.half_sphere(b)
    rows = len(S.orc_pack(plus, minus, np.zeros(b.npw, np.complex128)))
    start = np.random.default_rng(1).standard_normal((rows, BANDS))
    ew = E.energy(ROWS, POS, np.full(2, 4.0))
    r = scf_ref.run(ROWS, species, ECUT_HA, dims, [((0.0, 0.0, 0.0), 1.0)], True, BANDS, v_ion, [start], ew,
                    threshold_ha=5e-12, beta=0.5, max_iterations=100)
    assert r.converged
    assert abs(r.energy - REFERENCE_HA) < 1e-9, r.energy - REFERENCE_HA
    assert abs(r.energy - STRICT_HA) < 1e-9, r.energy - STRICT_HA


@pytest.mark.gpu
def test_gpu_scf_reproduces_the_reference_energy(ctx):
    from baandi_b200 import operands as O
    from baandi_b200.scf import GpuScf, ScfOptions
    from baandi_b200.systems import Workload
    ps = S.reference_test_pseudo(161)
    pseudo = O.Pseudo(ps.z, ps.r, ps.rab, ps.local, [p.l for p in ps.projectors], [p.u for p in ps.projectors],
                      ps.dij)
    w = Workload("si2_reference_identity_8ry", ROWS, [O.Species(pseudo, POS)], ECUT_HA, BANDS, 4,
                 [((0.0, 0.0, 0.0), 1.0)], True, seed=2026)
    r = GpuScf(w, ctx, ScfOptions(threshold_ha=5e-12, beta=0.5, max_iterations=100)).run()
    assert r.converged
    assert abs(r.energy_ha - REFERENCE_HA) < 1e-9, r.energy_ha - REFERENCE_HA
    assert abs(r.energy_ha - STRICT_HA) < 1e-9, r.energy_ha - STRICT_HA
