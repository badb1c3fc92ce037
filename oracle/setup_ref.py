"""Oracle (test infrastructure only): CPU restatement of the reference's operand setup
for the Hamiltonian-apply path -- cells, plane-wave spheres, FFT grids, Gamma mirror
maps, k meshes, radial transforms, real harmonics and projector tables.

Only tests/, the smoke check and bench.py's cpu_baseline leg may import this module;
the product (baandi_b200) never does.

Each function cites the reference file:line it follows (paths inside the reference
project).  Arithmetic that decides an ORDER (|G|^2 used by the basis sort) is written
with the same operation order as the reference so the Miller lists agree bit for bit;
everything else is vectorised numpy and agrees to rounding.

Parity is pinned by tests/test_oracle_pins.py against the reference's own test recipes
(dense-H equalities, free-electron spectrum, FFT sign conventions, mirror-map
invariants) and by the committed fixtures in tests/golden/.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TAU = 2.0 * math.pi
CUTOFF_TOLERANCE = 1e-12  # crates/dft-basis/src/lib.rs:12


# ----------------------------------------------------------------------------- cell
@dataclass
class Cell:
    """Lattice vectors are the ROWS of `rows` (user rows), the columns of A.

    crates/dft-geometry/src/lib.rs:46-94: A = columns(rows); inverse computed on
    A/scale (scale = max |A_ij|), volume = ((|det| scale) scale) scale,
    B[i][j] = 2 pi inverse[j][i].
    """

    rows: np.ndarray
    lattice: np.ndarray = field(init=False)  # A[cart][vec]
    recip: np.ndarray = field(init=False)  # B[cart][vec]
    volume: float = field(init=False)

    def __post_init__(self):
        rows = np.asarray(self.rows, dtype=np.float64)
        a = rows.T.copy()
        scale = float(np.max(np.abs(a)))
        s = a / scale
        inv, det = _inverse3(s)
        inv = inv / scale
        self.lattice = a
        self.volume = ((abs(det) * scale) * scale) * scale
        self.recip = np.array([[TAU * inv[j][i] for j in range(3)] for i in range(3)])


def _inverse3(m):
    """Cofactor inverse of a 3x3 matrix (exact for the small-integer scaled lattices used here)."""
    m = [[float(m[i][j]) for j in range(3)] for i in range(3)]
    c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1]
    c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2]
    c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0]
    det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02
    inv = np.empty((3, 3))
    inv[0][0] = c00 / det
    inv[1][0] = c01 / det
    inv[2][0] = c02 / det
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det
    return inv, det


# ----------------------------------------------------------------------------- k points
def wrap_fractional(k):
    """crates/dft-geometry/src/kpoints.rs:21-32."""
    out = []
    for x in k:
        x = float(x)
        out.append(x if -0.5 <= x < 0.5 else x - math.floor(x + 0.5))
    return out


def monkhorst_pack(grid, shift=(0.0, 0.0, 0.0)):
    """crates/dft-geometry/src/kpoints.rs:63-88 (unshifted grid includes Gamma)."""
    count = grid[0] * grid[1] * grid[2]
    pts = []
    for i in range(grid[0]):
        for j in range(grid[1]):
            for k in range(grid[2]):
                m = (i, j, k)
                pts.append((wrap_fractional([(m[a] + shift[a]) / grid[a] for a in range(3)]), 1.0 / count))
    return pts


def reduce_time_reversal(points):
    """crates/dft-geometry/src/kpoints.rs:93-116: merge k and -k, keep the first."""
    result = []
    for k, w in points:
        k = wrap_fractional(k)
        found = None
        for p in result:
            for s in (1.0, -1.0):
                if all(abs((k[a] - s * p[0][a]) - round(k[a] - s * p[0][a])) <= 1e-12 for a in range(3)):
                    found = p
                    break
            if found is not None:
                break
        if found is not None:
            found[1] += w
        else:
            result.append([k, w])
    return [(tuple(k), w) for k, w in result]


# ----------------------------------------------------------------------------- basis
@dataclass
class Basis:
    miller: np.ndarray  # (npw, 3) int32, sorted by |G|^2 then Miller
    gcart: np.ndarray  # (npw, 3) G
    gnorm2: np.ndarray  # |G|^2
    kcart: np.ndarray  # (3,)
    kfrac: tuple
    kpg: np.ndarray  # (npw, 3) k+G
    kpg2: np.ndarray  # |k+G|^2

    @property
    def npw(self):
        return len(self.miller)


def _bounding_box(cell: Cell, ecut_ha: float):
    """crates/dft-basis/src/lib.rs:55-74."""
    radius = math.sqrt(2.0 * ecut_ha * (1.0 + CUTOFF_TOLERANCE))
    a = cell.lattice
    bounds = []
    for i in range(3):
        norm = math.hypot(math.hypot(a[0][i], a[1][i]), a[2][i])
        bounds.append(int(math.ceil(norm * radius / TAU) + 1.0))
    return bounds


def basis_at_k(cell: Cell, ecut_ha: float, kfrac=(0.0, 0.0, 0.0)) -> Basis:
    """G-sphere enumeration and sort, crates/dft-basis/src/lib.rs:96-120 (inclusion
    test), :233-265 (bounds+1, k canonicalisation, sort by |G|^2 then Miller).

    The Cartesian components and norms use the reference's operation order:
    c_i = ((b_i0 m0) + b_i1 m1) + b_i2 m2 and |c|^2 = (c0 c0 + c1 c1) + c2 c2.
    """
    kf = wrap_fractional(kfrac)
    b = cell.recip
    kc = np.array([(b[i][0] * kf[0] + b[i][1] * kf[1]) + b[i][2] * kf[2] for i in range(3)])
    bounds = [x + 1 for x in _bounding_box(cell, ecut_ha)]
    r = [np.arange(-bb, bb + 1, dtype=np.int64) for bb in bounds]
    m = np.stack(np.meshgrid(r[0], r[1], r[2], indexing="ij"), axis=-1).reshape(-1, 3)
    mf = m.astype(np.float64)
    cart = np.stack([(b[i][0] * mf[:, 0] + b[i][1] * mf[:, 1]) + b[i][2] * mf[:, 2] for i in range(3)], axis=1)
    norm2 = (cart[:, 0] * cart[:, 0] + cart[:, 1] * cart[:, 1]) + cart[:, 2] * cart[:, 2]
    q = cart + kc[None, :]
    q2 = (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]
    keep = 0.5 * q2 <= ecut_ha * (1.0 + CUTOFF_TOLERANCE)
    m, cart, norm2 = m[keep], cart[keep], norm2[keep]
    order = np.lexsort((m[:, 2], m[:, 1], m[:, 0], norm2))
    m, cart, norm2 = m[order], cart[order], norm2[order]
    kpg = cart + kc[None, :]
    kpg2 = (kpg[:, 0] * kpg[:, 0] + kpg[:, 1] * kpg[:, 1]) + kpg[:, 2] * kpg[:, 2]
    return Basis(m.astype(np.int32), cart, norm2, kc, tuple(kf), kpg, kpg2)


def _smooth(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def grid_dims(cell: Cell, ecut_ha: float, override=None):
    """Alias-free density grid, crates/dft-basis/src/lib.rs:414-455: required =
    2 max|m|+1 over the unshifted 4*Ecut sphere, rounded up to 2,3,5-smooth."""
    dens = basis_at_k(cell, 4.0 * ecut_ha)
    req = [int(2 * np.abs(dens.miller[:, i]).max() + 1) for i in range(3)]
    if override is not None:
        if any(override[i] < req[i] for i in range(3)):
            raise ValueError(f"FFT override {override} is smaller than required {req}")
        return list(override), req
    dims = []
    for d in req:
        while not _smooth(d):
            d += 1
        dims.append(d)
    return dims, req


def g_to_fft(basis: Basis, dims):
    """crates/dft-basis/src/lib.rs:380-398, :491-502. Gamma: canonical interval
    [-n/2,(n-1)/2] else IndexOutOfRange; k != 0: Miller mod n. Returns (npw,3) indices."""
    m = basis.miller.astype(np.int64)
    out = np.empty_like(m)
    gamma = tuple(basis.kfrac) == (0.0, 0.0, 0.0)
    for i in range(3):
        n = dims[i]
        if gamma and (np.any(m[:, i] < -(n // 2)) or np.any(m[:, i] > (n - 1) // 2)):
            raise ValueError("Miller index outside the canonical frequencies")
        out[:, i] = np.mod(m[:, i], n)
    flat = (out[:, 0] * dims[1] + out[:, 1]) * dims[2] + out[:, 2]
    if len(np.unique(flat)) != len(flat):
        raise ValueError("two coefficients share one FFT index")
    return out


def fft_flat(idx, dims):
    return ((idx[:, 0] * dims[1] + idx[:, 1]) * dims[2] + idx[:, 2]).astype(np.int64)


def half_sphere(basis: Basis):
    """Gamma mirror maps, crates/dft-basis/src/half.rs:41-99: plus = [0] + indices with
    Miller > (0,0,0) lexicographically (ascending full-list order), minus = mirrors."""
    m = basis.miller
    if tuple(basis.kfrac) != (0.0, 0.0, 0.0) or tuple(m[0]) != (0, 0, 0):
        raise ValueError("not a Gamma sphere")
    lookup = {tuple(v): i for i, v in enumerate(m.tolist())}
    mirror = np.array([lookup[(-a, -b, -c)] for a, b, c in m.tolist()], dtype=np.int64)
    pos = [i for i, (a, b, c) in enumerate(m.tolist()) if (a, b, c) > (0, 0, 0)]
    plus = np.array([0] + pos, dtype=np.int64)
    minus = np.array([0] + [int(mirror[i]) for i in pos], dtype=np.int64)
    return plus, minus, mirror


def orc_pack(plus, minus, full):
    """half.rs:117-142: complex Hermitian vector -> ORC real rows."""
    n = len(full)
    real = np.empty(n)
    real[0] = full[0].real
    i = np.arange(1, len(plus))
    real[2 * i - 1] = math.sqrt(2.0) * full[plus[1:]].real
    real[2 * i] = math.sqrt(2.0) * full[plus[1:]].imag
    return real


def orc_unpack(plus, minus, real):
    """half.rs:144-157: ORC rows -> Hermitian complex vector."""
    n = len(real)
    full = np.empty(n, dtype=np.complex128)
    full[0] = real[0]
    i = np.arange(1, len(plus))
    z = (real[2 * i - 1] + 1j * real[2 * i]) / math.sqrt(2.0)
    full[plus[1:]] = z
    full[minus[1:]] = np.conj(z)
    return full


# ----------------------------------------------------------------------------- radial
@dataclass
class Projector:
    l: int
    u: np.ndarray  # r * beta(r) on the mesh (Bohr^-1/2)


@dataclass
class Pseudo:
    """Synthetic norm-conserving pseudopotential on a logarithmic mesh, in the
    reference's UPF conventions (scripts/gen_synthetic_upf.py:13-47,
    crates/dft-upf/tests/common/mod.rs:2-8): r_i = r0 expm1(i dx), rab = dx (r + r0).
    local in Ha, D (dij) in Ha, row-major over projectors."""

    z: float
    r: np.ndarray
    rab: np.ndarray
    local: np.ndarray
    projectors: list
    dij: np.ndarray
    rho_atom: np.ndarray | None = None  # PP_RHOATOM: 4 pi r^2 rho_atom(r) on the mesh


def log_mesh(points: int, end: float = 12.0, r0: float = 0.02):
    dx = math.log1p(end / r0) / (points - 1)
    r = np.array([r0 * math.expm1(i * dx) for i in range(points)])
    rab = dx * (r + r0)
    return r, rab


def synthetic_pseudo(z: float, rc: float, channels, r_beta, dij_ha, points=1201, rho_radius=None) -> Pseudo:
    """Gaussian-erf local part -Z erf(r/rc)/r (Ha) and r^l exp(-(r/r_beta)^2) projectors;
    with rho_radius, the Gaussian atomic charge of that radius as PP_RHOATOM."""
    r, rab = log_mesh(points)
    local = np.empty_like(r)
    local[0] = -2.0 * z / (rc * math.sqrt(math.pi))
    local[1:] = -z * np.array([math.erf(x / rc) for x in r[1:]]) / r[1:]
    projs = []
    for l, rb in zip(channels, r_beta):
        projs.append(Projector(l, r ** (l + 1) * np.exp(-(r / rb) ** 2)))
    rho = None if rho_radius is None else gaussian_rho_atom(z, rho_radius, r)
    return Pseudo(z, r, rab, local, projs, np.asarray(dij_ha, dtype=np.float64), rho)


def gaussian_rho_atom(z: float, radius: float, r: np.ndarray) -> np.ndarray:
    """4 pi r^2 rho(r) of the charge z spread as rho(r) = z exp(-(r/R)^2) / (pi^(3/2) R^3),
    the atomic-charge variant of the reference's synthetic fixtures
    (scripts/gen_synthetic_upf.py:64-65): 4 z / (sqrt(pi) R^3) r^2 exp(-(r/R)^2)."""
    r = np.asarray(r, dtype=np.float64)
    return 4.0 * z / (math.sqrt(math.pi) * radius ** 3) * r * r * np.exp(-(r / radius) ** 2)


def reference_test_pseudo(points=801) -> Pseudo:
    """The reference's dense-H test fixture, crates/dft-upf/tests/common/mod.rs:44-80:
    Z=4, local -8 erf(r)/r Ry, beta_i = r^(l+1) exp(-r^2/(i+1)) for l=(0,0,1),
    DIJ '2 0.4 0 0.4 4 0 0 0 6' Ry."""
    r, rab = log_mesh(points)
    local = np.empty_like(r)
    local[0] = -16.0 / math.sqrt(math.pi) / 2.0
    local[1:] = -8.0 * np.array([math.erf(x) for x in r[1:]]) / r[1:] / 2.0
    projs = [Projector(l, r ** (l + 1) * np.exp(-r * r / (i + 1))) for i, l in enumerate((0, 0, 1))]
    dij = np.array([2, 0.4, 0, 0.4, 4, 0, 0, 0, 6], dtype=np.float64) / 2.0
    return Pseudo(4.0, r, rab, local, projs, dij)


def simpson_weights(n: int) -> np.ndarray:
    """Index-coordinate composite Simpson 1/3 with a final 3/8 panel for even n,
    crates/dft-upf/src/radial.rs:58-81 (the reference sums panels with Kahan
    compensation; the weighted dot here agrees to rounding)."""
    w = np.zeros(n)
    if n < 2:
        return w
    if n == 2:
        w[:] = 0.5
        return w
    last = n - 4 if n % 2 == 0 else n - 1
    for i in range(0, last, 2):
        w[i] += 1.0 / 3.0
        w[i + 1] += 4.0 / 3.0
        w[i + 2] += 1.0 / 3.0
    if n % 2 == 0:
        for o, c in zip(range(4), (3.0 / 8.0, 9.0 / 8.0, 9.0 / 8.0, 3.0 / 8.0)):
            w[last + o] += c
    return w


def spherical_bessel(l: int, x: np.ndarray) -> np.ndarray:
    """j_l for l <= 3, radial.rs:89-117: power series for x < 4, upward recurrence else."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = x < 4.0
    xs = x[small]
    if xs.size:
        term = np.ones_like(xs)
        for k in range(1, l + 1):
            term = term * xs / (2 * k + 1)
        total = term.copy()
        for k in range(1, 80):
            term = term * (-xs * xs / (2 * k * (2 * l + 2 * k + 1)))
            total = total + term
        out[small] = total
    xl = x[~small]
    if xl.size:
        s, c = np.sin(xl), np.cos(xl)
        prev = s / xl
        if l == 0:
            out[~small] = prev
        else:
            cur = (prev - c) / xl
            for k in range(1, l):
                nxt = (2 * k + 1) / xl * cur - prev
                prev, cur = cur, nxt
            out[~small] = cur
    return out


def projector_transform(ps: Pseudo, index: int, q: np.ndarray) -> np.ndarray:
    """F(q) = 4 pi int r u(r) j_l(q r) dr, radial.rs:321-344 (vectorised over q)."""
    p = ps.projectors[index]
    n = len(p.u)
    w = simpson_weights(n)
    r, rab = ps.r[:n], ps.rab[:n]
    q = np.asarray(q, dtype=np.float64)
    out = np.empty(q.shape)
    flat = q.reshape(-1)
    res = out.reshape(-1)
    chunk = 256
    for s in range(0, flat.size, chunk):
        qq = flat[s:s + chunk]
        j = spherical_bessel(p.l, qq[:, None] * r[None, :])
        res[s:s + chunk] = 4.0 * math.pi * (((r * p.u)[None, :] * j) * rab[None, :]) @ w
    return out


def real_harmonics(lmax: int, direction: np.ndarray) -> np.ndarray:
    """Real normalised Y_lm (radial.rs:119-240) for rows of `direction`; output
    (n, (lmax+1)^2) indexed l*l+l+m. Condon-Shortley P_l^m with an extra (-1)^m,
    negative m sine, positive m cosine."""
    d = np.asarray(direction, dtype=np.float64)
    norm = np.hypot(np.hypot(d[:, 0], d[:, 1]), d[:, 2])
    z = np.clip(d[:, 2] / norm, -1.0, 1.0)
    phi = np.arctan2(d[:, 1], d[:, 0])
    out = np.empty((len(d), (lmax + 1) ** 2))
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            a = abs(m)
            p = np.ones_like(z)
            for k in range(1, a + 1):
                p = p * (-(2 * k - 1) * np.sqrt((1.0 - z) * (1.0 + z)))
            if l > a:
                prev = p
                p = p * ((2 * a + 1) * z)
                for k in range(a + 2, l + 1):
                    nxt = ((2 * k - 1) * z * p - (k + a - 1) * prev) / (k - a)
                    prev, p = p, nxt
            ratio = 1.0
            for k in range(l - a + 1, l + a + 1):
                ratio /= k
            nrm = math.sqrt((2 * l + 1) / (4.0 * math.pi) * ratio)
            if m == 0:
                ang = 1.0
            else:
                sign = 1.0 if a % 2 == 0 else -1.0
                ang = math.sqrt(2.0) * sign * (np.sin(a * phi) if m < 0 else np.cos(a * phi))
            out[:, l * l + l + m] = nrm * p * ang
    return out


@dataclass
class Species:
    pseudo: Pseudo
    positions: np.ndarray  # (natoms, 3) Cartesian Bohr


@dataclass
class Nonlocal:
    table: np.ndarray  # (npw, nproj) complex, column-major use
    channels: list  # per atom channel count
    couplings: list  # per atom (count*count,) row-major D (Ha)


def nonlocal_table(basis: Basis, volume: float, species) -> Nonlocal:
    """Projector table beta_{a,(i,l,m)}(k+G) = (-i)^l Y_lm(k+G) F_i(|k+G|)/sqrt(Omega)
    * exp(-i (k+G).tau_a), crates/dft-physics/src/hamiltonian.rs:2605-2760 (channels
    per projector i with m=-l..l, direction (0,0,1) at |k+G|=0, coupling D_ij on
    equal (l,m)); phase from hamiltonian.rs:57-63."""
    cols, channels, couplings = [], [], []
    q = np.sqrt(basis.kpg2)
    uq, inv = np.unique(basis.kpg2, return_inverse=True)
    direction = basis.kpg.copy()
    direction[basis.kpg2 == 0.0] = [0.0, 0.0, 1.0]
    vr = math.sqrt(volume)
    for s in species:
        ps = s.pseudo
        npj = len(ps.projectors)
        for i in range(npj):
            for j in range(npj):
                if ps.projectors[i].l != ps.projectors[j].l and ps.dij[i * npj + j] != 0.0:
                    raise ValueError("angular coupling between different l")
        chans = [(i, p.l, m) for i, p in enumerate(ps.projectors) for m in range(-p.l, p.l + 1)]
        lmax = max([p.l for p in ps.projectors], default=0)
        ylm = real_harmonics(lmax, direction)
        radial = np.stack([projector_transform(ps, i, np.sqrt(uq))[inv] for i in range(npj)], axis=1)
        table = []
        for (i, l, m) in chans:
            pref = (-1j) ** l
            table.append(pref * ylm[:, l * l + l + m] * radial[:, i] / vr)
        nc = len(chans)
        coupling = np.zeros(nc * nc)
        for a, (i, l, m) in enumerate(chans):
            for bb, (j, ll, mm) in enumerate(chans):
                if l == ll and m == mm:
                    coupling[a * nc + bb] = ps.dij[i * npj + j]
        for tau in np.atleast_2d(s.positions):
            angle = (basis.kpg[:, 0] * tau[0] + basis.kpg[:, 1] * tau[1]) + basis.kpg[:, 2] * tau[2]
            phase = np.cos(-angle) + 1j * np.sin(-angle)
            for col in table:
                cols.append(col * phase)
            channels.append(nc)
            couplings.append(coupling.copy())
    table = np.stack(cols, axis=1) if cols else np.zeros((basis.npw, 0), dtype=np.complex128)
    del q
    return Nonlocal(table, channels, couplings)


def coupling_matrix(nl: Nonlocal) -> np.ndarray:
    """Block-diagonal D over all projector columns."""
    n = sum(nl.channels)
    d = np.zeros((n, n))
    o = 0
    for c, v in zip(nl.channels, nl.couplings):
        d[o:o + c, o:o + c] = np.asarray(v).reshape(c, c)
        o += c
    return d


def static_diagonal(kinetic: np.ndarray, nl: Nonlocal) -> np.ndarray:
    """T_g + sum_atom sum_ij D_ij Re(P_gi conj(P_gj)), crates/dft-physics/src/
    distributed_complex.rs:29-53 (pairs added in (atom, i, j) order, zero D skipped)."""
    diag = kinetic.astype(np.float64).copy()
    off = 0
    for c, v in zip(nl.channels, nl.couplings):
        for i in range(c):
            for j in range(c):
                dd = v[i * c + j]
                if dd == 0.0:
                    continue
                diag += (dd * nl.table[:, off + i] * np.conj(nl.table[:, off + j])).real
        off += c
    return diag


def orc_projectors(plus, table: np.ndarray) -> np.ndarray:
    """Real ORC projector rows, crates/dft-physics/src/distributed_real_gamma.rs:358-398
    (row 0 Re P(0), row 2i-1 sqrt2 Re P(plus i), row 2i sqrt2 Im P(plus i))."""
    n = table.shape[0]
    out = np.empty((n, table.shape[1]))
    out[0] = table[0].real
    i = np.arange(1, len(plus))
    out[2 * i - 1] = math.sqrt(2.0) * table[plus[1:]].real
    out[2 * i] = math.sqrt(2.0) * table[plus[1:]].imag
    return out


def orc_kinetic(plus, kpg2):
    """distributed_real_gamma.rs:345-355: kinetic in ORC order (each pair row shares
    its representative's 0.5 |G|^2)."""
    n = len(kpg2)
    out = np.empty(n)
    out[0] = 0.5 * kpg2[0]
    i = np.arange(1, len(plus))
    out[2 * i - 1] = 0.5 * kpg2[plus[1:]]
    out[2 * i] = 0.5 * kpg2[plus[1:]]
    return out


# ----------------------------------------------------------------------------- local part
def local_form_factor(ps: Pseudo, volume: float, g: np.ndarray) -> np.ndarray:
    """V_loc(|G|) in Ha with the erf(r) Coulomb subtraction, crates/dft-upf/src/radial.rs:
    246-305 (endpoint = last mesh point <= min(r_end, 10) Bohr; G=0 gives alpha_Z =
    4 pi/Omega short(0) + pi Z/Omega)."""
    n = int(np.searchsorted(ps.r, min(ps.r[-1], 10.0), side="right"))
    r, rab = ps.r[:n], ps.rab[:n]
    w = simpson_weights(n)
    erf_r = np.array([math.erf(x) for x in r])
    short = r * r * ps.local[:n] + ps.z * r * erf_r
    g = np.asarray(g, dtype=np.float64)
    out = np.empty(g.shape)
    flat, res = g.reshape(-1), out.reshape(-1)
    for s in range(0, flat.size, 256):
        gg = flat[s:s + 256]
        j0 = spherical_bessel(0, gg[:, None] * r[None, :])
        integral = ((short[None, :] * j0) * rab[None, :]) @ w
        with np.errstate(divide="ignore", invalid="ignore"):
            val = 4.0 * math.pi / volume * (integral - ps.z * np.exp(-gg * gg / 4.0) / (gg * gg))
        zero = gg == 0.0
        val[zero] = 4.0 * math.pi / volume * integral[zero] + math.pi * ps.z / volume
        res[s:s + 256] = val
    return out


# ----------------------------------------------------------------------------- start density
def has_atomic_charge(ps: Pseudo) -> bool:
    """crates/dft-engine/src/refstart.rs:56-59: PP_RHOATOM on the whole mesh, not all zero."""
    rho = ps.rho_atom
    return rho is not None and len(rho) == len(ps.r) and bool(np.any(np.asarray(rho) != 0.0))


def atomic_charge_transform(ps: Pseudo, volume: float, q: np.ndarray) -> np.ndarray:
    """rho_atom(|G|) / Omega = (integral of PP_RHOATOM j0(q r) dr) / Omega on the mesh
    (Simpson in the index with rab, radial.rs:40-47), the exact per-shell quadrature of the
    reference's Gamma start (refstart.rs:1213-1226; j0 taken as 1 at q = 0)."""
    n = len(ps.r)
    w = simpson_weights(n) * ps.rab
    rho = np.asarray(ps.rho_atom, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64).reshape(-1)
    out = np.empty(q.size)
    for s in range(0, q.size, 256):
        qq = q[s:s + 256]
        j0 = spherical_bessel(0, qq[:, None] * ps.r[None, :])
        j0[qq == 0.0, :] = 1.0
        out[s:s + 256] = ((rho[None, :] * j0) @ w) / volume
    return out


def atomic_density(cell: Cell, ecut_ha: float, dims, species):
    """The reference's atomic start density (refstart.rs:704-757 with the rho channel of
    atomic_fields :1166-1230), or None when any species carries no atomic charge (the
    uniform start, refstart.rs:708-710, 725-735).  rho(G) = sum_s rho_s(|G|) S_s(G) / Omega
    on the 4 Ecut density sphere; n(r) = sum_G rho(G) e^{iGr} on the grid (C order),
    negative values set to 0, then scaled so that sum n Omega / N_points = N_e."""
    if not all(has_atomic_charge(s.pseudo) for s in species):
        return None
    dens = basis_at_k(cell, 4.0 * ecut_ha)
    q2u, inv = np.unique(dens.gnorm2, return_inverse=True)
    rg = np.zeros(dens.npw, np.complex128)
    for sp in species:
        ff = atomic_charge_transform(sp.pseudo, cell.volume, np.sqrt(q2u))[inv]
        sf = np.zeros(dens.npw, np.complex128)
        for tau in np.atleast_2d(sp.positions):
            ang = (dens.gcart[:, 0] * tau[0] + dens.gcart[:, 1] * tau[1]) + dens.gcart[:, 2] * tau[2]
            sf += np.cos(-ang) + 1j * np.sin(-ang)
        rg += ff * sf
    box = np.zeros(dims, np.complex128)
    idx = g_to_fft(dens, dims)
    box[idx[:, 0], idx[:, 1], idx[:, 2]] = rg
    n = np.ascontiguousarray((np.fft.ifftn(box) * box.size).real)
    n = np.maximum(n, 0.0)
    electrons = float(sum(s.pseudo.z * np.atleast_2d(s.positions).shape[0] for s in species))
    charge = float(n.sum()) * cell.volume / n.size
    if not np.isfinite(charge) or charge <= 0.0:
        raise ValueError("invalid atomic charge")
    return n * (electrons / charge)


def ionic_local(density: Basis, volume: float, species) -> np.ndarray:
    """V_ion(G) on the density sphere, crates/dft-physics/src/hamiltonian.rs:211-300:
    sum over species of V_loc(|G|) S(G), S(G) = sum_I exp(-i G.tau_I)."""
    out = np.zeros(density.npw, dtype=np.complex128)
    q = np.sqrt(density.gnorm2)
    for s in species:
        ff = local_form_factor(s.pseudo, volume, q)
        sf = np.zeros(density.npw, dtype=np.complex128)
        for tau in np.atleast_2d(s.positions):
            ang = (density.gcart[:, 0] * tau[0] + density.gcart[:, 1] * tau[1]) + density.gcart[:, 2] * tau[2]
            sf += np.cos(-ang) + 1j * np.sin(-ang)
        out += ff * sf
    return out
