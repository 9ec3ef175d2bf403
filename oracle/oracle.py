"""CPU oracle for the fixed-charge nonbonded path (TEST INFRASTRUCTURE ONLY).

This module is the correctness checker. Only the test-suite, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import it; the product path in
``torchff_b200`` never does, and fails loudly when its CUDA library is missing.

It restates, in float64 numpy, the reference's pure-torch path (THGLab/torchff-lib):

* minimum image through the inverse box, ``ds - floor(ds + 0.5)``
  (``torchff/pbc.py:59-62``);
* exclusion COO -> symmetric CSR (``torchff/nblist.py:50-123``);
* the half neighbour list within the cutoff minus exclusions
  (``torchff/nblist.py:39-48, 137-140``; device kernel ``csrc/nblist/nblist_nsquared_cuda.cu:29-116``);
* shifted Coulomb (``torchff/coulomb.py:22-44``), Lennard-Jones 12-6 with per-pair
  sigma/epsilon or type tables (``torchff/vdw.py:86-111, 230-261``), the fused
  Coulomb + LJ term with Lorentz-Berthelot combining from per-atom parameters
  (``torchff/nonbonded.py:40-69``, combining rule of
  ``csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:86-90``);
* rank-0 real-space Ewald Coulomb with the erfc-1 exclusion correction
  (``torchff/multipoles.py:106-127, 244-341``);
* rank-0 smooth PME reciprocal space with order-6 B-splines
  (``torchff/pme_ref.py:11-469``, ``torchff/pme.py:67-126``);
* harmonic bonds and angles of flexible water (``torchff/bond.py:34-43``,
  ``torchff/angle.py:8-34, 103-112``).

Energies and all first derivatives are analytic. The tests pin this module against the
golden fixtures in ``tests/golden`` which were produced by running the reference's own
pure-torch code with autograd (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math

import numpy as np

# ---------------------------------------------------------------------------
# periodic boundary conditions
# ---------------------------------------------------------------------------


def min_image(dr: np.ndarray, box: np.ndarray | None) -> np.ndarray:
    """Minimum-image displacement, rows of ``box`` are the box vectors (torchff/pbc.py:59-62)."""
    if box is None:
        return dr
    box_inv = np.linalg.inv(box)
    ds = dr @ box_inv
    ds = ds - np.floor(ds + 0.5)
    return ds @ box


# ---------------------------------------------------------------------------
# neighbour list
# ---------------------------------------------------------------------------


def exclusions_coo_to_csr(pairs: np.ndarray, natoms: int) -> tuple[np.ndarray, np.ndarray]:
    """Symmetrise, deduplicate and compress exclusion pairs (torchff/nblist.py:50-123)."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    both = np.concatenate([pairs, pairs[:, ::-1]], 0)
    keys = np.unique(both[:, 0] * natoms + both[:, 1])
    rows = keys // natoms
    cols = keys % natoms
    counts = np.bincount(rows, minlength=natoms)
    row_ptr = np.zeros(natoms + 1, dtype=np.int64)
    row_ptr[1:] = np.cumsum(counts)
    return row_ptr, cols.astype(np.int64)


def nblist_pairs(
    coords: np.ndarray,
    box: np.ndarray | None,
    cutoff: float,
    excl_row_ptr: np.ndarray | None = None,
    excl_col: np.ndarray | None = None,
    include_self: bool = False,
    chunk: int = 1024,
) -> np.ndarray:
    """All pairs (i, j), i >= j, with |r_ij| <= cutoff, minus CSR exclusions.

    Returned in canonical order (sorted by i then j) with i the larger index, as the
    reference's kernels emit them (``csrc/nblist/nblist_nsquared_cuda.cu:74-76``,
    ``csrc/nblist/nblist_clist_cuda.cu:300-305``). Self pairs (i, i) are included only
    when ``include_self``.
    """
    x = np.asarray(coords, dtype=np.float64)
    n = x.shape[0]
    rc2 = float(cutoff) * float(cutoff)
    box_inv = None if box is None else np.linalg.inv(box)
    excluded = set()
    if excl_col is not None and excl_row_ptr is not None:
        for i in range(n):
            for e in range(excl_row_ptr[i], excl_row_ptr[i + 1]):
                excluded.add(i * n + int(excl_col[e]))
    out = []
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        ii = np.arange(i0, i1)
        dr = x[ii, None, :] - x[None, : i1, :]          # (ci, i1, 3)
        if box is not None:
            ds = dr @ box_inv
            ds -= np.floor(ds + 0.5)
            dr = ds @ box
        d2 = np.einsum("abk,abk->ab", dr, dr)
        jj = np.arange(i1)[None, :]
        lower = jj < ii[:, None] if not include_self else jj <= ii[:, None]
        mask = lower & (d2 <= rc2)
        a, b = np.nonzero(mask)
        out.append(np.stack([ii[a], b], 1))
    pairs = np.concatenate(out, 0) if out else np.zeros((0, 2), np.int64)
    if excluded:
        keys = pairs[:, 0] * n + pairs[:, 1]
        keep = np.fromiter((k not in excluded for k in keys.tolist()), bool, len(keys))
        pairs = pairs[keep]
    order = np.lexsort((pairs[:, 1], pairs[:, 0]))
    return pairs[order].astype(np.int64)


def canonical_pairs(pairs: np.ndarray) -> np.ndarray:
    """Drop -1 padding, orient each pair as (max, min) and sort: the set view used for parity."""
    p = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    p = p[(p[:, 0] >= 0) & (p[:, 1] >= 0)]
    hi = np.maximum(p[:, 0], p[:, 1])
    lo = np.minimum(p[:, 0], p[:, 1])
    q = np.stack([hi, lo], 1)
    order = np.lexsort((q[:, 1], q[:, 0]))
    return q[order]


# ---------------------------------------------------------------------------
# pair terms
# ---------------------------------------------------------------------------


def _pair_geometry(coords, pairs, box):
    i = pairs[:, 0]
    j = pairs[:, 1]
    dr = min_image(coords[i] - coords[j], box)   # r_i - r_j
    r = np.sqrt(np.einsum("ab,ab->a", dr, dr))
    return i, j, dr, r


def _scatter_vec(n, i, j, g_i_vec):
    """Gradient accumulation for a pair quantity depending on r_i - r_j."""
    g = np.zeros((n, 3))
    np.add.at(g, i, g_i_vec)
    np.add.at(g, j, -g_i_vec)
    return g


def coulomb(coords, pairs, box, q, k, cutoff, do_shift=True):
    """Shifted Coulomb (torchff/coulomb.py:22-44); returns E, dE/dx, dE/dq."""
    coords = np.asarray(coords, np.float64)
    n = coords.shape[0]
    pairs = np.asarray(pairs, np.int64)
    pairs = pairs[(pairs[:, 0] >= 0) & (pairs[:, 1] >= 0)]
    i, j, dr, r = _pair_geometry(coords, pairs, box)
    m = r <= cutoff
    i, j, dr, r = i[m], j[m], dr[m], r[m]
    rinv = 1.0 / r
    shifted = rinv - (1.0 / cutoff if do_shift else 0.0)
    e = k * q[i] * q[j] * shifted
    de_dr = -k * q[i] * q[j] * rinv * rinv
    gx = _scatter_vec(n, i, j, (de_dr * rinv)[:, None] * dr)
    gq = np.zeros(n)
    np.add.at(gq, i, k * q[j] * shifted)
    np.add.at(gq, j, k * q[i] * shifted)
    return float(e.sum()), gx, gq


def _lj_terms(r, sig, eps):
    sr6 = (sig / r) ** 6
    e = 4.0 * eps * sr6 * (sr6 - 1.0)
    de_dr = -24.0 * eps * sr6 * (2.0 * sr6 - 1.0) / r
    de_dsig = 24.0 * eps * sr6 * (2.0 * sr6 - 1.0) / sig
    de_deps = 4.0 * sr6 * (sr6 - 1.0)
    return e, de_dr, de_dsig, de_deps


def lennard_jones(coords, pairs, box, sigma, epsilon, cutoff, atom_types=None):
    """LJ 12-6 (torchff/vdw.py:86-111, 230-261).

    ``sigma``/``epsilon`` are per pair, shape (P,), or type tables (T, T) when
    ``atom_types`` is given. Returns E, dE/dx, dE/dsigma, dE/depsilon (same shapes as
    the parameter inputs).
    """
    coords = np.asarray(coords, np.float64)
    n = coords.shape[0]
    pairs = np.asarray(pairs, np.int64)
    valid = (pairs[:, 0] >= 0) & (pairs[:, 1] >= 0)
    idx = np.nonzero(valid)[0]
    pairs = pairs[valid]
    i, j, dr, r = _pair_geometry(coords, pairs, box)
    m = r <= cutoff
    if atom_types is None:
        sig = np.asarray(sigma)[idx]
        eps = np.asarray(epsilon)[idx]
    else:
        ti = atom_types[i]
        tj = atom_types[j]
        sig = np.asarray(sigma)[ti, tj]
        eps = np.asarray(epsilon)[ti, tj]
    e, de_dr, de_ds, de_de = _lj_terms(r, sig, eps)
    e = np.where(m, e, 0.0)
    de_dr = np.where(m, de_dr, 0.0)
    de_ds = np.where(m, de_ds, 0.0)
    de_de = np.where(m, de_de, 0.0)
    gx = _scatter_vec(n, i, j, (de_dr / r)[:, None] * dr)
    if atom_types is None:
        gs = np.zeros(np.asarray(sigma).shape)
        ge = np.zeros(np.asarray(epsilon).shape)
        gs[idx] = de_ds
        ge[idx] = de_de
    else:
        gs = np.zeros(np.asarray(sigma).shape)
        ge = np.zeros(np.asarray(epsilon).shape)
        np.add.at(gs, (ti, tj), de_ds)
        np.add.at(ge, (ti, tj), de_de)
    return float(e.sum()), gx, gs, ge


def nonbonded(coords, pairs, box, sigma, epsilon, q, k, cutoff, do_shift=True):
    """Fused shifted Coulomb + LJ with LB combining of per-atom sigma/epsilon.

    Restates ``torchff/nonbonded.py:40-69`` (Coulomb ``torchff/coulomb.py:22-44`` plus LJ
    ``torchff/vdw.py:86-111``) with sigma_ij = (sigma_i + sigma_j)/2 and
    epsilon_ij = sqrt(epsilon_i epsilon_j) as in
    ``csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:86-90``.

    Returns E, dE/dx, dE/dq, dE/dsigma, dE/depsilon. The epsilon derivative of a pair
    with epsilon_ij = 0 is taken as 0 (the chain rule through sqrt is singular there).
    """
    coords = np.asarray(coords, np.float64)
    n = coords.shape[0]
    e_c, gx_c, gq = coulomb(coords, pairs, box, q, k, cutoff, do_shift)
    pairs = np.asarray(pairs, np.int64)
    pairs = pairs[(pairs[:, 0] >= 0) & (pairs[:, 1] >= 0)]
    i, j, dr, r = _pair_geometry(coords, pairs, box)
    m = r <= cutoff
    i, j, dr, r = i[m], j[m], dr[m], r[m]
    sig = 0.5 * (sigma[i] + sigma[j])
    eps = np.sqrt(epsilon[i] * epsilon[j])
    e, de_dr, de_ds, de_de = _lj_terms(r, sig, eps)
    gx = gx_c + _scatter_vec(n, i, j, (de_dr / r)[:, None] * dr)
    gs = np.zeros(n)
    np.add.at(gs, i, 0.5 * de_ds)
    np.add.at(gs, j, 0.5 * de_ds)
    ge = np.zeros(n)
    safe = eps > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        fi = np.where(safe, de_de * epsilon[j] / (2.0 * np.where(safe, eps, 1.0)), 0.0)
        fj = np.where(safe, de_de * epsilon[i] / (2.0 * np.where(safe, eps, 1.0)), 0.0)
    np.add.at(ge, i, fi)
    np.add.at(ge, j, fj)
    return e_c + float(e.sum()), gx, gq, gs, ge


def _erfc(x):
    from scipy.special import erfc as _scipy_erfc

    return _scipy_erfc(x)


def ewald_real(coords, box, pairs, q, cutoff, alpha, prefactor, pairs_excl=None):
    """Rank-0 real-space Ewald Coulomb with exclusion correction.

    E = prefactor [sum_{pairs, r<=rc} q_i q_j erfc(a r)/r
                   + sum_{excl, r<=rc} q_i q_j (erfc(a r) - 1)/r]
    (torchff/multipoles.py:106-127, 244-341; kernel csrc/multipoles/multipoles_forward.cuh:356-617).
    With ``alpha < 0`` the plain 1/r Coulomb is used and exclusions are ignored, as in
    ``torchff/multipoles.py:317``. Returns E, dE/dx, dE/dq.
    """
    coords = np.asarray(coords, np.float64)
    n = coords.shape[0]
    e_tot = 0.0
    gx = np.zeros((n, 3))
    gq = np.zeros(n)
    lists = [(np.asarray(pairs, np.int64), False)]
    if pairs_excl is not None and alpha > 0:
        lists.append((np.asarray(pairs_excl, np.int64), True))
    for pl, is_excl in lists:
        pl = pl[(pl[:, 0] >= 0) & (pl[:, 1] >= 0)]
        i, j, dr, r = _pair_geometry(coords, pl, box)
        m = r <= cutoff
        i, j, dr, r = i[m], j[m], dr[m], r[m]
        if alpha >= 0:
            u = alpha * r
            damp = _erfc(u) - (1.0 if is_excl else 0.0)
            # d/dr [damp / r] = -damp/r^2 - (2 a / sqrt(pi)) exp(-u^2) / r
            dfdr = -damp / r**2 - (2.0 * alpha / math.sqrt(math.pi)) * np.exp(-u * u) / r
        else:
            damp = np.ones_like(r)
            dfdr = -1.0 / r**2
        f = damp / r
        e_tot += prefactor * float(np.sum(q[i] * q[j] * f))
        gx += _scatter_vec(n, i, j, (prefactor * q[i] * q[j] * dfdr / r)[:, None] * dr)
        np.add.at(gq, i, prefactor * q[j] * f)
        np.add.at(gq, j, prefactor * q[i] * f)
    return e_tot, gx, gq


# ---------------------------------------------------------------------------
# PME (rank 0)
# ---------------------------------------------------------------------------

PME_ORDER = 6


def bspline6(u: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Cardinal B-spline M_6(u) on [0, 6) and its derivative.

    Uses the Cox-de Boor style recursion of Essmann et al., J. Chem. Phys. 103, 8577
    (1995), eq. 4.1: M_n(u) = u/(n-1) M_{n-1}(u) + (n-u)/(n-1) M_{n-1}(u-1), with
    M_2(u) = 1 - |u - 1| on [0, 2], and M_n'(u) = M_{n-1}(u) - M_{n-1}(u-1).
    """
    u = np.asarray(u, dtype=np.float64)

    def m(n, x):
        if n == 2:
            return np.where((x >= 0) & (x <= 2), 1.0 - np.abs(x - 1.0), 0.0)
        return (x * m(n - 1, x) + (n - x) * m(n - 1, x - 1.0)) / (n - 1)

    val = np.where((u >= 0) & (u < 6), m(6, u), 0.0)
    der = np.where((u >= 0) & (u < 6), m(5, u) - m(5, u - 1.0), 0.0)
    return val, der


def bspline_moduli(K: int) -> np.ndarray:
    """theta(k) = sum_{m=-3}^{2} M_6(m+3) cos(2 pi m k / K) (torchff/bsplines.py:20-63)."""
    m = np.arange(-3, 3)
    w, _ = bspline6(m + 3.0)
    k = np.arange(K)
    return np.sum(w[:, None] * np.cos(2.0 * np.pi * m[:, None] * k[None, :] / K), 0)


def signed_frequency(K: int) -> np.ndarray:
    """FFT index -> signed integer frequency, Nyquist mapped to -K/2 (torchff/pme_ref.py:146-150)."""
    i = np.arange(K)
    return np.where(2 * i >= K, i - K, i)


def _pme_stencil(coords, box, K):
    """Per-atom grid origin m0 (N,3), spline values and derivatives (N, 3, 6)."""
    recip = (np.array([K, K, K])[:, None] * np.linalg.inv(box).T)   # row d: K_d * inv(box)[:, d]
    frac = coords @ recip.T                                           # (N, 3) in grid units
    m0 = np.ceil(frac).astype(np.int64)
    u0 = (m0 - frac) + PME_ORDER / 2
    shifts = np.arange(-3, 3)
    u = u0[:, :, None] + shifts[None, None, :]
    val, der = bspline6(u)
    return recip, m0, val, der, shifts


def pme(coords, box, q, alpha, K):
    """Rank-0 PME reciprocal energy (incl. self term), dE/dx and dE/dq = phi.

    Restates ``torchff/pme_ref.py:11-469`` + ``torchff/pme.py:95-126`` for rank 0:
    spread Q, S = FFT(Q), Phi = IFFT(C S / theta^2) with C(k) = 4 pi exp(-k^2/4a^2)/(V k^2)
    and C(0) = 0, phi_i = sum_g theta_i(g) Phi(g) - 2 a q_i / sqrt(pi),
    E = 1/2 sum_i q_i phi_i. Units are those of the reference (e^2/nm); callers scale by
    the Coulomb prefactor.
    Returns E, dE/dx (N,3), dE/dq (N,), and the potential grid Phi.
    """
    coords = np.asarray(coords, np.float64)
    q = np.asarray(q, np.float64)
    n = coords.shape[0]
    recip, m0, val, der, shifts = _pme_stencil(coords, box, K)
    idx = (m0[:, :, None] + shifts[None, None, :]) % K                # (N, 3, 6)
    w3 = (val[:, 0, :, None, None] * val[:, 1, None, :, None] * val[:, 2, None, None, :])
    flat = (idx[:, 0, :, None, None] * K * K + idx[:, 1, None, :, None] * K
            + idx[:, 2, None, None, :])                                # (N,6,6,6)
    grid = np.zeros(K * K * K)
    np.add.at(grid, flat.reshape(n, -1), (q[:, None, None, None] * w3).reshape(n, -1))
    grid = grid.reshape(K, K, K)
    S = np.fft.fftn(grid)
    f = signed_frequency(K).astype(np.float64)
    mx, my, mz = np.meshgrid(f, f, f, indexing="ij")
    box_inv = np.linalg.inv(box)
    kvec = 2.0 * np.pi * (np.stack([mx, my, mz], -1) @ box_inv.T)    # k_c = 2 pi sum_d m_d inv(box)[c, d]
    ksq = np.sum(kvec * kvec, -1)
    vol = abs(np.linalg.det(box))
    th = bspline_moduli(K)
    theta = th[:, None, None] * th[None, :, None] * th[None, None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        C = 4.0 * np.pi / vol / ksq * np.exp(-ksq / (4.0 * alpha * alpha))
    C[0, 0, 0] = 0.0
    phik = C * S / (theta * theta)
    Phi = np.real(np.fft.ifftn(phik, norm="forward"))
    loc = Phi.reshape(-1)[flat.reshape(n, -1)].reshape(n, 6, 6, 6)
    phi = np.sum(loc * w3, axis=(1, 2, 3))
    # d theta / d u_d, then du_d/dr = -recip[d, :]
    gu = np.stack(
        [
            np.sum(loc * der[:, 0, :, None, None] * val[:, 1, None, :, None] * val[:, 2, None, None, :], (1, 2, 3)),
            np.sum(loc * val[:, 0, :, None, None] * der[:, 1, None, :, None] * val[:, 2, None, None, :], (1, 2, 3)),
            np.sum(loc * val[:, 0, :, None, None] * val[:, 1, None, :, None] * der[:, 2, None, None, :], (1, 2, 3)),
        ],
        1,
    )
    dphi_dr = -(gu @ recip)
    gx = q[:, None] * dphi_dr
    pot = phi - 2.0 * alpha / math.sqrt(math.pi) * q
    energy = 0.5 * float(np.sum(q * pot))
    return energy, gx, pot, Phi


# ---------------------------------------------------------------------------
# bonded terms (flexible water)
# ---------------------------------------------------------------------------


def harmonic_bond(coords, bonds, b0, k):
    """E = sum 1/2 k (r - b0)^2 over bonds (i, j), r = |x_j - x_i| with no periodic image.

    Restates ``compute_harmonic_bond_energy_ref`` (``torchff/bond.py:34-43``). Returns E,
    dE/dx (N,3), dE/db0 (M,), dE/dk (M,).
    """
    x = np.asarray(coords, np.float64)
    b = np.asarray(bonds, np.int64)
    b0 = np.asarray(b0, np.float64)
    k = np.asarray(k, np.float64)
    d = x[b[:, 1]] - x[b[:, 0]]
    r = np.linalg.norm(d, axis=1)
    dr = r - b0
    e = float(np.sum(0.5 * k * dr * dr))
    g = (k * dr / r)[:, None] * d  # dE/dx_j; dE/dx_i = -g
    gx = np.zeros_like(x)
    np.add.at(gx, b[:, 1], g)
    np.add.at(gx, b[:, 0], -g)
    return e, gx, -k * dr, 0.5 * dr * dr


def angles(coords, triples):
    """Angle at the central atom j of each (i, j, k), radians (``torchff/angle.py:8-34``)."""
    x = np.asarray(coords, np.float64)
    a = np.asarray(triples, np.int64)
    v1 = x[a[:, 0]] - x[a[:, 1]]
    v2 = x[a[:, 2]] - x[a[:, 1]]
    c = np.sum(v1 * v2, 1) / (np.linalg.norm(v1, axis=1) * np.linalg.norm(v2, axis=1))
    return np.arccos(np.clip(c, -1.0, 1.0))


def harmonic_angle(coords, triples, theta0, k):
    """E = sum 1/2 k (theta - theta0)^2 (``compute_harmonic_angle_energy_ref``,
    ``torchff/angle.py:103-112``). Returns E, dE/dx, dE/dtheta0, dE/dk.

    With u = v1/|v1|, w = v2/|v2| and c = u.w: dtheta/dv1 = -(w - c u) / (|v1| sin theta),
    dtheta/dv2 = -(u - c w) / (|v2| sin theta).
    """
    x = np.asarray(coords, np.float64)
    a = np.asarray(triples, np.int64)
    th0 = np.asarray(theta0, np.float64)
    k = np.asarray(k, np.float64)
    v1 = x[a[:, 0]] - x[a[:, 1]]
    v2 = x[a[:, 2]] - x[a[:, 1]]
    n1 = np.linalg.norm(v1, axis=1)
    n2 = np.linalg.norm(v2, axis=1)
    u = v1 / n1[:, None]
    w = v2 / n2[:, None]
    c = np.clip(np.sum(u * w, 1), -1.0, 1.0)
    th = np.arccos(c)
    s = np.sqrt(np.maximum(1.0 - c * c, 1e-300))
    dth = th - th0
    e = float(np.sum(0.5 * k * dth * dth))
    f = k * dth
    g1 = (f / (n1 * s))[:, None] * -(w - c[:, None] * u)
    g3 = (f / (n2 * s))[:, None] * -(u - c[:, None] * w)
    gx = np.zeros_like(x)
    np.add.at(gx, a[:, 0], g1)
    np.add.at(gx, a[:, 2], g3)
    np.add.at(gx, a[:, 1], -g1 - g3)
    return e, gx, -f, 0.5 * dth * dth


# ---------------------------------------------------------------------------
# TIP3P-style composition (examples/tip3p/model.py:100-133, nonbonded part)
# ---------------------------------------------------------------------------


def fixed_charge_energy(coords, box, charges, sigma_table, epsilon_table, atom_types,
                        nblist_excl, coulomb_excl, cutoff, alpha, K, prefactor,
                        pairs=None):
    """LJ (type tables) + real-space Ewald with exclusion correction + prefactor * PME.

    Mirrors the nonbonded part of ``Tip3pTorchFF.energy_components``
    (``examples/tip3p/model.py:100-123``). Returns a dict of energy components,
    the total dE/dx and dE/dq, and the neighbour pairs used.
    """
    n = coords.shape[0]
    if pairs is None:
        rp, col = exclusions_coo_to_csr(nblist_excl, n)
        pairs = nblist_pairs(coords, box, cutoff, rp, col, include_self=False)
    e_lj, gx_lj, _, _ = lennard_jones(coords, pairs, box, sigma_table, epsilon_table, cutoff, atom_types)
    e_c, gx_c, gq_c = ewald_real(coords, box, pairs, charges, cutoff, alpha, prefactor, coulomb_excl)
    e_p, gx_p, pot, _ = pme(coords, box, charges, alpha, K)
    total = e_lj + e_c + prefactor * e_p
    return {
        "lj": e_lj,
        "coul_real": e_c,
        "pme_raw": e_p,
        "total": total,
        "grad_coords": gx_lj + gx_c + prefactor * gx_p,
        "grad_charges": gq_c + prefactor * pot,
        "pairs": pairs,
    }


# ---------------------------------------------------------------------------
# large orthorhombic boxes: the same energy and forces without an O(N^2) pair list
# ---------------------------------------------------------------------------


def _real_pair_terms(r, qq, sig, eps, alpha, prefactor):
    """Per pair: LJ 12-6 (torchff/vdw.py:86-111) + prefactor q_i q_j erfc(a r)/r
    (torchff/multipoles.py:244-341, rank 0) and dE/dr."""
    e_lj, de_lj, _, _ = _lj_terms(r, np.where(sig > 0, sig, 1.0), eps)
    u = alpha * r
    ec = _erfc(u)
    e_c = prefactor * qq * ec / r
    de_c = prefactor * qq * (-ec / r**2 - (2.0 * alpha / math.sqrt(math.pi)) * np.exp(-u * u) / r)
    return e_lj + e_c, de_lj + de_c


def real_space_cells(coords, box, q, atom_types, sigma_table, epsilon_table, coulomb_excl, cutoff, alpha,
                     prefactor):
    """Total real-space energy (LJ with type tables + Ewald real space with the erfc-1
    exclusion correction) of an orthorhombic box with at least 3 cells of edge >= cutoff per
    axis, by cell binning: every pair within the cutoff is visited once through the cell
    and its 13 forward neighbour cells. Same sums as ``lennard_jones`` + ``ewald_real`` over
    the half neighbour list (``torchff/nblist.py:137-140``, exclusions removed), with the
    excluded pairs' correction of ``torchff/multipoles.py:312-341``."""
    coords = np.asarray(coords, np.float64)
    L = np.diag(np.asarray(box, np.float64))
    nc = np.floor(L / cutoff).astype(np.int64)
    assert np.all(nc >= 3) and np.allclose(box, np.diag(L)), "orthorhombic box, >= 3 cells per axis"
    frac = coords / L
    frac -= np.floor(frac)
    cidx = np.minimum((frac * nc).astype(np.int64), nc - 1)
    flat = (cidx[:, 0] * nc[1] + cidx[:, 1]) * nc[2] + cidx[:, 2]
    order = np.argsort(flat, kind="stable")
    start = np.searchsorted(flat[order], np.arange(nc.prod() + 1))
    x = coords[order]
    qs = np.asarray(q, np.float64)[order]
    ts = np.asarray(atom_types)[order]
    offs = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1) if (a, b, c) > (0, 0, 0)]
    rc2 = cutoff * cutoff
    energy = 0.0
    for cx in range(nc[0]):
        for cy in range(nc[1]):
            for cz in range(nc[2]):
                c0 = (cx * nc[1] + cy) * nc[2] + cz
                a = np.arange(start[c0], start[c0 + 1])
                for off in [(0, 0, 0)] + offs:
                    c1 = (((cx + off[0]) % nc[0]) * nc[1] + (cy + off[1]) % nc[1]) * nc[2] + (cz + off[2]) % nc[2]
                    b = np.arange(start[c1], start[c1 + 1])
                    d = x[a][:, None, :] - x[b][None, :, :]
                    d -= L * np.floor(d / L + 0.5)
                    r2 = np.einsum("abk,abk->ab", d, d)
                    m = r2 <= rc2
                    if off == (0, 0, 0):
                        m &= a[:, None] < b[None, :]
                    ia, ib = np.nonzero(m)
                    if ia.size == 0:
                        continue
                    i, j = a[ia], b[ib]
                    r = np.sqrt(r2[ia, ib])
                    e, _ = _real_pair_terms(r, qs[i] * qs[j], sigma_table[ts[i], ts[j]], epsilon_table[ts[i], ts[j]],
                                            alpha, prefactor)
                    energy += float(np.sum(e))
    # excluded pairs: take out the pair terms counted above, add the correction
    ex = np.asarray(coulomb_excl, np.int64)
    qv = np.asarray(q, np.float64)
    tv = np.asarray(atom_types)
    d = min_image(coords[ex[:, 0]] - coords[ex[:, 1]], box)
    r = np.sqrt(np.einsum("ab,ab->a", d, d))
    m = r <= cutoff
    i, j, r = ex[m, 0], ex[m, 1], r[m]
    e_in, _ = _real_pair_terms(r, qv[i] * qv[j], sigma_table[tv[i], tv[j]], epsilon_table[tv[i], tv[j]], alpha,
                               prefactor)
    corr = prefactor * qv[i] * qv[j] * (_erfc(alpha * r) - 1.0) / r
    return energy - float(np.sum(e_in)) + float(np.sum(corr))


def real_space_grad_subset(coords, box, q, atom_types, sigma_table, epsilon_table, coulomb_excl, cutoff, alpha,
                           prefactor, subset, chunk: int = 16):
    """dE/dx of the real-space energy of ``real_space_cells`` for the atoms ``subset``, from
    their distances to every atom (minimum image of an orthorhombic box)."""
    coords = np.asarray(coords, np.float64)
    qv = np.asarray(q, np.float64)
    tv = np.asarray(atom_types)
    L = np.diag(np.asarray(box, np.float64))
    ex = np.asarray(coulomb_excl, np.int64)
    subset = np.asarray(subset, np.int64)
    out = np.zeros((subset.size, 3))
    for c0 in range(0, subset.size, chunk):
        s = subset[c0:c0 + chunk]
        d = coords[s][:, None, :] - coords[None, :, :]
        d -= L * np.floor(d / L + 0.5)
        r2 = np.einsum("abk,abk->ab", d, d)
        m = (r2 <= cutoff * cutoff) & (np.arange(coords.shape[0])[None, :] != s[:, None])
        for k_, a in enumerate(s):
            partners = np.concatenate([ex[ex[:, 0] == a, 1], ex[ex[:, 1] == a, 0]])
            m[k_, partners] = False
        ia, jb = np.nonzero(m)
        r = np.sqrt(r2[ia, jb])
        i = s[ia]
        _, dedr = _real_pair_terms(r, qv[i] * qv[jb], sigma_table[tv[i], tv[jb]], epsilon_table[tv[i], tv[jb]],
                                   alpha, prefactor)
        g = (dedr / r)[:, None] * d[ia, jb]
        np.add.at(out, c0 + ia, g)
        for k_, a in enumerate(s):   # excluded partners: the erfc-1 correction only
            partners = np.concatenate([ex[ex[:, 0] == a, 1], ex[ex[:, 1] == a, 0]])
            dd = min_image(coords[a] - coords[partners], box)
            rr = np.sqrt(np.einsum("ab,ab->a", dd, dd))
            keep = rr <= cutoff
            dd, rr, p = dd[keep], rr[keep], partners[keep]
            u = alpha * rr
            damp = _erfc(u) - 1.0
            dfdr = -damp / rr**2 - (2.0 * alpha / math.sqrt(math.pi)) * np.exp(-u * u) / rr
            out[c0 + k_] += np.sum((prefactor * qv[a] * qv[p] * dfdr / rr)[:, None] * dd, axis=0)
    return out


def pme_subset(coords, box, q, alpha, K, subset):
    """``pme`` (energy incl. self term) with dE/dx gathered for the atoms ``subset`` only;
    the charge grid is spread from every atom with a weighted bincount (large N)."""
    coords = np.asarray(coords, np.float64)
    q = np.asarray(q, np.float64)
    n = coords.shape[0]
    grid = np.zeros(K * K * K)
    for c0 in range(0, n, 65536):
        sl = slice(c0, min(n, c0 + 65536))
        _, m0, val, _, shifts = _pme_stencil(coords[sl], box, K)
        idx = (m0[:, :, None] + shifts[None, None, :]) % K
        w3 = val[:, 0, :, None, None] * val[:, 1, None, :, None] * val[:, 2, None, None, :]
        flat = idx[:, 0, :, None, None] * K * K + idx[:, 1, None, :, None] * K + idx[:, 2, None, None, :]
        grid += np.bincount(flat.reshape(-1), weights=(q[sl, None, None, None] * w3).reshape(-1), minlength=K ** 3)
    grid = grid.reshape(K, K, K)
    S = np.fft.fftn(grid)
    f = signed_frequency(K).astype(np.float64)
    mx, my, mz = np.meshgrid(f, f, f, indexing="ij")
    kvec = 2.0 * np.pi * (np.stack([mx, my, mz], -1) @ np.linalg.inv(box).T)
    ksq = np.sum(kvec * kvec, -1)
    vol = abs(np.linalg.det(box))
    th = bspline_moduli(K)
    theta = th[:, None, None] * th[None, :, None] * th[None, None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        C = 4.0 * np.pi / vol / ksq * np.exp(-ksq / (4.0 * alpha * alpha))
    C[0, 0, 0] = 0.0
    Phi = np.real(np.fft.ifftn(C * S / (theta * theta), norm="forward"))
    energy = 0.5 * float(np.sum(grid * Phi)) - alpha / math.sqrt(math.pi) * float(np.sum(q * q))
    subset = np.asarray(subset, np.int64)
    recip, m0, val, der, shifts = _pme_stencil(coords[subset], box, K)
    idx = (m0[:, :, None] + shifts[None, None, :]) % K
    flat = idx[:, 0, :, None, None] * K * K + idx[:, 1, None, :, None] * K + idx[:, 2, None, None, :]
    loc = Phi.reshape(-1)[flat]
    gu = np.stack([
        np.sum(loc * der[:, 0, :, None, None] * val[:, 1, None, :, None] * val[:, 2, None, None, :], (1, 2, 3)),
        np.sum(loc * val[:, 0, :, None, None] * der[:, 1, None, :, None] * val[:, 2, None, None, :], (1, 2, 3)),
        np.sum(loc * val[:, 0, :, None, None] * val[:, 1, None, :, None] * der[:, 2, None, None, :], (1, 2, 3)),
    ], 1)
    return energy, q[subset, None] * (-(gu @ recip))
