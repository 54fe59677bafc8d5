"""Banded-matrix arithmetic and band-operator coefficients (oracle).

Restates:
  mod_bandmat.f90:65-155    LUDCMPB  (unpivoted band LU, batched)
  mod_bandmat.f90:320-401   LUBKSBB  (forward/back substitution)
  mod_bandmat.f90:792-830   BANDAUX  (per-system sizes; here each system is
                                       solved on its own leading block, which
                                       is what BANDAUX's bookkeeping amounts to)
  mod_bandmat.f90:1111-1153 BANMULR  (band x vector)
  mod_bandmat.f90:1288-1345 BANBANMUL (band x band -> band)
  mod_bandmat.f90:832-938   MR_BAN_MUL / VR_BAN_MUL (matrix x band)
  mod_lin_legendre.f90:910-981    BAND_LOGLEG_XM
  mod_lin_legendre.f90:1166-1237  BAND_LOGLEG_XP
  mod_lin_legendre.f90:1419-1489  BAND_LOGLEG_X
  mod_lin_legendre.f90:1683-1757  BAND_LOGLEG_XXDX
  mod_lin_legendre.f90:1986-2092  BAND_LOGLEG_RAT_DEL2H

Band storage follows the reference: BAND(i, j) multiplies x(i + j - c), with
c the 0-based column of the main diagonal.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import numpy as np


def banmul(band, c, x):
    """y = BAND * x (BANMULR semantics; x shape (N, ...), band shape (N, w))."""
    n = x.shape[0]
    y = np.zeros_like(x, dtype=np.result_type(band, x))
    ext = (slice(None),) + (None,) * (x.ndim - 1)
    for j in range(band.shape[1]):
        s = j - c
        c0, c1 = max(0, -s), min(n, n - s)
        if c1 <= c0:
            continue
        y[c0:c1] += band[c0:c1, j][ext] * x[c0 + s:c1 + s]
    return y


def mat_banmul(mat, band, c):
    """MAT * BAND with BAND applied as an N x N matrix (MR_BAN_MUL)."""
    n = band.shape[0]
    full = band_to_full(band, c, n)
    return mat @ full


def band_to_full(band, c, n=None):
    """MTRX: band form -> dense (n x n)."""
    if n is None:
        n = band.shape[0]
    full = np.zeros((n, n), dtype=band.dtype)
    for i in range(n):
        for j in range(band.shape[1]):
            col = i + j - c
            if 0 <= col < n:
                full[i, col] = band[i, j]
    return full


def banbanmul(A, ac, B, bc):
    """BANBANMUL(A, AC, B, BC), mod_bandmat.f90:1288-1345 -> (C, cc)."""
    nn = A.shape[0]
    aw, bw = A.shape[1], B.shape[1]
    C = np.zeros((nn, aw + bw - 1), dtype=np.result_type(A, B))
    for i in range(aw):
        as_ = i - ac
        a0, a1 = max(0, -as_), min(nn, nn - as_)
        for j in range(bw):
            k = i + j
            bs = j - bc
            b0, b1 = max(0, -bs), min(nn, nn - bs)
            c0, c1 = max(a0, b0 - as_), min(a1, b1 - as_)
            if c1 > c0:
                C[c0:c1, k] += A[c0:c1, i] * B[c0 + as_:c1 + as_, j]
    return C, ac + bc


def band_lu_solve(bands, c, rhs, sizes=None):
    """LUDCMPB + LUBKSBB: unpivoted banded Gaussian elimination, batched.

    bands : (S, N, w) real, system s uses its leading sizes[s] x sizes[s] block
    rhs   : (S, N) complex, overwritten rows >= sizes[s] are left untouched
    Systems shorter than N are padded with identity rows, which leaves the
    elimination on the leading block unchanged (no coupling across the pad).
    """
    bands = np.array(bands, dtype=np.float64, copy=True)
    x = np.array(rhs, dtype=np.complex128, copy=True)
    S, N, w = bands.shape
    if sizes is None:
        sizes = np.full(S, N)
    sizes = np.asarray(sizes)
    # identity padding + cut the coupling of each leading block to its pad
    for s in range(S):
        ns = int(sizes[s])
        if ns < N:
            bands[s, ns:, :] = 0.0
            bands[s, ns:, c] = 1.0
            for i in range(max(0, ns - w), ns):
                for j in range(w):
                    if i + j - c >= ns:
                        bands[s, i, j] = 0.0
    keep = x.copy()
    lo = c            # number of sub-diagonals
    up = w - c - 1    # number of super-diagonals
    # forward elimination (Doolittle), mirrors LUDCMPB's update order
    for nn in range(N):
        piv = bands[:, nn, c]
        for j in range(1, lo + 1):
            r = nn + j
            if r >= N:
                break
            l = bands[:, r, c - j] / piv
            bands[:, r, c - j] = l
            for i in range(1, up + 1):
                if c - j + i < w:
                    bands[:, r, c - j + i] -= l * bands[:, nn, c + i]
            x[:, r] -= l * x[:, nn]
    # back substitution
    for nn in range(N - 1, -1, -1):
        acc = x[:, nn].copy()
        for i in range(1, up + 1):
            col = nn + i
            if col < N:
                acc -= bands[:, nn, c + i] * x[:, col]
        x[:, nn] = acc / bands[:, nn, c]
    for s in range(S):
        ns = int(sizes[s])
        x[s, ns:] = keep[s, ns:]
    return x


# ----------------------------------------------------------------------
# Band-operator coefficients (normalised with LOGNORM), for order m.
# ----------------------------------------------------------------------

def _lognorm_scale(band, lognorm, offsets):
    ni = band.shape[0]
    if ni <= 1:
        return band
    for col, off in offsets:
        if off < 0:
            d = -off
            if ni > d:
                band[d:ni, col] *= np.exp(lognorm[0:ni - d] - lognorm[d:ni])
        elif off > 0:
            d = off
            if ni > d:
                band[0:ni - d, col] *= np.exp(lognorm[d:ni] - lognorm[0:ni - d])
    return band


def band_xm(ni, m, lognorm):
    """BAND_LOGLEG_XM (1-x)*, mod_lin_legendre.f90:910-981."""
    am = abs(m)
    b = np.zeros((ni, 3))
    nn = np.arange(1, ni + 1)
    n = am + nn - 1.0
    b[:, 0] = np.where(nn - 1 >= 1, -(n - am) / (2 * n - 1.0), 0.0)
    b[:, 1] = 1.0
    b[:, 2] = np.where(nn + 1 <= ni, -(n + am + 1.0) / (2 * n + 3.0), 0.0)
    return _lognorm_scale(b, lognorm, [(0, -1), (2, 1)])


def band_xp(ni, m, lognorm):
    """BAND_LOGLEG_XP (1+x)*, mod_lin_legendre.f90:1166-1237."""
    am = abs(m)
    b = np.zeros((ni, 3))
    nn = np.arange(1, ni + 1)
    n = am + nn - 1.0
    b[:, 0] = np.where(nn - 1 >= 1, (n - am) / (2 * n - 1.0), 0.0)
    b[:, 1] = 1.0
    b[:, 2] = np.where(nn + 1 <= ni, (n + am + 1.0) / (2 * n + 3.0), 0.0)
    return _lognorm_scale(b, lognorm, [(0, -1), (2, 1)])


def band_xxdx(ni, m, lognorm):
    """BAND_LOGLEG_XXDX (1-x^2) d/dx, mod_lin_legendre.f90:1683-1757."""
    am = abs(m)
    b = np.zeros((ni, 3))
    nn = np.arange(1, ni + 1)
    n = am + nn - 1.0
    b[:, 0] = np.where(nn - 1 >= 1, -(n - 1.0) * (n - am) / (2 * n - 1.0), 0.0)
    b[:, 2] = np.where(nn + 1 <= ni, (n + 2.0) * (n + am + 1.0) / (2 * n + 3.0), 0.0)
    return _lognorm_scale(b, lognorm, [(0, -1), (2, 1)])


def band_del2h(ni, m, ell, lognorm):
    """BAND_LOGLEG_RAT_DEL2H (S = 0), mod_lin_legendre.f90:1986-2092."""
    am = abs(m)
    ell2 = ell ** 2.0
    b = np.zeros((ni, 5))
    nn = np.arange(1, ni + 1)
    n = am + nn - 1.0
    b[:, 0] = np.where(nn - 2 >= 1, -(n - am - 1.0) * (n - am) * (n - 2) * (n - 1)
                       / (2 * n - 3.0) / (2 * n - 1.0) / ell2, 0.0)
    b[:, 1] = np.where(nn - 1 >= 1, 2.0 * n * (n - am) * (n - 1) / (2 * n - 1.0) / ell2, 0.0)
    b[:, 2] = (-2.0 * n * (n + 1.0) * (3.0 * n * n + 3 * n - am ** 2 - 2)) / (2 * n - 1.0) / (2 * n + 3.0) / ell2
    b[:, 3] = np.where(nn + 1 <= ni, 2.0 * (n + 1) * (n + am + 1.0) * (n + 2) / (2 * n + 3.0) / ell2, 0.0)
    b[:, 4] = np.where(nn + 2 <= ni, -(n + am + 1.0) * (n + am + 2.0) * (n + 3) * (n + 2)
                       / (2 * n + 3.0) / (2 * n + 5.0) / ell2, 0.0)
    if ni <= 1:
        return b
    _lognorm_scale(b, lognorm, [(1, -1), (3, 1)])
    if ni <= 2:
        return b
    return _lognorm_scale(b, lognorm, [(0, -2), (4, 2)])
