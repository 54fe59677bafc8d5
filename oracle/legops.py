"""Spectral operators on the hot path (oracle).

Restates mod_legops.f90:
  76-133    DELSQH        136-241  IDELSQH (initial condition only)
  371-428   MULXM         680-748  XXDX           751-820  DEL2
  823-1010  IDEL2         1013-1176 IDEL2LN       1204-1354 IHELM
  1409-1592 IHELMP (VISC%SW = 2, with HYPERV of mod_march.f90:1639-1686)
  1727-1786 GRAD          1789-1853 PC2VEL        1856-1919 PC2VOR
  1972-2133 VPRODSUB      2136-2232 VDOTPSUB      2277-2339 VEL2PLN
  2397-2545 PROJECT       2548-2648 EOMUL / OEMUL
Every operator reads the grid's *current* NRCHOPS (the reference's global
CHOPSET state), exactly like the Fortran.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import numpy as np

from .bandmat import (band_del2h, band_lu_solve, band_xm, band_xxdx, banbanmul,
                      banmul, mat_banmul)
from .grid import FFF, PFF, PPP
from .transforms import plnfft, rtran


def _require(A, space, name):
    if A.space != space:
        raise ValueError("%s: INPUT NOT IN SPACE %d" % (name, space))


def _apply_band(g, A, make_band, c):
    """B(:NN,m,k) = BAND_m(:NN) * A(:NN,m,k) for every m, k (MULXM/XXDX pattern)."""
    B = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        band = make_band(nn, mm)
        B.E[:nn, mm, :] = banmul(band, c, A.E[:nn, mm, :])
    g.chopdo(B)
    return B


def delsqh(g, A):
    """DELSQH(A, B), mod_legops.f90:76-133: B = (1-x)^-2 del^2_h A = -n(n+1)/L^2 A."""
    _require(A, FFF, "DELSQH")
    B = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        n = g.M[mm] + np.arange(nn)
        B.E[:nn, mm, :] = -A.E[:nn, mm, :] * (n * (n + 1) / g.ELL2)[:, None]
    g.chopdo(B)
    B.E[0, 0, 0] = A.LN / g.ELL2 / g.NORM0[0]
    return B


def idelsqh(g, B):
    """IDELSQH(B, A), mod_legops.f90:136-241 (log term returned in A.LN)."""
    _require(B, FFF, "IDELSQH")
    A = g.alloc(FFF)
    A.LN = float((B.E[0, 0, 0] * g.NORM0[0] * g.ELL2).real)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        for i in range(nn):
            n = int(g.M[mm]) + i
            if n == 0:
                A.E[0, 0, :] = 0.0
            else:
                A.E[i, mm, :] = -B.E[i, mm, :] * (g.ELL2 / (n * (n + 1)))
    A.E[0, 0, :] = A.E[0, 0, :] - g.calcat1(A) / g.AT1[0]
    return A


def mulxm(g, A):
    """MULXM(A, B), mod_legops.f90:371-428: B = (1-x) A."""
    _require(A, FFF, "MULXM")
    return _apply_band(g, A, lambda nn, mm: band_xm(nn, g.M[mm], g.LOGNORM[:, mm]), 1)


def xxdx(g, A):
    """XXDX(A, B), mod_legops.f90:680-748: B = (1-x^2) dA/dx = r dA/dr."""
    _require(A, FFF, "XXDX")
    B = _apply_band(g, A, lambda nn, mm: band_xxdx(nn, g.M[mm], g.LOGNORM[:, mm]), 1)
    B.E[0, 0, 0] += A.LN / g.NORM0[0]
    B.E[1, 0, 0] += A.LN / g.NORM0[1]
    return B


def del2(g, A):
    """DEL2(A, B), mod_legops.f90:751-820: B = del^2 A (incl. -k^2, log term)."""
    _require(A, FFF, "DEL2")
    B = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        band = band_del2h(nn, g.M[mm], g.ELL, g.LOGNORM[:, mm])
        a = A.E[:nn, mm, :]
        B.E[:nn, mm, :] = banmul(band, 2, a) - (g.AK[mm, :] ** 2)[None, :] * a
    g.chopdo(B)
    B.E[0, 0, 0] += 4.0 / 3 * A.LN / g.ELL2 / g.NORM0[0]
    B.E[1, 0, 0] -= 2.0 * A.LN / g.ELL2 / g.NORM0[1]
    B.E[2, 0, 0] += 2.0 / 3 * A.LN / g.ELL2 / g.NORM0[2]
    return B


def _solve_m_nonzero(g, A, alpha=0.0, mstart=1):
    """Penta-diagonal (del^2_h - k^2 - alpha) solves for m >= mstart, all k."""
    K = A.E.shape[2]
    for mm in range(mstart, A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        band0 = band_del2h(nn, g.M[mm], g.ELL, g.LOGNORM[:, mm])
        band0[:, 2] -= alpha
        bands = np.repeat(band0[None, :, :], K, axis=0)
        bands[:, :, 2] -= (g.AK[mm, :] ** 2)[:, None]
        A.E[:nn, mm, :] = band_lu_solve(bands, 2, A.E[:nn, mm, :].T).T
    return A


def idel2(g, B, LN=None):
    """IDEL2(B, A, LN), mod_legops.f90:823-1010 (7-band m=0, log-term BC)."""
    _require(B, FFF, "IDEL2")
    A = g.copy0(B)
    A.LN = 0.0
    K = A.E.shape[2]
    nn = int(g.NRCHOPS[0])
    np_ = nn + 1
    d0 = np.zeros((np_, 7))
    d0[:, 1:6] = band_del2h(np_, g.M[0], g.ELL, g.LOGNORM[:, 0])
    op = np.repeat(d0[None, :, :], K, axis=0)
    op[:, :, 3] -= (g.AK[0, :] ** 2)[:, None]
    # m = 0, k = 0: log-term column, then shift the system by one row (917-932)
    n0 = g.NORM0
    o = op[0]
    o[0, 3] += 4.0 / 3 / g.ELL2
    o[1, 2] -= 2 * n0[0] / n0[1] / g.ELL2
    o[2, 1] += 2.0 / 3 * n0[0] / n0[2] / g.ELL2
    o[1:np_, 0:5] = o[0:np_ - 1, 1:6].copy()
    o[:, 5:7] = 0
    o[0, :] = 0
    o[0, 3] = 1
    A.E[1:nn, 0, 0] = A.E[0:nn - 1, 0, 0].copy()
    A.E[0, 0, 0] = (LN / n0[0]) if LN is not None else 0.0
    A.E[:nn, 0, :] = band_lu_solve(op[:, :nn, :], 3, A.E[:nn, 0, :].T).T
    _solve_m_nonzero(g, A, 0.0, 1)
    if LN is not None:
        A.LN = float(A.E[0, 0, 0].real * n0[0])
    g.chopdo(A)
    nr = g.NRCHOP
    A.E[0, 0, :] = A.E[0, 0, :] - (g.AT1[:nr] @ A.E[:nr, 0, :]) / g.AT1[0]
    return A


def idel2ln(g, B):
    """IDEL2LN(B, A), mod_legops.f90:1013-1176 (log term solved into A.LN)."""
    _require(B, FFF, "IDEL2LN")
    A = g.copy0(B)
    A.LN = 0.0
    K = A.E.shape[2]
    nn = int(g.NRCHOPS[0])
    np_ = nn + 1
    d0 = band_del2h(np_, g.M[0], g.ELL, g.LOGNORM[:, 0])
    op = np.repeat(d0[None, :, :], K, axis=0)
    op[:, :, 2] -= (g.AK[0, :] ** 2)[:, None]
    n0 = g.NORM0
    op[0, 0, 2] += 4.0 / 3 / g.ELL2
    op[0, 1, 1] -= 2 * n0[0] / n0[1] / g.ELL2
    op[0, 2, 0] += 2.0 / 3 * n0[0] / n0[2] / g.ELL2
    A.E[:nn, 0, :] = band_lu_solve(op[:, :nn, :], 2, A.E[:nn, 0, :].T).T
    A.LN = float(A.E[0, 0, 0].real * n0[0])
    A.E[0, 0, 0] = 0
    _solve_m_nonzero(g, A, 0.0, 1)
    g.chopdo(A)
    nr = g.NRCHOP
    A.E[0, 0, :] = A.E[0, 0, :] - (g.AT1[:nr] @ A.E[:nr, 0, :]) / g.AT1[0]
    return A


def ihelm(g, B, alp):
    """IHELM(B, A, ALP), mod_legops.f90:1204-1354: A = (del^2 - alp)^-1 B.

    m = 0 is solved as (H * XM) y = rhs on NN-1 rows, A = XM * y (y_NN = 0);
    the log term is A.LN = -B.LN/alp and its del^2 is moved to the rhs.
    """
    _require(B, FFF, "IHELM")
    if alp == 0.0:
        raise ValueError("IHELM: ALP CAN'T BE ZERO")
    A = g.copy0(B)
    A.LN = -B.LN / alp
    n0 = g.NORM0
    A.E[0, 0, 0] -= A.LN * (4.0 / 3 / g.ELL2) / n0[0]
    A.E[1, 0, 0] -= A.LN * (-2 / n0[1] / g.ELL2)
    A.E[2, 0, 0] -= A.LN * (+2.0 / 3 / n0[2] / g.ELL2)
    K = A.E.shape[2]
    nn = int(g.NRCHOPS[0])
    np_ = nn + 1
    nm = nn - 1
    xm = band_xm(np_, g.M[0], g.LOGNORM[:, 0])
    h0 = band_del2h(np_, g.M[0], g.ELL, g.LOGNORM[:, 0])
    h0[:, 2] -= alp
    ops = np.zeros((K, np_, 7))
    for kk in range(K):
        h = h0.copy()
        h[:, 2] -= g.AK[0, kk] ** 2
        ops[kk], _ = banbanmul(h, 2, xm, 1)
    y = band_lu_solve(ops[:, :nm, :], 3, A.E[:nm, 0, :].T).T
    A.E[:nm, 0, :] = y
    A.E[nn - 1, 0, :] = 0
    A.E[:nn, 0, :] = banmul(xm[:nn, :], 1, A.E[:nn, 0, :])
    _solve_m_nonzero(g, A, alp, 1)
    g.chopdo(A)
    return A


def ihelmp(g, B, p, alp, nu=0.0):
    """IHELMP(P, B, A, ALP, NUIN), mod_legops.f90:1409-1592:
    A = (DEL^P + NU DEL^2 - ALP)^-1 B, P even in 4..14.

    The log term: A.LN = -B.LN / ALP and its contribution AL + NU AL2 moves
    to the (m, k) = (0, 0) right-hand side, AL2 the DEL2 image of LN(-log(1-x))
    on the first three rows and AL = DEL2H^(P/2-1) AL2 (BANMUL, 1444-1466).
    Per m the band of (DEL2H - k^2)^(P/2) is expanded binomially from the
    powers DEL2H^q (BANBANMUL at size NN + P) exactly as the reference writes
    each P out (1476-1573), plus NU (DEL2H - k^2) - ALP, and solved by the
    unpivoted band LU on the leading NN = NRCHOPS(m) rows; then the far-field
    fix A(1,1,:) -= CALCAT1(A) / PF(1,1,1) and CHOPDO.
    """
    _require(B, FFF, "IHELMP")
    if alp == 0.0:
        raise ValueError("IHELMP: ALP CANNOT BE ZERO.")
    if p < 4 or p > 14 or p % 2:
        raise ValueError("P OUT OF RANGE. P=%d" % p)
    hp = p // 2
    A = g.copy0(B)
    A.LN = -B.LN / alp
    nrc = int(g.NRCHOP)
    n0 = g.NORM0
    al2 = np.zeros(nrc)
    al2[0] = A.LN * (4.0 / 3 / g.ELL2) / n0[0]
    al2[1] = A.LN * (-2 / n0[1] / g.ELL2)
    al2[2] = A.LN * (+2.0 / 3 / n0[2] / g.ELL2)
    al = al2.copy()
    d2 = band_del2h(nrc, g.M[0], g.ELL, g.LOGNORM[:, 0])
    for _ in range(4, p + 1, 2):
        al = banmul(d2, 2, al)
    A.E[:nrc, 0, 0] = A.E[:nrc, 0, 0] - al - nu * al2
    K = A.E.shape[2]
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        np_ = nn + p
        d1 = band_del2h(np_, g.M[mm], g.ELL, g.LOGNORM[:, mm])
        dq = {1: d1}
        for q in range(2, hp + 1):
            dq[q], _ = banbanmul(dq[q - 1], 2 * q - 2, d1, 2)
        bands = np.zeros((K, nn, 2 * p + 1))
        for kk in range(K):
            k2 = g.AK[mm, kk] ** 2
            h = np.zeros((np_, 2 * p + 1))
            h[:, :] = dq[hp]
            c = 1.0
            for j in range(1, hp + 1):
                c = c * (-k2)
                binom = 1.0
                for q in range(1, j + 1):
                    binom = binom * (hp - q + 1) / q
                q = hp - j
                if q == 0:
                    h[:, p] += c
                else:
                    h[:, p - 2 * q:p + 2 * q + 1] += (binom * c) * dq[q]
            dv = d1.copy()
            dv[:, 2] -= k2
            h[:nn, p - 2:p + 3] += nu * dv[:nn, :]
            h[:nn, p] -= alp
            bands[kk] = h[:nn]
        A.E[:nn, mm, :] = band_lu_solve(bands, p, A.E[:nn, mm, :].T).T
    A.E[0, 0, :] = A.E[0, 0, :] - g.calcat1(A) / g.PF[0, 0, 0]
    g.chopdo(A)
    return A


def hyperv(g, A, nu, nup, p, dt):
    """HYPERV(A, NU, NUP, P, DT, WK), mod_march.f90:1639-1686: returns the new A,
    IHELMP(P, ALP A, A, -ALP, BET), ALP = (-1)^(P/2) / (DT NUP), BET = -(-1)^(P/2) NU / NUP."""
    if nup == 0.0:
        raise ValueError("HYPERV: NUP CAN'T BE ZERO")
    _require(A, FFF, "HYPERV")
    ph = p // 2
    alp = 1 / dt / nup * (-1) ** ph
    bet = -(-1) ** ph * nu / nup
    WK = A.copy()
    WK.E = alp * A.E
    WK.LN = alp * A.LN
    return ihelmp(g, WK, p, -alp, bet)


def grad(g, A):
    """GRAD(A), mod_legops.f90:1727-1786 -> (r dA/dr, dA/dphi, dA/dz)."""
    RR = xxdx(g, A)
    RP = g.alloc(FFF)
    GZ = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        mv = g.M[mm]
        RP.E[:nn, mm, :] = 1j * mv * A.E[:nn, mm, :]
        GZ.E[:nn, mm, :] = 1j * g.AK[mm, :][None, :] * A.E[:nn, mm, :]
    return RR, RP, GZ


def pc2vel(g, PSI, CHI):
    """PC2VEL(PSI, CHI), mod_legops.f90:1789-1853 -> (r u_r, r u_phi, u_z)."""
    RUR = xxdx(g, CHI)
    RUP = xxdx(g, PSI)
    for mm in range(PSI.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        mv = g.M[mm]
        kv = g.AK[mm, :][None, :]
        RUR.E[:nn, mm, :] = 1j * mv * PSI.E[:nn, mm, :] + (1j * kv) * RUR.E[:nn, mm, :]
        RUP.E[:nn, mm, :] = -RUP.E[:nn, mm, :] - (mv * kv) * CHI.E[:nn, mm, :]
    UZ = delsqh(g, CHI)
    W = mulxm(g, UZ)
    UZ = mulxm(g, W)
    UZ.E = -UZ.E
    return RUR, RUP, UZ


def pc2vor(g, PSI, CHI):
    """PC2VOR(PSI, CHI), mod_legops.f90:1856-1919 -> (r w_r, r w_phi, w_z)."""
    OZ = del2(g, CHI)
    ROR = xxdx(g, PSI)
    ROP = xxdx(g, OZ)
    for mm in range(PSI.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        mv = g.M[mm]
        kv = g.AK[mm, :][None, :]
        ROR.E[:nn, mm, :] = -1j * mv * OZ.E[:nn, mm, :] + 1j * kv * ROR.E[:nn, mm, :]
        ROP.E[:nn, mm, :] = ROP.E[:nn, mm, :] - (kv * mv) * PSI.E[:nn, mm, :]
    OZ = delsqh(g, PSI)
    W = mulxm(g, OZ)
    OZ = mulxm(g, W)
    OZ.E = -OZ.E
    return ROR, ROP, OZ


def vprodsub(g, RUR, RUP, UZ, ROR, ROP, OZ):
    """VPRODSUB cross product, mod_legops.f90:2105-2130 (NADD = 0, no monitor).

    (ROR, ROP, OZ) <- (A2 B3 - A3 B2, A3 B1 - A1 B3, (A1 B2 - A2 B1)/r^2),
    applied separately to the real and the imaginary (packed) samples.
    """
    nr, nth = g.NR, g.NTH
    sl = (slice(0, nr), slice(0, nth), slice(None))

    def parts(X):
        v = X.E[sl]
        return v.real, v.imag

    a1, c1 = parts(RUR)
    a2, c2 = parts(RUP)
    a3, c3 = parts(UZ)
    b1, d1 = parts(ROR)
    b2, d2 = parts(ROP)
    b3, d3 = parts(OZ)
    r2 = (g.R[:nr] ** 2.0)[:, None, None]
    nr_ = (a2 * b3 - a3 * b2) + 1j * (c2 * d3 - c3 * d2)
    np_ = (a3 * b1 - a1 * b3) + 1j * (c3 * d1 - c1 * d3)
    nz_ = ((a1 * b2 - a2 * b1) + 1j * (c1 * d2 - c2 * d1)) / r2
    ROR.E[sl] = nr_
    ROP.E[sl] = np_
    OZ.E[sl] = nz_


def vdotpsub(g, RAR, RAP, AZ, RBR, RBP, BZ):
    """VDOTPSUB, mod_legops.f90:2136-2232: (A1 B1 + A2 B2)/r^2 + A3 B3 per part."""
    nr, nth = g.NR, g.NTH
    sl = (slice(0, nr), slice(0, nth), slice(None))
    out = np.zeros(RAR.E.shape, dtype=np.complex128)
    r2 = (g.R[:nr] ** 2)[:, None, None]
    a1, a2, a3 = RAR.E[sl], RAP.E[sl], AZ.E[sl]
    b1, b2, b3 = RBR.E[sl], RBP.E[sl], BZ.E[sl]
    re = (a1.real * b1.real + a2.real * b2.real) / r2 + a3.real * b3.real
    im = (a1.imag * b1.imag + a2.imag * b2.imag) / r2 + a3.imag * b3.imag
    out[sl] = re + 1j * im
    return out


def vel2pln(g, RUP, PSI, LN=None):
    """VEL2PLN(RUP, PSI, LN), mod_legops.f90:2277-2339.  RUP in PFF, in place.

    Extracts PSI.LN = -RUP_00(r -> inf)/2 from the (m,k) = (0,0) line,
    removes -LN (1 + x) from that line, then overrides PSI.LN with LN.
    """
    _require(RUP, PFF, "VEL2PLN")
    nr, nrh = g.NR, g.NRH
    w = g.W[:nrh]
    line = RUP.E[:, 0, 0]
    be = (line[:nrh] + line[nr - 1:nrh - 1:-1]) * w
    bo = (line[:nrh] - line[nr - 1:nrh - 1:-1]) * w
    nn = int(g.NRCHOPS[0])
    fff = np.zeros(nn, dtype=np.complex128)
    pf = g.PF[:nrh, :, 0]
    fff[0:nn:2] = be @ pf[:, 0:nn:2]
    fff[1:nn:2] = bo @ pf[:, 1:nn:2]
    psi_ln = -float(np.sum(fff.real * np.exp(g.LOGNORM[:nn, 0]))) / 2.0
    be2 = -pf[:, 0] * psi_ln / g.NORM0[0]
    bo2 = -pf[:, 1] * psi_ln / g.NORM0[1]
    line[:nrh] -= (be2 + bo2)
    line[nr - 1:nrh - 1:-1] -= (be2 - bo2)
    PSI.LN = psi_ln if LN is None else float(LN)
    return psi_ln


def eomul(A, B):
    """EOMUL(A, B, C), mod_legops.f90:2548-2598 (even/odd folded GEMM)."""
    nj = B.shape[0]
    njh = A.shape[1]
    be = B[:njh] + B[nj - 1:njh - 1:-1]
    bo = B[:njh] - B[nj - 1:njh - 1:-1]
    C = np.zeros((A.shape[0], B.shape[1]), dtype=np.complex128)
    C[0::2] = A[0::2] @ be
    if A.shape[0] > 1:
        C[1::2] = A[1::2] @ bo
    return C


def oemul(A, B):
    """OEMUL(A, B, C), mod_legops.f90:2601-2648 (odd/even folded GEMM)."""
    nj = B.shape[0]
    njh = A.shape[1]
    be = B[:njh] + B[nj - 1:njh - 1:-1]
    bo = B[:njh] - B[nj - 1:njh - 1:-1]
    C = np.zeros((A.shape[0], B.shape[1]), dtype=np.complex128)
    C[0::2] = A[0::2] @ bo
    C[1::2] = A[1::2] @ be
    return C


def project_weights(g, mm):
    """V, D, T matrices of PROJECT for order index mm (mod_legops.f90:2485-2497)."""
    nrh = g.NRH
    nn = int(g.NRCHOPS[mm])
    mv = int(g.M[mm])
    fff = (1 - g.X[:nrh] ** 2) / g.W[:nrh]
    pf = g.PF[:nrh, :nn + 1, mm]
    pfd = mat_banmul(pf, band_xxdx(nn + 1, mv, g.LOGNORM[:, mm]), 1)
    i = np.arange(1, nn + 1)
    n = np.maximum(1, mv + i - 1)
    den = (n * (n + 1))[:, None] * fff[None, :]
    V = pf[:, :nn].T / den
    D = pfd[:, :nn].T / den
    T = pf[:, :nn].T * g.W[:nrh][None, :]
    return V, D, T


def project(g, RUR, RUP, UZ, LN=None):
    """PROJECT(RUR, RUP, UZ, PSI, CHI, LN), mod_legops.f90:2397-2545.

    Inputs in PPP/FFF/PFF (transformed to PFF in place).  Returns (PSI, W)
    with W = del^2 chi in FFF; far-field fix PSI(1,1,:) -= CALCAT1/AT1(1).
    LN: None (no log-term handling), a number (VEL2PLN with that LN), or
    "psi" for the steppers' PROJECT(..., PSI, W, PSI%LN) call.
    """
    if not (RUR.space == RUP.space == UZ.space):
        raise ValueError("PROJECT: RUR, RUP, UZ MUST BE IN THE SAME SPACE.")
    if RUR.space == PPP:
        for F in (RUR, RUP, UZ):
            plnfft(g, F, -1)
    elif RUR.space == FFF:
        for F in (RUR, RUP, UZ):
            rtran(g, F, 1)
    elif RUR.space != PFF:
        raise ValueError("PROJECT: bad space")
    PSI = g.alloc(FFF)
    CHI = g.alloc(FFF)
    if isinstance(LN, str) and LN == "psi":
        # PROJECT(..., PSI, W, PSI%LN) passes PSI%LN by reference: VEL2PLN
        # zeroes and then writes PSI%LN through the PSI dummy before reading
        # LN back (2317, 2325, 2337), so the caller's log term becomes the
        # value extracted from the far field of RUP.
        PSI.LN = vel2pln(g, RUP, PSI, None)
    elif LN is not None:
        PSI.LN = float(LN)
        vel2pln(g, RUP, PSI, LN)
    nr = g.NR
    for mm in range(RUR.E.shape[1]):
        mv = int(g.M[mm])
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        V, D, T = project_weights(g, mm)
        rur = RUR.E[:nr, mm, :]
        rup = RUP.E[:nr, mm, :]
        uz = UZ.E[:nr, mm, :]
        W1 = eomul(V, rur) if mv != 0 else 0.0
        W2 = oemul(D, rup)
        PSI.E[:nn, mm, :] = -(1j * mv) * W1 - W2
        W1 = oemul(D, rur)
        if mv != 0:
            W2 = eomul(V, rup)
        CH = eomul(T, uz)
        kv = g.AK[mm, :][None, :]
        CHI.E[:nn, mm, :] = (1j * kv) * W1 + mv * kv * W2 - CH
    g.chopdo(PSI)
    g.chopdo(CHI)
    PSI.E[0, 0, :] = PSI.E[0, 0, :] - g.calcat1(PSI) / g.AT1[0]
    return PSI, CHI
