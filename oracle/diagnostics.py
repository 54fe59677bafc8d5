"""Energy diagnostics (oracle).

Restates mod_scalar3.f90:
  470-526  PRODCT_MK_ALLK     528-554  PRODCT_MK_HALFK
  750-806  L2NORM_MK_ALLK     808-841  L2NORM_MK_HALFK
and mod_boussinesq.f90:
  112-136  CALC_BOUSSI_PE     139-232  CALC_BOUSSI_ENERGY (without the file output)
and mod_march.f90:
  1689-1966 DIAGNOST (values and checks; no printing or stored initial values)
  1967-2225 CALCXY, ABSVEC2, MULRCOSTH, MULRSINTH, MULR2
  3649-3682 INTEG_P          and mod_scalar3.f90:312-353 INTEG, 398-468 PRODCT
for one process (INTH = INX = 0, ZLEN0 = ZLEN).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import math

import numpy as np

from .grid import FFF, PFF
from .grid import PPP
from .legops import del2, delsqh, pc2vor, xxdx
from .transforms import rtran, toff, tofp


def _scale(g):
    return 4.0 * math.pi * g.ZLEN * g.ELL2


def prodct_mk_allk(g, A, B):
    """PRODCT_MK_ALLK: 4 pi ZLEN0 ELL2 sum_r Re(A conj B) w_r per (m, k), m = 0 halved."""
    if A.space != PFF or B.space != PFF:
        raise ValueError("PRODCT_MK() -- NOT IN PFF_SPACE")
    nr = g.NR
    wk = np.real(A.E[:nr] * np.conj(B.E[:nr]))              # (NR, NTCHOPDIM, NXCHOPDIM)
    out = _scale(g) * np.einsum("rmk,r->mk", wk, g.W[:nr])
    out[0, :] *= 0.5
    return out


def l2norm_mk_allk(g, A):
    """L2NORM_MK_ALLK: 4 pi ZLEN0 ELL2 sum_r |A|^2 / (1 - x_r)^2 w_r per (m, k), m = 0 halved."""
    if A.space != PFF:
        raise ValueError("L2NORM_MK() -- NOT IN PFF_SPACE")
    nr = g.NR
    wk = np.abs(A.E[:nr]) ** 2 / ((1 - g.X[:nr]) ** 2)[:, None, None]
    out = _scale(g) * np.einsum("rmk,r->mk", wk, g.W[:nr])
    out[0, :] *= 0.5
    return out


def halfk(g, allk):
    """*_MK_HALFK: fold k and -k into k = 0 .. NXCHOP-1; (NTCHOP, NXCHOP) result."""
    out = np.zeros((g.NTCHOP, g.NXCHOP))
    nt = allk.shape[0]
    out[:nt, 0] = allk[:, 0]
    for kk in range(1, g.NXCHOP):
        kc = g.NXCHOPDIM - kk
        out[:nt, kk] = allk[:, kc] + allk[:, kk]
    return out


def boussi_pe(g, B, bv0):
    """CALC_BOUSSI_PE(B) at the current chop."""
    wk = g.copy0(B)
    wk.LN = 0.0
    rtran(g, wk, 1)
    return halfk(g, l2norm_mk_allk(g, wk)) / 2.0 / bv0 ** 2


def boussi_energy(g, PSI, CHI, B, bv0):
    """CALC_BOUSSI_ENERGY(PSI, CHI, B): (KE, PE, DKE), each (NTCHOP, NXCHOP)."""
    for F in (PSI, CHI, B):
        if F.space != FFF:
            raise ValueError("CALC_BOUSSI_ENERGY: NOT IN FFF_SPACE")
    if B.LN != 0.0:
        raise ValueError("B has non-zero LN, this is not expected in Boussinesq")
    g.chopset(3)
    try:
        W1 = g.copy0(PSI)
        W1.LN = 2.0 * PSI.LN
        W2 = delsqh(g, W1)
        W1.LN = 0.0
        W2.LN = 0.0
        rtran(g, W1, 1)
        rtran(g, W2, 1)
        ke = -halfk(g, prodct_mk_allk(g, W1, W2))
        W1 = del2(g, CHI)
        W2 = delsqh(g, CHI)
        W1.LN = 0.0
        W2.LN = 0.0
        rtran(g, W1, 1)
        rtran(g, W2, 1)
        ke = ke + halfk(g, prodct_mk_allk(g, W1, W2))
        ke = ke / 2.0
        W3 = g.copy0(B)
        W3.LN = 0.0
        rtran(g, W3, 1)
        dke = halfk(g, prodct_mk_allk(g, W3, W2))
        pe = halfk(g, l2norm_mk_allk(g, W3)) / 2.0 / bv0 ** 2
    finally:
        g.chopset(-3)
    return ke, pe, dke


def integ(g, F):
    """INTEG(F), mod_scalar3.f90:312-353: 4 pi ZLEN ELL2 Re E(1,1,1) NORM(1,1)."""
    if F.space != FFF:
        raise ValueError("INTEG: NOT IN FFF_SPACE")
    return 4.0 * math.pi * g.ZLEN * g.ELL2 * F.E[0, 0, 0].real * g.NORM0[0]


def integ_p(g, F):
    """INTEG_P(F), mod_march.f90:3649-3682, on the RTRAN(+1) image F_COPY that
    it forms (the reference's DOT_PRODUCT reads F%E(:NR,1,1) of the FFF input,
    whose first dimension NRCHOPDIM is below NR unless NRCHOP = NR - 6)."""
    if F.space != FFF:
        raise ValueError("INTEG_P: NOT IN FFF_SPACE")
    fc = g.copy0(F)
    rtran(g, fc, 1)
    nr = g.NR
    return 2.0 * math.pi * g.ZLEN * g.ELL2 * float(
        np.dot(fc.E[:nr, 0, 0].real / (1.0 - g.X[:nr]) ** 2, g.W[:nr]))


def prodct(g, A, B):
    """PRODCT(A, B), mod_scalar3.f90:398-468 (the sum of PRODCT_MK_ALLK)."""
    return float(prodct_mk_allk(g, A, B).sum())


DIAGNOST_KEYS = ("VALVOR", "VALZMO", "VALANG", "VALENE", "VALHEL", "PAT1_SPREAD", "CAT1_SPREAD", "NORM_CHECK",
                 "VALX", "VALY", "VALR")


def calcxy(g, ROR, ROP, OZ):
    """CALCXY(ROR, ROP, OZ), mod_march.f90:1967-2047, at the current chop:
    TOFP of the vorticity, ABSVEC2 (2050-2099) into OZ, then INTEG(TOFF(.)) of
    the enstrophy times 1, R cos(th), R sin(th), R^2 (MULRCOSTH / MULRSINTH /
    MULR2, 2102-2225; THR(j) = 2 pi j / NTH, THI(j) = 2 pi (j + 1/2) / NTH).
    Returns (<X>, <Y>, <R>)."""
    for F in (ROR, ROP, OZ):
        tofp(g, F)
    nr, nth = g.NR, g.NTH
    r = g.R[:nr][:, None, None]
    f = ((1.0 - g.X[:nr]) ** 2)[:, None, None]
    u, v, w = (F.E[:nr, :nth, :] for F in (ROR, ROP, OZ))
    re = ((u.real ** 2 + v.real ** 2) / r ** 2 + w.real ** 2) / f
    im = ((u.imag ** 2 + v.imag ** 2) / r ** 2 + w.imag ** 2) / f
    OZ.E[:nr, :nth, :] = re + 1j * im
    j = np.arange(nth)[None, :, None]
    thr = 2.0 * math.pi / nth * j
    thi = 2.0 * math.pi / nth * (j + 0.5)
    weights = ((1.0, 1.0), (r * np.cos(thr), r * np.cos(thi)), (r * np.sin(thr), r * np.sin(thi)),
               (r * r, r * r))
    mom = []
    for wr, wi in weights:
        A = OZ.copy()
        A.E[:nr, :nth, :] = wr * re + 1j * (wi * im)
        toff(g, A)
        mom.append(integ(g, A))
    return mom[1] / mom[0], mom[2] / mom[0], math.sqrt(mom[3] / mom[0])


class DiagnostError(ValueError):
    """The reference's MPI_ABORT in DIAGNOST: code 11 dealiasing, 12 divergence."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def diagnost(g, PSI, CHI):
    """DIAGNOST(PSI, CHI), mod_march.f90:1689-1966, as a dict of DIAGNOST_KEYS."""
    for F in (PSI, CHI):
        if F.space != FFF:
            raise ValueError("DIAGNOST: NOT IN FFF_SPACE")
    out = {"NORM_CHECK": abs(PSI.E[1, 0, 0].imag + CHI.E[1, 0, 0].imag)}   # 1733-1741
    # dealiasing check, 1746-1765 (at the base chop)
    chk = 0.0
    for mm in range(min(2, PSI.E.shape[1])):
        tail = PSI.E[g.NRCHOPS[mm]:, mm, :]
        chk += float(np.abs(tail).max()) if tail.size else 0.0
    if chk > 1.0e-12:
        raise DiagnostError(11, "DIAG: DEALIASING INCOMPLETE")
    # divergence check, 1770-1787
    kmax = min(5, PSI.E.shape[2])
    mmax = min(6, PSI.E.shape[1])
    nmax = min(5, g.NRCHOP)
    if np.any(np.abs(PSI.E[:nmax, 1:mmax, :kmax]) > 100.0):
        raise DiagnostError(12, "DIAG: DIVERGENCE")
    g.chopset(3)
    try:
        out["VALVOR"] = integ(g, _neg(delsqh(g, PSI)))    # OZH of PC2VOR(..., 'H')
        out["VALZMO"] = integ(g, _neg(delsqh(g, CHI)))    # UZH of PC2VEL(..., 'H')
        rur = g.copy0(PSI)
        rur.LN = 0.0
        out["VALANG"] = -integ_p(g, xxdx(g, rur))
        rup = g.copy0(PSI)
        rup.LN = 2.0 * PSI.LN
        rur = delsqh(g, rup)
        rtran(g, rur, 1)
        rup = g.copy0(PSI)
        rup.LN = 0.0
        rtran(g, rup, 1)
        ene1 = prodct(g, rur, rup)
        rup = del2(g, CHI)
        rtran(g, rup, 1)
        rur = delsqh(g, CHI)
        rtran(g, rur, 1)
        ene2 = prodct(g, rur, rup)
        out["VALENE"] = -ene1 + ene2
        rur = delsqh(g, PSI)
        rtran(g, rur, 1)
        out["VALHEL"] = 2.0 * prodct(g, rur, rup)
        pat1 = np.abs(g.calcat1(PSI))
        cat1 = np.abs(g.calcat1(CHI))
        out["PAT1_SPREAD"] = float(pat1.max() - pat1.min())
        out["CAT1_SPREAD"] = float(cat1.max() - cat1.min())
        out["VALX"], out["VALY"], out["VALR"] = calcxy(g, *pc2vor(g, PSI, CHI))
    finally:
        g.chopset(-3)
    return out


def _neg(F):
    F.E = -F.E
    return F
