"""Energy diagnostics (oracle).

Restates mod_scalar3.f90:
  470-526  PRODCT_MK_ALLK     528-554  PRODCT_MK_HALFK
  750-806  L2NORM_MK_ALLK     808-841  L2NORM_MK_HALFK
and mod_boussinesq.f90:
  112-136  CALC_BOUSSI_PE     139-232  CALC_BOUSSI_ENERGY (without the file output)
for one process (INTH = INX = 0, ZLEN0 = ZLEN).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import math

import numpy as np

from .grid import FFF, PFF
from .legops import del2, delsqh
from .transforms import rtran


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
