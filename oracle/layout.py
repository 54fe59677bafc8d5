"""Initial conditions (oracle).

Restates:
  mod_layout.f90:64-117   LAY      (analytic field at collocation points, /(1-x)^IP)
  mod_layout.f90:449-609  QVORTEX  (omega_z = 2Q exp(-B r^2/R0^2)/R0^2 -> psi via IDELSQH)
  mod_layout.f90:640-672  GAUS (with the z-waviness DX, DY, K, DP and the core
                          modulation DR, RK, RP of a QPAIR entry)
The seeded spectral perturbation that the benchmark configurations add on
top of the vortex is synthetic input data, generated by the caller and
passed in as FFF coefficient arrays.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import numpy as np

from .grid import FFF, PPP
from .legops import idelsqh
from .transforms import toff


def gaus_ppp(g, q, b=1.0, r0=1.0, xc=0.0, yc=0.0, ip=2):
    """LAY(A, GAUS, IP) into a fresh PPP field (mod_layout.f90:64-117, 640-672)."""
    A = g.alloc(PPP)
    r = g.R[:, None]
    f = (1 - g.X[:, None]) ** ip

    def gaus(th):
        x = r * np.cos(th)[None, :]
        y = r * np.sin(th)[None, :]
        r2 = ((x - xc) ** 2.0 + (y - yc) ** 2.0) / r0 ** 2.0
        return q / r0 ** 2.0 * np.exp(-b * r2)

    vr = gaus(g.THR[:g.NTH]) / f
    vi = gaus(g.THI[:g.NTH]) / f
    A.E[:g.NR, :g.NTH, :] = (vr + 1j * vi)[:, :, None]
    g.chopdo(A)
    return A


VORTEX_KEYS = ("x", "y", "q", "h", "b", "dx", "dy", "k", "dp", "r", "dr", "rk", "rp")


def vortex(**kw):
    """One QPAIR entry with the reference's defaults (Q = 1, B = 1, R = 1, rest 0)."""
    v = dict(x=0.0, y=0.0, q=1.0, h=0.0, b=1.0, dx=0.0, dy=0.0, k=0.0, dp=0.0, r=1.0, dr=0.0, rk=0.0, rp=0.0)
    v.update(kw)
    return v


def lay_gaus(g, A, q, b, v):
    """A += LAY(GAUS, IP = 2) of one vortex with GAUSDATA%Q = q, %B = b and the
    centre / core modulation of v (GAUS, mod_layout.f90:640-672; Z = ZLEN (KK-1) / NX)."""
    r = g.R[:g.NR, None, None]
    f = (1 - g.X[:g.NR, None, None]) ** 2
    z = g.Z[None, None, :g.NX]
    ak1 = 2 * np.pi * v["k"] / g.ZLEN
    rk = 2 * np.pi * v["rk"] / g.ZLEN
    dp = np.pi / 180.0 * v["dp"]
    rp = np.pi / 180.0 * v["rp"]
    xc = v["x"] + v["dx"] * np.sin(ak1 * z - dp)
    yc = v["y"] + v["dy"] * np.sin(ak1 * z - dp)
    r0 = v["r"] + v["dr"] * np.sin(rk * z - rp)

    def gaus(th):
        x = r * np.cos(th)[None, :, None]
        y = r * np.sin(th)[None, :, None]
        r2 = ((x - xc) ** 2.0 + (y - yc) ** 2.0) / r0 ** 2.0
        return q / r0 ** 2.0 * np.exp(-b * r2)

    A.E[:g.NR, :g.NTH, :g.NX] += gaus(g.THR[:g.NTH]) / f + 1j * (gaus(g.THI[:g.NTH]) / f)
    return A


def qvortex_list(g, vortices):
    """QVORTEX(PSI, CHI), mod_layout.f90:449-609, NOISE = 0, for a QPAIR list."""
    out = []
    for field in ("psi", "chi"):
        A = g.alloc(PPP)
        for v in vortices:
            if field == "psi":
                lay_gaus(g, A, 2.0 * v["q"], 1.0, v)
            else:
                lay_gaus(g, A, v["h"], v["b"], v)
        g.chopdo(A)
        toff(g, A)
        A.E = -A.E
        A.LN = 0.0
        out.append(idelsqh(g, A))
    return out[0], out[1]


def qvortex(g, q=1.0, h=0.0, b=1.0, r0=1.0, xc=0.0, yc=0.0):
    """QVORTEX(PSI, CHI) for one vortex, mod_layout.f90:449-609 (NOISE = 0)."""
    A = gaus_ppp(g, 2.0 * q, 1.0, r0, xc, yc)
    toff(g, A)
    A.E = -A.E
    A.LN = 0.0
    PSI = g.copy0(idelsqh(g, A))
    PSI.LN = idelsqh(g, A).LN
    if h != 0.0:
        A = gaus_ppp(g, h, b, r0, xc, yc)
        toff(g, A)
        A.E = -A.E
        A.LN = 0.0
        C = idelsqh(g, A)
        CHI = g.copy0(C)
        CHI.LN = C.LN
    else:
        CHI = g.alloc(FFF)
    return PSI, CHI


def add_coefficients(g, F, coef):
    """Add an FFF coefficient array (same shape as F.E) and re-apply the chop."""
    F.E = F.E + coef
    g.chopdo(F)
    return F


def initial_state(g, coef_psi, coef_chi, coef_b, q=1.0, r0=1.0):
    """Vortex + seeded perturbation (construction documented in
    mlegs_b200/inputs.py): psi' = IDELSQH(-c_psi), chi' = IDELSQH(-c_chi),
    b' = c_b with the CALCAT1 far-field fix at m = 0."""
    psi, chi = qvortex(g, q=q, r0=r0)
    b = g.alloc(FFF)
    for F, c in ((psi, coef_psi), (chi, coef_chi)):
        P = g.alloc(FFF)
        P.E = -np.asarray(c, dtype=np.complex128).copy()
        g.chopdo(P)
        Q = idelsqh(g, P)
        F.E = F.E + Q.E
        F.LN = F.LN + Q.LN
        g.chopdo(F)
    P = g.alloc(FFF)
    P.E = np.asarray(coef_b, dtype=np.complex128).copy()
    g.chopdo(P)
    P.E[0, 0, :] -= g.calcat1(P) / g.AT1[0]
    b.E = b.E + P.E
    return psi, chi, b
