"""Initial conditions (oracle).

Restates:
  mod_layout.f90:64-117   LAY      (analytic field at collocation points, /(1-x)^IP)
  mod_layout.f90:449-609  QVORTEX  (omega_z = 2Q exp(-B r^2/R0^2)/R0^2 -> psi via IDELSQH)
  mod_layout.f90:640-672  GAUS (with the z-waviness DX, DY, K, DP and the core
                          modulation DR, RK, RP of a QPAIR entry)
  mod_layout.f90:165-278  NOISE, RAN0, FLATTEN (QPAIR%NOISE = 1, seeds explicit)
The seeded spectral perturbation that the benchmark configurations add on
top of the vortex is synthetic input data, generated by the caller and
passed in as FFF coefficient arrays.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import numpy as np

from .grid import FFF, PPP
from .legops import idelsqh
from .transforms import toff, tofp


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


def gaus_value(v, q, b, x, y, z, zlen):
    """GAUS(R, TH, Z), mod_layout.f90:640-672, at Cartesian (x, y) and axial z
    (broadcasting): strength q / R0^2, decay b, the centre displaced by
    DX, DY sin(AK1 Z - DP) and the core R0 = R + DR sin(RK Z - RP)."""
    ak1 = 2 * np.pi * v["k"] / zlen
    rk = 2 * np.pi * v["rk"] / zlen
    dp = np.pi / 180.0 * v["dp"]
    rp = np.pi / 180.0 * v["rp"]
    xc = v["x"] + v["dx"] * np.sin(ak1 * z - dp)
    yc = v["y"] + v["dy"] * np.sin(ak1 * z - dp)
    r0 = v["r"] + v["dr"] * np.sin(rk * z - rp)
    r2 = ((x - xc) ** 2.0 + (y - yc) ** 2.0) / r0 ** 2.0
    return q / r0 ** 2.0 * np.exp(-b * r2)


def lay_gaus(g, A, q, b, v):
    """A += LAY(GAUS, IP = 2) of one vortex with GAUSDATA%Q = q, %B = b and the
    centre / core modulation of v (mod_layout.f90:64-117; Z = ZLEN (KK-1) / NX)."""
    r = g.R[:g.NR, None, None]
    f = (1 - g.X[:g.NR, None, None]) ** 2
    z = g.Z[None, None, :g.NX]

    def gaus(th):
        return gaus_value(v, q, b, r * np.cos(th)[None, :, None], r * np.sin(th)[None, :, None], z, g.ZLEN)

    A.E[:g.NR, :g.NTH, :g.NX] += gaus(g.THR[:g.NTH]) / f + 1j * (gaus(g.THI[:g.NTH]) / f)
    return A


class Ran0:
    """RAN0(IDUM), mod_layout.f90:196-214: Park-Miller minimal standard by
    Schrage's method, with the XOR mask applied around each call."""
    IA, IM, IQ, IR, MASK = 16807, 2147483647, 127773, 2836, 123459876

    def __init__(self, iseed):
        self.idum = int(iseed)

    def __call__(self):
        idum = self.idum ^ self.MASK
        k = int(idum / self.IQ)                 # Fortran integer division truncates
        idum = self.IA * (idum - k * self.IQ) - self.IR * k
        if idum < 0:
            idum += self.IM
        val = (1.0 / self.IM) * idum
        self.idum = idum ^ self.MASK
        return val


def noise(g, A, alevel, iseed):
    """NOISE(A, ALEVEL), mod_layout.f90:165-226, on an FFF field with an explicit
    ISEED.  The reference is compiled with default REAL of 8 bytes (-r8 or
    -fdefault-real-8 in its Makefile), so the literal 0.1, FLOAT(N) and
    CMPLX(X, Y) are double precision."""
    ran = Ran0(iseed)
    refval = alevel * np.abs(A.E).max()
    akmax = np.abs(g.AK[:g.NTCHOP, :g.NXCHOP]).max()
    if akmax == 0.0:
        akmax = 1.0
    for mm in range(min(g.NTCHOP, A.E.shape[1])):
        for nn in range(int(g.NRCHOPS[mm])):
            n = int(g.M[mm]) + nn
            q = float(n) / g.NRCHOP
            for kk in range(A.E.shape[2]):
                akr = g.AK[mm, kk] / akmax
                fac = 0.1 * np.exp(-12.0 * (akr * akr + q * q))
                x = fac * ran()
                y = fac * ran()
                A.E[nn, mm, kk] += complex(x * refval, y * refval)
    g.chopdo(A)
    return A


def flatten(g, A, B):
    """FLATTEN(A, B), mod_layout.f90:228-278 (PPP): A = B + (A - B) tanh(20 B / REFVAL)^2,
    REFVAL = max |Re A| (1 if zero), real and imaginary samples apart."""
    refval = np.abs(A.E.real).max()
    if refval == 0.0:
        refval = 1.0
    fr = np.tanh(B.E.real / refval * 20) ** 2
    fi = np.tanh(B.E.imag / refval * 20) ** 2
    A.E = (B.E.real + (A.E.real - B.E.real) * fr) + 1j * (B.E.imag + (A.E.imag - B.E.imag) * fi)
    return A


def qvortex_list(g, vortices, noise_seeds=None):
    """QVORTEX(PSI, CHI), mod_layout.f90:449-609, for a QPAIR list; NOISE = 1
    when noise_seeds gives the two RAN0 seeds (PSI, CHI)."""
    out = []
    for f, field in enumerate(("psi", "chi")):
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
        if noise_seeds is not None:
            B = g.copy0(A)
            noise(g, A, 0.02, noise_seeds[f])
            tofp(g, A)
            tofp(g, B)
            flatten(g, A, B)
            toff(g, A)
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
