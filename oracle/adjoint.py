"""Adjoints (vector-Jacobian products) of the transform and nonlinear-term
maps (oracle).

Each function takes the cotangent of a map's output and returns the cotangent
of its input, for the real inner product <a, b> = sum(Re a Re b + Im a Im b)
on complex arrays (and LN * LN_bar for the log-term scalar), so that
<y, F(x)> = <F^T(y), x> for the forward maps of oracle/transforms.py:

  rtran_T(g, Y, +1)   RTRAN(A, +1) FFF -> PFF, mod_fft.f90:1264-1336 (with the
                      (m, k) = (0, 0) log term of 1318-1324: LN_bar = sum_i
                      Re Y(i, 0, 0) (-log(1 - x_i)))
  rtran_T(g, Y, -1)   RTRAN(A, -1) PFF -> FFF, mod_fft.f90:1189-1261
  verfft_T(g, Y, IS)  VERFFT(A, IS), mod_fft.f90:928-1113
  horfft_T(g, Y, IS)  HORFFT(A, IS), mod_fft.f90:771-926
  tofp_T / toff_T     TOFP / TOFF, mod_fft.f90:1342-1398 (reverse order)
  vprodsub_T          VPRODSUB (mod_legops.f90:1972-2133) with VDOTPSUB
                      (2136-2232) as the nonlinear term of CALC_BOUSSI_NONLIN
                      forms them, pointwise in PPP

Every CHOPDO along the way is a 0/1 projection and is its own adjoint.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import numpy as np
import scipy.fft as sfft

from .grid import FFF, PFF, PFP, PPP, Field


def _field(E, space, LN=0.0):
    return Field(np.array(E, dtype=np.complex128), space, float(LN))


def rtran_T(g, Y, IS):
    """Adjoint of RTRAN(A, IS)."""
    nr, nrh = g.NR, g.NRH
    W = g.W[:nrh]
    if IS == 1:  # Y in PFF -> (E_bar in FFF, LN_bar)
        if Y.space != PFF:
            raise ValueError("rtran_T(+1): cotangent not in PFF")
        y = _field(Y.E, PFF)
        g.chopdo(y)
        y.E[:, max(0, g.NTCHOP):, :] = 0
        A = g.alloc(FFF)
        lo = y.E[:nrh]
        hi = y.E[nr - 1:nrh - 1:-1] if nrh > 0 else y.E[:0]
        be, bo = lo + hi, lo - hi
        for mm in range(A.E.shape[1]):
            nn = int(g.NRCHOPS[mm])
            pf = g.PF[:nrh, :, mm]
            if nn >= 1:
                A.E[0:nn:2, mm, :] = pf[:, 0:nn:2].T @ be[:, mm, :]
            if nn >= 2:
                A.E[1:nn:2, mm, :] = pf[:, 1:nn:2].T @ bo[:, mm, :]
        A.LN = float(np.dot(y.E[:nr, 0, 0].real, g.LNX[:nr]))
        return A
    if Y.space != FFF:
        raise ValueError("rtran_T(-1): cotangent not in FFF")
    y = _field(Y.E, FFF)
    g.chopdo(y)
    A = g.alloc(PFF)
    for mm in range(y.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        pf = g.PF[:nrh, :, mm]
        be = pf[:, 0:nn:2] @ y.E[0:nn:2, mm, :]
        bo = pf[:, 1:nn:2] @ y.E[1:nn:2, mm, :] if nn >= 2 else 0.0
        A.E[:nrh, mm, :] = (be + bo) * W[:, None]
        A.E[nr - 1:nrh - 1:-1, mm, :] = (be - bo) * W[:, None]
    return A


def verfft_T(g, Y, IS):
    """Adjoint of VERFFT(A, IS)."""
    nx, nxc = g.NX, g.NXCHOP
    if IS == 1:  # Y in PFP -> PFF
        y = _field(Y.E, PFP)
        g.chopdo(y)
        b = sfft.fft(y.E[:, :g.NTCHOPDIM, :nx], axis=2)          # sum_z y e^{-2 pi i k z / NX}
        A = g.alloc(PFF)
        A.E[:, :, :nxc] = b[:, :, :nxc]
        A.E[:, :, nxc:] = b[:, :, g.NXCHOPH - 1:]
        g.chopdo(A)
        return A
    y = _field(Y.E, PFF)                                          # Y in PFF -> PFP
    g.chopdo(y)
    c = np.zeros((g.NDIMR, g.NTCHOPDIM, nx), dtype=np.complex128)
    c[:, :, :nxc] = y.E[:, :, :nxc]
    c[:, :, g.NXCHOPH - 1:] = y.E[:, :, nxc:]
    A = g.alloc(PFP)
    A.E[:, :g.NTCHOPDIM, :nx] = sfft.ifft(c, axis=2)              # (1/NX) sum_k c e^{+...}
    g.chopdo(A)
    return A


def horfft_T(g, Y, IS):
    """Adjoint of HORFFT(A, IS)."""
    nth, ntc = g.NTH, g.NTCHOP
    if IS == 1:  # Y in PPP (packed samples) -> PFP
        y = _field(Y.E, PPP)
        g.chopdo(y)
        c = np.empty(y.E.shape[:1] + (2 * nth,) + y.E.shape[2:], dtype=np.float64)
        c[:, 0::2, :] = y.E[:, :nth, :].real
        c[:, 1::2, :] = y.E[:, :nth, :].imag
        X = sfft.rfft(c, axis=1)                                  # sum_s c e^{-i pi m s / NTH}
        X[:, 1:, :] *= 2.0
        X[:, 0, :] = X[:, 0, :].real
        X[:, ntc:, :] = 0
        A = g.alloc(PFP)
        A.E[:, :nth + 1, :] = X
        g.chopdo(A)
        return A
    y = _field(Y.E, PFP)                                          # Y in PFP -> PPP
    g.chopdo(y)
    Z = np.array(y.E[:, :nth + 1, :])
    Z[:, ntc:, :] = 0
    Z[:, 0, :] = 2.0 * Z[:, 0, :].real
    c = sfft.irfft(Z, n=2 * nth, axis=1) / 2.0
    A = g.alloc(PPP)
    A.E[:, :nth, :] = c[:, 0::2, :] + 1j * c[:, 1::2, :]
    g.chopdo(A)
    return A


def tofp_T(g, Y):
    """Adjoint of TOFP (FFF -> PPP): RTRAN(+1)^T VERFFT(+1)^T HORFFT(+1)^T."""
    return rtran_T(g, verfft_T(g, horfft_T(g, Y, 1), 1), 1)


def toff_T(g, Y):
    """Adjoint of TOFF (PPP -> FFF): HORFFT(-1)^T VERFFT(-1)^T RTRAN(-1)^T."""
    return horfft_T(g, verfft_T(g, rtran_T(g, Y, -1), -1), -1)


def vprodsub_T(g, U, OM, NB_bar):
    """Adjoint of the bilinear products of the nonlinear term, pointwise on the
    packed PPP samples (real and imaginary parts are independent samples):
        N_r = u_t w_z - u_z w_t,  N_t = u_z w_r - u_r w_z,
        N_z = (u_r w_t - u_t w_r) / r^2,
    U = (RUR, RUP, UZ), OM = (ROR, ROP, OZ) in PPP; NB_bar = cotangents of
    (N_r, N_t, N_z).  Returns (U_bar, OM_bar) as lists of three PPP arrays."""
    r2 = (g.R[:g.NR] ** 2)[:, None, None]
    sl = (slice(0, g.NR), slice(0, g.NTH), slice(None))   # the samples VPRODSUB writes
    out_u = [np.zeros_like(U[0]) for _ in range(3)]
    out_w = [np.zeros_like(U[0]) for _ in range(3)]
    for part in (0, 1):
        pick = (lambda a: a.real) if part == 0 else (lambda a: a.imag)
        u1, u2, u3 = (pick(a[sl]) for a in U)
        w1, w2, w3 = (pick(a[sl]) for a in OM)
        b1, b2, b3 = (pick(a[sl]) for a in NB_bar)
        b3r = b3 / r2
        # N_r = u2 w3 - u3 w2, N_t = u3 w1 - u1 w3, N_z = (u1 w2 - u2 w1) / r^2
        du = [-b2 * w3 + b3r * w2, b1 * w3 - b3r * w1, -b1 * w2 + b2 * w1]
        dw = [b2 * u3 - b3r * u2, -b1 * u3 + b3r * u1, b1 * u2 - b2 * u1]
        for q in range(3):
            f = 1.0 if part == 0 else 1j
            out_u[q][sl] += f * du[q]
            out_w[q][sl] += f * dw[q]
    return out_u, out_w
