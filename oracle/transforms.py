"""Space transitions FFF <-> PFF <-> PFP <-> PPP (oracle).

Restates:
  mod_fft.f90:771-926    HORFFT (theta real FFT of length 2*NTH on packed samples)
  mod_fft.f90:928-1113   VERFFT (z complex FFT of length NX, k chop/unchop)
  mod_fft.f90:1115-1148  PLNFFT
  mod_fft.f90:1150-1340  RTRAN  (mapped-Legendre parity GEMMs)
  mod_fft.f90:1342-1398  TOFF / TOFP
  mod_eig.f90:583-655    complex x real .MUL. (two real GEMMs)

FFTW (the reference's un-vendored FFT; version not pinned by the reference)
is replaced by scipy.fft; the sign/scaling conventions follow the calls the
reference makes (FFTW_FORWARD/BACKWARD, r2c/c2r, explicit 1/N scaling).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import numpy as np
import scipy.fft as sfft

from .grid import FFF, PFF, PFP, PPP, Field

WORKERS = -1


def horfft(g, A, IS):
    """HORFFT(A, IS), mod_fft.f90:771-926.  In place on A."""
    g.chopdo(A)
    nth = g.NTH
    E = A.E
    if IS == -1:
        if A.space != PPP:
            raise ValueError("HORFFT: NOT IN PHYSICAL SPACE")
        # C(2j-1) = Re E(j), C(2j) = Im E(j)  (844-848): samples at theta = pi*s/NTH
        c = np.empty(E.shape[:1] + (2 * nth,) + E.shape[2:], dtype=np.float64)
        c[:, 0::2, :] = E[:, :nth, :].real
        c[:, 1::2, :] = E[:, :nth, :].imag
        B = sfft.rfft(c, axis=1, workers=WORKERS) / (2 * nth)   # 851
        B[:, g.NTCHOP:, :] = 0                                  # 863
        B[:, 0, :] = B[:, 0, :].real                            # 866
        E[:, :, :] = B
        A.space = PFP
    else:
        if A.space != PFP:
            raise ValueError("HORFFT: NOT IN PFP SPACE")
        E[:, 0, :] = E[:, 0, :].real                            # 883
        E[:, g.NTCHOP:, :] = 0                                  # 886
        c = sfft.irfft(E[:, :nth + 1, :], n=2 * nth, axis=1, workers=WORKERS) * (2 * nth)
        E[:, :nth, :] = c[:, 0::2, :] + 1j * c[:, 1::2, :]      # 908-910
        E[:, nth, :] = 0
        A.space = PPP
    g.chopdo(A)
    return A


def verfft(g, A, IS):
    """VERFFT(A, IS), mod_fft.f90:928-1113 (single process: no transposes)."""
    LN = A.LN
    g.chopdo(A)
    nx, nxc = g.NX, g.NXCHOP
    if IS == -1:
        if A.space != PFP:
            raise ValueError("VERFFT: NOT IN PFP SPACE")
        a = A.E[:, :g.NTCHOPDIM, :]
        b = sfft.fft(a, axis=2, workers=WORKERS) / nx           # FFTW_FORWARD, /NX
        out = np.zeros(g.shape(PFF), dtype=np.complex128)
        out[:, :, :nxc] = b[:, :, :nxc]
        out[:, :, nxc:] = b[:, :, g.NXCHOPH - 1:]
        A.E = out
        A.space = PFF
    else:
        if A.space != PFF:
            raise ValueError("VERFFT: NOT IN PFF SPACE")
        b = np.zeros((g.NDIMR, g.NTCHOPDIM, nx), dtype=np.complex128)
        b[:, :, :nxc] = A.E[:, :, :nxc]
        b[:, :, g.NXCHOPH - 1:] = A.E[:, :, nxc:]
        b = sfft.ifft(b, axis=2, workers=WORKERS) * nx          # FFTW_BACKWARD, unscaled
        out = np.zeros(g.shape(PFP), dtype=np.complex128)
        out[:, :g.NTCHOPDIM, :] = b
        A.E = out
        A.space = PFP
    A.LN = LN
    g.chopdo(A)
    return A


def plnfft(g, A, IS):
    """PLNFFT(A, IS), mod_fft.f90:1115-1148."""
    if IS == -1:
        horfft(g, A, -1)
        verfft(g, A, -1)
    else:
        verfft(g, A, 1)
        horfft(g, A, 1)
    return A


def rtran(g, A, IS):
    """RTRAN(A, IS), mod_fft.f90:1150-1340.

    IS = -1 (PFF -> FFF): per m, BE(:,i) = (A(i) + A(NR+1-i)) W(i),
    BO = (A(i) - A(NR+1-i)) W(i); B(1:NN:2) = (BE . PF(:,1:NN:2))^T,
    B(2:NN:2) = (BO . PF(:,2:NN:2))^T, NN = NRCHOPS(m) (current chop).
    IS = +1 (FFF -> PFF): BE = PF(:,1:NN:2) A(1:NN:2), BO likewise;
    B(1:NRH) = BE + BO, B(NR:NRH+1:-1) = BE - BO; (m,k) = (0,0) adds
    LN * (-log(1-x)) (1318-1324).  Both directions reset A%LN to 0 (the
    SFREE of A at 1245/1326 zeroes it).
    """
    nr, nrh = g.NR, g.NRH
    W = g.W[:nrh]
    if IS == -1:
        if A.space != PFF:
            raise ValueError("RTRAN: NOT IN PFF_SPACE")
        B = g.alloc(FFF)
        E = A.E
        lo = E[:nrh, :, :]
        hi = E[nr - 1:nrh - 1:-1, :, :] if nrh > 0 else E[:0]
        be = (lo + hi) * W[:, None, None]
        bo = (lo - hi) * W[:, None, None]
        for mm in range(E.shape[1]):
            nn = int(g.NRCHOPS[mm])
            if nn < 1:
                continue
            pf = g.PF[:nrh, :, mm]
            B.E[0:nn:2, mm, :] = pf[:, 0:nn:2].T @ be[:, mm, :]
            if nn >= 2:
                B.E[1:nn:2, mm, :] = pf[:, 1:nn:2].T @ bo[:, mm, :]
        g.chopdo(B)
        B.LN = 0.0
        A.E, A.space, A.LN = B.E, FFF, 0.0
    else:
        if A.space != FFF:
            raise ValueError("RTRAN: NOT IN FFF_SPACE")
        B = g.alloc(PFF)
        E = A.E
        for mm in range(E.shape[1]):
            nn = int(g.NRCHOPS[mm])
            pf = g.PF[:nrh, :, mm]
            be = pf[:, 0:nn:2] @ E[0:nn:2, mm, :] if nn >= 1 else 0.0
            bo = pf[:, 1:nn:2] @ E[1:nn:2, mm, :] if nn >= 2 else 0.0
            B.E[:nrh, mm, :] = be + bo
            B.E[nr - 1:nrh - 1:-1, mm, :] = be - bo
        B.E[:, max(0, g.NTCHOP):, :] = 0
        if A.LN != 0.0:
            B.E[:nr, 0, 0] += A.LN * g.LNX[:nr]
        A.E, A.space, A.LN = B.E, PFF, 0.0
    g.chopdo(A)
    return A


def toff(g, A):
    """TOFF(A), mod_fft.f90:1342-1369."""
    if A.space == PPP:
        horfft(g, A, -1)
        verfft(g, A, -1)
        rtran(g, A, -1)
    elif A.space == PFP:
        verfft(g, A, -1)
        rtran(g, A, -1)
    elif A.space == PFF:
        rtran(g, A, -1)
    return A


def tofp(g, A):
    """TOFP(A), mod_fft.f90:1371-1398."""
    if A.space == FFF:
        rtran(g, A, 1)
        verfft(g, A, 1)
        horfft(g, A, 1)
    elif A.space == PFF:
        verfft(g, A, 1)
        horfft(g, A, 1)
    elif A.space == PFP:
        horfft(g, A, 1)
    return A


def physical_samples(g, A):
    """Real samples f(r_i, theta_s, z_l), theta_s = pi*s/NTH, from a PPP field
    (the packed layout of mod_fft.f90:844-848 unpacked)."""
    E = A.E[:g.NR, :g.NTH, :]
    out = np.empty((g.NR, 2 * g.NTH, g.NX))
    out[:, 0::2, :] = E.real
    out[:, 1::2, :] = E.imag
    return out


def field_from_samples(g, f):
    """Inverse of physical_samples: a PPP field whose packed values are f."""
    A = g.alloc(PPP)
    A.E[:g.NR, :g.NTH, :] = f[:, 0::2, :] + 1j * f[:, 1::2, :]
    return A


__all__ = ["horfft", "verfft", "plnfft", "rtran", "toff", "tofp",
           "physical_samples", "field_from_samples", "Field"]
