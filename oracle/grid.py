"""Grid set-up, Legendre tables, field container and truncation (oracle).

Restates:
  mod_fft.f90:180-367        LEGINIT (sizes, M, AK, TFM kit)
  mod_lin_legendre.f90:79-131  GAUSS_LEGENDRE (Newton, EPS = 1e-15)
  mod_lin_legendre.f90:133-175 LEG_ZERO (r = ELL*sqrt((1+x)/(1-x)))
  mod_lin_legendre.f90:205-278 LEG_NORMT (NORM, used for m = 0 only)
  mod_lin_legendre.f90:306-377 LEG_LOG_NORMT (LOGNORM)
  mod_lin_legendre.f90:526-644 LEG_TBL3 (orthonormal P^m_n(x_i) table PF)
  mod_scalar3.f90:41-47      TYPE(SCALAR)      -> Field
  mod_scalar3.f90:165-211    CHOPSET           -> Grid.chopset
  mod_scalar3.f90:213-257    CHOPDO            -> Grid.chopdo
  mod_scalar3.f90:262-310    CALCAT0/CALCAT1   -> Grid.calcat0/calcat1
  mod_fft.f90:603-670        SALLOC            -> Grid.alloc

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import math

import numpy as np

PPP, FFF, PFP, PFF = 0, 1, 2, 3  # mod_scalar3.f90:82-85


class Field:
    """TYPE(SCALAR) (mod_scalar3.f90:41-47): E array, LN log term, space tag."""

    __slots__ = ("E", "LN", "space")

    def __init__(self, E, space, LN=0.0):
        self.E = E
        self.space = space
        self.LN = float(LN)

    def copy(self):
        return Field(self.E.copy(), self.space, self.LN)


def gauss_legendre(n):
    """GAUSS_LEGENDRE(-1, 1, X, W, N), mod_lin_legendre.f90:79-131.

    Newton iteration from z = cos(pi (i - 1/4)/(n + 1/2)) until |dz| <= 1e-15;
    x ascending from -1 to 1; the weight uses P'_n at the last-but-one iterate
    exactly as the reference does.
    """
    m = int(math.ceil((n + 1) / 2.0))
    x = np.zeros(n)
    w = np.zeros(n)
    eps = 1e-15
    for i in range(1, m + 1):
        z = math.cos(math.pi * (i - 0.25) / (n + 0.5))
        z1 = 2.0
        pp = 1.0
        while abs(z - z1) > eps:
            p1, p2 = 1.0, 0.0
            for j in range(1, n + 1):
                p3 = p2
                p2 = p1
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j
            pp = n * (z * p1 - p2) / (z * z - 1)
            z1 = z
            z = z1 - p1 / pp
        x[i - 1] = -z
        x[n - i] = z
        w[i - 1] = 2.0 / ((1 - z * z) * pp * pp)
        w[n - i] = w[i - 1]
    return x, w


def leg_log_norm(ndim, ms):
    """LEG_LOG_NORMT(NDIM, MS), mod_lin_legendre.f90:306-377 (FP64, as written)."""
    ms = [abs(int(m)) for m in ms]
    me = max(ms)
    wk = np.zeros(me + 1)
    wk[0] = math.log(0.5)
    for m in range(1, me + 1):
        wk[m] = wk[m - 1] + math.log(2 * m + 1.0) - math.log(2 * m * (2 * m - 1.0) ** 2)
    out = np.zeros((ndim, len(ms)))
    for mm, m in enumerate(ms):
        out[0, mm] = wk[m]
        for nn in range(2, ndim + 1):
            n = m + (nn - 1)
            out[nn - 1, mm] = (out[nn - 2, mm] + math.log(2 * n + 1.0) - math.log(2 * n - 1.0)
                               + math.log(1.0 * (n - m)) - math.log(1.0 * (n + m)))
    return 0.5 * out


def leg_norm_m0(ndim):
    """LEG_NORMT(NDIM, (/0/)), mod_lin_legendre.f90:205-278, m = 0 column.

    The reference multiplies by 100**m before the square root and 10**-m after;
    both are 1 at m = 0.  Only NORM(:, m=0) is read on the hot path
    (DELSQH/XXDX/DEL2/IDEL2LN/IHELM/VEL2PLN/IDELSQH log-term rows).
    """
    out = np.zeros(ndim)
    out[0] = 0.5
    for nn in range(2, ndim + 1):
        n = nn - 1
        out[nn - 1] = out[nn - 2] * (2 * n + 1.0) / (2 * n - 1.0) * n / n
    return np.sqrt(out)


def leg_table(x, ne, ms):
    """Orthonormal associated Legendre table PF(i, nn, mm) = Pbar^m_{m+nn-1}(x_i).

    Same functions as LEG_TBL3 (mod_lin_legendre.f90:526-644): Condon-Shortley
    phase (-1)^m, normalised so that int_{-1}^{1} Pbar^2 dx = 1.  The reference
    runs the unnormalised recurrence in 50-digit FM arithmetic to dodge
    under/overflow and flushes values below the FP64 range to zero (617-633).
    Here the standard normalised three-term recurrence runs in 80-bit extended
    precision (exponent range 1e+-4932, so nothing underflows before the final
    rounding), then values below the FP64 normal range are flushed to zero
    like the reference.  Pinned against 50-digit mpmath restatements of
    LEG_TBL3 in tests/golden/.
    """
    ld = np.longdouble
    x = np.asarray(x, dtype=ld)
    s2 = (ld(1) - x * x)
    out = np.zeros((len(x), ne, len(ms)), dtype=np.float64)
    tiny = np.finfo(np.float64).tiny
    for mm, m in enumerate(ms):
        m = abs(int(m))
        # Pbar^m_m = (-1)^m sqrt((2m+1)/2 * (2m-1)!!^2/(2m)!) (1-x^2)^(m/2)
        c = ld(0.5)
        for k in range(1, m + 1):
            c *= ld(2 * k + 1) / ld(2 * k * (2 * k - 1) ** 2) * ld(2 * k - 1) ** 2
        p0 = ((-1) ** m) * np.sqrt(c) * np.power(s2, ld(m) / 2)
        vals = np.zeros((len(x), ne), dtype=ld)
        vals[:, 0] = p0
        if ne > 1:
            vals[:, 1] = x * np.sqrt(ld(2 * m + 3)) * p0
        for nn in range(2, ne):
            n = m + nn
            a = np.sqrt(ld(4 * n * n - 1) / ld(n * n - m * m))
            b = np.sqrt(ld((n - 1) ** 2 - m * m) * ld(2 * n + 1) / (ld(n * n - m * m) * ld(2 * n - 3)))
            vals[:, nn] = a * x * vals[:, nn - 1] - b * vals[:, nn - 2]
        v = vals.astype(np.float64)
        v[np.abs(v) < tiny] = 0.0
        out[:, :, mm] = v
    return out


class Grid:
    """LEGINIT (mod_fft.f90:180-367) for a single process, plus the chop state.

    Parameters follow read.input: nr, nth, nx, nrchop, ntchop, nxchop, ell, zlen.
    MINC = 1 and MKLINK = 0 (the only values the configured runs use).
    """

    def __init__(self, nr, nth, nx, nrchop, ntchop, nxchop, ell=1.0, zlen=2 * math.pi):
        self.NR, self.NTH, self.NX = nr, nth, nx
        self.ELL = float(ell)
        self.ELL2 = self.ELL ** 2.0
        self.ZLEN = float(zlen)
        self.NRH = nr // 2
        self.NDIMR = nr + 3
        self.NDIMTH = nth + 1
        self.NDIMX = nx
        self.NRCHOP0 = nrchop
        self.NRCHOP = nrchop
        self.NTCHOP = ntchop
        self.NXCHOP = nxchop
        self.NRCHOPDIM = min(nrchop + 6, nr)          # mod_fft.f90:231
        self.NTCHOPDIM = min(ntchop, nth)
        self.NXCHOPDIM = nxchop * 2 - 1
        self.NXCHOPH = nx - nxchop + 2
        if nxchop == 1:
            self.NXCHOPH = 1
        if 2 * nxchop > nx and (nx > 1 or nxchop > 1):   # mod_fft.f90:237-243
            raise ValueError("NXCHOP MUST BE < NX/2, UNLESS NX = NXCHOP = 1")
        self.M = np.arange(self.NTCHOPDIM)              # MINC*(MM-1)
        self.chop_offset = 0
        self.NRCHOPS = np.zeros(nth, dtype=np.int64)
        self._set_nrchops()
        kv = np.arange(self.NXCHOPDIM)
        kv = np.where(kv + 1 > nxchop, -(self.NXCHOPDIM - (kv + 1) + 1), kv)
        self.KV = kv
        self.AK = np.tile(2 * math.pi / self.ZLEN * kv, (self.NTCHOPDIM, 1))  # AK(MM,KK)
        # TFM kit
        self.X, self.W = gauss_legendre(nr)
        self.R = self.ELL * np.sqrt((1 + self.X) / (1 - self.X))
        self.LNX = -np.log(1 - self.X)                   # TFM%LN, mod_fft.f90:287
        self.NORM0 = leg_norm_m0(self.NRCHOPDIM + 14)    # TFM%NORM(:,1)
        self.LOGNORM = leg_log_norm(self.NRCHOPDIM + 14, self.M)
        self.PF = leg_table(self.X[:self.NRH], self.NRCHOPDIM + 1, self.M)
        n = np.arange(self.NRCHOPDIM)
        self.AT1 = np.sqrt((2 * n + 1) / 2.0)            # Pbar_n(+1), mod_fft.f90:304
        self.AT0 = self.AT1 * (-1.0) ** n                # Pbar_n(-1), mod_fft.f90:303
        self.THR = 2 * math.pi / nth * np.arange(nth + 1)
        self.THI = 2 * math.pi / nth * (np.arange(nth + 1) + 0.5)
        self.Z = self.ZLEN * np.arange(nx + 1) / nx

    # ------------------------------------------------------------------
    def _set_nrchops(self):
        nrdeg = self.NRCHOP
        self.NRCHOPS[:] = 0
        for mm in range(self.NTCHOPDIM):
            self.NRCHOPS[mm] = max(min(self.NRCHOP, nrdeg - int(self.M[mm])), 0)

    def chopset(self, iof):
        """CHOPSET(IOF), mod_scalar3.f90:165-211."""
        self.NRCHOP += iof
        self.chop_offset += iof
        if self.NRCHOP > self.NRCHOPDIM:
            raise ValueError("CHOPSET: NRCHOP TOO LARGE (%d > %d)" % (self.NRCHOP, self.NRCHOPDIM))
        self._set_nrchops()

    # ------------------------------------------------------------------
    def shape(self, space):
        if space == FFF:
            return (self.NRCHOPDIM, self.NTCHOPDIM, self.NXCHOPDIM)
        if space == PFF:
            return (self.NDIMR, self.NTCHOPDIM, self.NXCHOPDIM)
        return (self.NDIMR, self.NDIMTH, self.NDIMX)

    def alloc(self, space=FFF):
        """SALLOC (mod_fft.f90:603-670); zero-filled (the reference leaves the
        array uninitialised and relies on CHOPDO / full overwrites)."""
        return Field(np.zeros(self.shape(space), dtype=np.complex128), space, 0.0)

    def chopdo(self, A):
        """CHOPDO(A), mod_scalar3.f90:213-257."""
        E = A.E
        if A.space == FFF:
            for mm in range(min(E.shape[1], self.NTCHOP)):
                E[self.NRCHOPS[mm]:, mm, :] = 0
            E[:, self.NTCHOP:, :] = 0
        elif A.space == PFF:
            E[self.NR:, :, :] = 0
        else:
            if A.space == PPP:
                E[:, self.NTH, :] = 0
            E[self.NR:, :, :] = 0
        return A

    def copy0(self, A):
        """B = A (COPY0, mod_fft.f90:705-769): copy, then CHOPDO for FFF."""
        B = A.copy()
        if B.space == FFF:
            self.chopdo(B)
        return B

    def calcat1(self, A):
        """CALCAT1 (mod_scalar3.f90:286-310): value at r = inf per k (m = 0)."""
        n = self.NRCHOP
        return self.AT1[:n] @ A.E[:n, 0, :]

    def calcat0(self, A):
        """CALCAT0 (mod_scalar3.f90:262-284): value at r = 0 per k (m = 0)."""
        n = self.NRCHOP
        return self.AT0[:n] @ A.E[:n, 0, :]
