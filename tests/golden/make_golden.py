"""Generate the golden fixtures that pin the oracle (and, through it, the GPU).

Run from the repository root:  python tests/golden/make_golden.py

legendre_golden.npz -- for (NR, m-set, NE) cases:
  * Gauss-Legendre nodes and weights at 50 digits (mpmath), the values
    GAUSS_LEGENDRE (mod_lin_legendre.f90:79-131) converges to in FP64;
  * the orthonormal associated Legendre table PF(i, nn, m) evaluated at the
    FP64-rounded nodes with the recurrence of LEG_TBL3
    (mod_lin_legendre.f90:567-616) in 50-digit arithmetic -- the reference
    runs it in FM with FM_SET(50) -- normalised with the exact norm
    (the reference multiplies by exp(LOGNORM + LOGFACT) computed in FP64,
    which differs from exact by ~1e-14 relative at the largest degrees);
    values below the FP64 normal range are flushed to zero as in 617-633.
  * LOGNORM from LEG_LOG_NORMT (mod_lin_legendre.f90:306-377) in 50 digits.
These are restatements of the reference's algorithm (the Fortran itself
cannot be compiled in this environment: no Fortran compiler, MPI or FFTW).
"""

import os

import mpmath as mp
import numpy as np

mp.mp.dps = 50
HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    (16, [0, 1, 2, 5], 12),
    (64, [0, 3, 15], 64),
    (192, [0, 42, 84], 135),     # the headline grid's extremes (m = 84 is NTCHOPDIM-1)
    (256, [169], 40),            # m where (1-x^2)^(m/2) underflows FP64 near x = +-1
]


def _pn(n, z):
    p1, p2 = mp.mpf(1), mp.mpf(0)
    for j in range(1, n + 1):
        p3, p2 = p2, p1
        p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j
    return p1, n * (z * p1 - p2) / (z * z - 1)


def gauss(n):
    """Nodes/weights at 50 digits: Newton on P_n from the FP64 nodes."""
    x0, _ = np.polynomial.legendre.leggauss(n)
    xs, ws = [], []
    for xv in x0:
        z = mp.mpf(float(xv))
        for _ in range(60):
            p, dp = _pn(n, z)
            dz = p / dp
            z -= dz
            if abs(dz) < mp.mpf(10) ** -48:
                break
        p, dp = _pn(n, z)
        xs.append(z)
        ws.append(2 / ((1 - z * z) * dp * dp))
    return xs, ws


def lognorm(ndim, m):
    wk = mp.log(mp.mpf(1) / 2)
    for mm in range(1, m + 1):
        wk += mp.log(2 * mm + 1) - mp.log(2 * mm * (2 * mm - 1) ** 2)
    out = [wk]
    for nn in range(2, ndim + 1):
        n = m + nn - 1
        out.append(out[-1] + mp.log(2 * n + 1) - mp.log(2 * n - 1) + mp.log(n - m) - mp.log(n + m))
    return [v / 2 for v in out]


def table(xd, ne, m):
    """LEG_TBL3 recurrence at 50 digits, exact normalisation (see module doc)."""
    ln = lognorm(ne, m)
    out = np.zeros((len(xd), ne))
    tiny = np.finfo(np.float64).tiny
    for ii, xv in enumerate(xd):
        x = mp.mpf(float(xv))
        q = [mp.mpf(0)] * ne
        q[0] = (-1) ** m * mp.sqrt(1 - x * x) ** m if m else mp.mpf(1)
        if ne > 1:
            q[1] = x * q[0]
        for nn in range(3, ne + 1):
            n = m + nn - 1
            q[nn - 1] = (q[nn - 2] * x - q[nn - 3] * (n + m - 1) / (2 * n - 1) / (2 * n - 3)) / (n - m)
        for nn in range(1, ne + 1):
            n = m + nn - 1
            logfact = mp.loggamma(2 * n + 1) - n * mp.log(2) - mp.loggamma(n + 1)
            v = float(q[nn - 1] * mp.exp(ln[nn - 1] + logfact))
            out[ii, nn - 1] = 0.0 if abs(v) < tiny else v
    return out


def main():
    data = {}
    for ci, (nr, ms, ne) in enumerate(CASES):
        xs, ws = gauss(nr)
        xd = np.array([float(v) for v in xs])
        data["c%d_nr" % ci] = np.array(nr)
        data["c%d_ms" % ci] = np.array(ms)
        data["c%d_x" % ci] = xd
        data["c%d_w" % ci] = np.array([float(v) for v in ws])
        nrh = nr // 2
        data["c%d_pf" % ci] = np.stack([table(xd[:nrh], ne, m) for m in ms], axis=2)
        data["c%d_lognorm" % ci] = np.stack([np.array([float(v) for v in lognorm(ne + 14, m)])
                                             for m in ms], axis=1)
        print("case", ci, nr, ms, ne, "done", flush=True)
    np.savez_compressed(os.path.join(HERE, "legendre_golden.npz"), **data)


if __name__ == "__main__":
    main()
