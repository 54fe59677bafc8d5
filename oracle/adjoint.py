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
  vprodsub_T          the VPRODSUB cross products (mod_legops.f90:2105-2130),
                      pointwise in PPP
  mulxm_T, xxdx_T, delsqh_T, del2_T   MULXM (371-428), XXDX (680-748), DELSQH
                      (76-133), DEL2 (751-820), log-term rows included
  grad_T, pc2vel_T, pc2vor_T          GRAD (1727-1786), PC2VEL (1789-1853),
                      PC2VOR (1856-1919)
  vdotpsub_T          VDOTPSUB (2136-2232), pointwise in PPP
  project_T           PROJECT (2397-2545) of PFF inputs without the log term,
                      with EOMUL/OEMUL (2548-2648) and the far-field fix
                      (farfield_T, CALCAT1 of mod_scalar3.f90:286-310)
  vel2pln_T           VEL2PLN's update of RUP (2277-2339)
  idel2ln_T, idel2_T  IDEL2LN (1013-1176), IDEL2 (823-1010): transposed banded
                      solves with their log columns, row shift and far field
  boussi_nonlin_vjp   CALC_BOUSSI_NONLIN (mod_boussinesq.f90:235-314)
  etdab_cn_step_vjp   one steady STEP_BOUSSI_ETDAB_CN (mod_march.f90:811-901)
                      as a map of the whole state (psi, chi, b, history)
  ihelm_T, visc2_T    IHELM (1204-1354), VISC2 (mod_march.f90:1579-1636)
  boussi_force_vjp    CALC_BOUSSI_FORCE (mod_boussinesq.f90:317-410)
  ab_cn_step_vjp      one steady STEP_BOUSSI_AB_CN (mod_march.f90:609-661)
  trajectory_grad     reverse accumulation of the step VJPs over a trajectory
  energy_objective(_grad)  J = KE of the fluctuations + 1/2 int b^2 dV
                      (mod_boussinesq.f90:112-206 quadratures) and its gradient
  visc1_T, rich_fe_be_vjp  VISC1 (mod_march.f90:1529-1576), RICH_BOUSSI_FE_BE
                      (535-606)
  idelsqh_T, initial_state_T  IDELSQH (mod_legops.f90:136-241) and the seeded
                      initial state's dependence on its perturbation coefficients
  etdfe_be_vjp, rich_etdfe_be_vjp  STEP_BOUSSI_ETDFE_BE (mod_march.f90:664-753)
                      and RICH_BOUSSI_ETDFE_BE (756-808)

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


# ----------------------------------------------------------------------
# FFF operators (mod_legops.f90).  Per (m, k) column each is a real band
# matrix M acting on the rows n < NRCHOPS(m), so the adjoint applies M^T; the
# (m, k) = (0, 0) log-term rows give LN_bar = sum_rows coef * Re Y(row, 0, 0).

def _band_T(g, Y, make_band, c):
    from .bandmat import band_to_full
    y = _field(Y.E, FFF)
    g.chopdo(y)
    A = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        full = band_to_full(make_band(nn, mm), c, nn)
        A.E[:nn, mm, :] = full.T @ y.E[:nn, mm, :]
    return A, y


def mulxm_T(g, Y):
    """Adjoint of MULXM (371-428)."""
    from .bandmat import band_xm
    A, _ = _band_T(g, Y, lambda nn, mm: band_xm(nn, g.M[mm], g.LOGNORM[:, mm]), 1)
    return A


def xxdx_T(g, Y):
    """Adjoint of XXDX (680-748) with its log-term rows (742-745)."""
    from .bandmat import band_xxdx
    A, y = _band_T(g, Y, lambda nn, mm: band_xxdx(nn, g.M[mm], g.LOGNORM[:, mm]), 1)
    A.LN = float(y.E[0, 0, 0].real / g.NORM0[0] + y.E[1, 0, 0].real / g.NORM0[1])
    return A


def delsqh_T(g, Y):
    """Adjoint of DELSQH (76-133): the diagonal -n(n+1)/L^2, and B(0,0,0) = LN / L^2 / NORM(1,1)."""
    y = _field(Y.E, FFF)
    g.chopdo(y)
    A = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        n = g.M[mm] + np.arange(nn)
        A.E[:nn, mm, :] = -y.E[:nn, mm, :] * (n * (n + 1) / g.ELL2)[:, None]
    A.E[0, 0, 0] = 0.0                      # the forward overwrites B(0, 0, 0)
    A.LN = float(y.E[0, 0, 0].real / g.ELL2 / g.NORM0[0])
    return A


def del2_T(g, Y):
    """Adjoint of DEL2 (751-820): band del^2_h minus k^2, log-term rows 813-817."""
    from .bandmat import band_del2h, band_to_full
    y = _field(Y.E, FFF)
    g.chopdo(y)
    A = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        full = band_to_full(band_del2h(nn, g.M[mm], g.ELL, g.LOGNORM[:, mm]), 2, nn)
        A.E[:nn, mm, :] = full.T @ y.E[:nn, mm, :] - (g.AK[mm, :] ** 2)[None, :] * y.E[:nn, mm, :]
    A.LN = float((4.0 / 3 * y.E[0, 0, 0].real / g.NORM0[0] - 2.0 * y.E[1, 0, 0].real / g.NORM0[1]
                  + 2.0 / 3 * y.E[2, 0, 0].real / g.NORM0[2]) / g.ELL2)
    return A


def _scale_T(g, Y, fac):
    """Adjoint of A -> fac(m, k) A on rows n < NRCHOPS(m): multiply by conj(fac)."""
    A = g.alloc(FFF)
    for mm in range(A.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        A.E[:nn, mm, :] = np.conj(fac(mm))[None, :] * Y.E[:nn, mm, :]
    return A


def _add(*fs):
    out = fs[0].copy()
    for f in fs[1:]:
        out.E = out.E + f.E
        out.LN = out.LN + f.LN
    return out


def grad_T(g, RR, RP, GZ):
    """Adjoint of GRAD (1727-1786) -> A_bar (FFF, with LN_bar)."""
    a = xxdx_T(g, RR)
    b = _scale_T(g, RP, lambda mm: 1j * g.M[mm] * np.ones(g.NXCHOPDIM))
    c = _scale_T(g, GZ, lambda mm: 1j * g.AK[mm, :])
    return _add(a, b, c)


def _neg(F):
    out = F.copy()
    out.E = -out.E
    out.LN = -out.LN
    return out


def pc2vel_T(g, RUR, RUP, UZ):
    """Adjoint of PC2VEL (1789-1853) -> (PSI_bar, CHI_bar)."""
    kv = lambda mm: g.AK[mm, :]
    mv = lambda mm: g.M[mm] * np.ones(g.NXCHOPDIM)
    # RUR = i m PSI + i k XXDX(CHI);  RUP = -XXDX(PSI) - m k CHI;  UZ = -MULXM(MULXM(DELSQH(CHI)))
    psi = _add(_scale_T(g, RUR, lambda mm: 1j * mv(mm)), _neg(xxdx_T(g, _field(RUP.E, FFF))))
    chi = _add(xxdx_T(g, _scale_T(g, RUR, lambda mm: 1j * kv(mm))),
               _scale_T(g, RUP, lambda mm: -mv(mm) * kv(mm)),
               delsqh_T(g, mulxm_T(g, mulxm_T(g, _neg(_field(UZ.E, FFF))))))
    return psi, chi


def pc2vor_T(g, ROR, ROP, OZ):
    """Adjoint of PC2VOR (1856-1919) -> (PSI_bar, CHI_bar)."""
    kv = lambda mm: g.AK[mm, :]
    mv = lambda mm: g.M[mm] * np.ones(g.NXCHOPDIM)
    # W = DEL2(CHI); ROR = -i m W + i k XXDX(PSI); ROP = XXDX(W) - k m PSI;
    # OZ = -MULXM(MULXM(DELSQH(PSI)))
    w_bar = _add(_scale_T(g, ROR, lambda mm: -1j * mv(mm)), xxdx_T(g, _field(ROP.E, FFF)))
    chi = del2_T(g, w_bar)
    psi = _add(xxdx_T(g, _scale_T(g, ROR, lambda mm: 1j * kv(mm))),
               _scale_T(g, ROP, lambda mm: -kv(mm) * mv(mm)),
               delsqh_T(g, mulxm_T(g, mulxm_T(g, _neg(_field(OZ.E, FFF))))))
    return psi, chi


def vdotpsub_T(g, A, B, Y):
    """Adjoint of VDOTPSUB (2136-2232), out = (a1 b1 + a2 b2)/r^2 + a3 b3 per
    packed part: returns (A_bar, B_bar), lists of three PPP arrays."""
    r2 = (g.R[:g.NR] ** 2)[:, None, None]
    sl = (slice(0, g.NR), slice(0, g.NTH), slice(None))
    out_a = [np.zeros_like(A[0]) for _ in range(3)]
    out_b = [np.zeros_like(A[0]) for _ in range(3)]
    for part, f in ((0, 1.0), (1, 1j)):
        pick = (lambda a: a.real) if part == 0 else (lambda a: a.imag)
        a = [pick(x[sl]) for x in A]
        b = [pick(x[sl]) for x in B]
        y = pick(Y[sl])
        w = [y / r2, y / r2, y]
        for q in range(3):
            out_a[q][sl] += f * (w[q] * b[q])
            out_b[q][sl] += f * (w[q] * a[q])
    return out_a, out_b


def _fold_T(A, Cbar, nj, odd_first):
    """Adjoint of EOMUL (odd_first False) / OEMUL (True) with respect to B:
    C = A[0::2] . (even or odd fold of B), C[1::2] = A[1::2] . (the other)."""
    njh = A.shape[1]
    x0 = A[0::2].T @ Cbar[0::2]
    x1 = A[1::2].T @ Cbar[1::2] if A.shape[0] > 1 else np.zeros_like(x0)
    be_bar, bo_bar = (x1, x0) if odd_first else (x0, x1)
    Bbar = np.zeros((nj,) + Cbar.shape[1:], dtype=np.complex128)
    Bbar[:njh] = be_bar + bo_bar
    Bbar[nj - 1:njh - 1:-1] = be_bar - bo_bar
    return Bbar


def farfield_T(g, Y):
    """Adjoint of the far-field fix PSI(1,1,:) -= CALCAT1(PSI)/AT1(1)
    (mod_legops.f90:2540; CALCAT1 mod_scalar3.f90:286-310) on a chopped field:
    row 0 of m = 0 becomes -sum_{1 <= n < NRCHOP} AT1(n)/AT1(0) row n."""
    X = _field(Y.E, FFF, Y.LN)
    nr = g.NRCHOP
    y0 = np.array(Y.E[0, 0, :])
    X.E[1:nr, 0, :] = Y.E[1:nr, 0, :] - (g.AT1[1:nr] / g.AT1[0])[:, None] * y0[None, :]
    X.E[0, 0, :] = 0.0
    return X


def project_T(g, PSI_bar, CHI_bar):
    """Adjoint of PROJECT (2397-2545) of PFF inputs without log-term handling
    (LN absent): returns (RUR_bar, RUP_bar, UZ_bar) in PFF."""
    from .legops import project_weights
    nr = g.NR
    ps = farfield_T(g, PSI_bar)
    g.chopdo(ps)
    ch = _field(CHI_bar.E, FFF)
    g.chopdo(ch)
    out = [g.alloc(PFF) for _ in range(3)]
    for mm in range(ps.E.shape[1]):
        mv = int(g.M[mm])
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        V, D, T = project_weights(g, mm)
        kv = g.AK[mm, :][None, :]
        yp = ps.E[:nn, mm, :]
        yc = ch.E[:nn, mm, :]
        # PSI = -(i m) EO(V, rur) - OE(D, rup);  CHI = (i k) OE(D, rur) + m k EO(V, rup) - EO(T, uz)
        rur = _fold_T(D, np.conj(1j * kv) * yc, nr, True)
        rup = _fold_T(D, -yp, nr, True)
        if mv != 0:
            rur = rur + _fold_T(V, np.conj(-1j * mv) * yp, nr, False)
            rup = rup + _fold_T(V, (mv * kv) * yc, nr, False)
        uz = _fold_T(T, -yc, nr, False)
        out[0].E[:nr, mm, :] = rur
        out[1].E[:nr, mm, :] = rup
        out[2].E[:nr, mm, :] = uz
    return out


def _solve_T_column(band, c, nn, y):
    """x with M^T x = y, M the dense form of a (nn x nn) band (the transposed
    banded solve; the forward runs the unpivoted band LU of M)."""
    from .bandmat import band_to_full
    return np.linalg.solve(band_to_full(band[:nn], c, nn).T, y)


def idel2ln_T(g, A_bar):
    """Adjoint of IDEL2LN(B, A) (mod_legops.f90:1013-1176) as the map
    B -> (A, A%LN): the far-field fix, CHOPDO, the transposed m >= 1 penta-band
    solves, A%LN = Re A(1,1,1) NORM(1,1) with A(1,1,1) then zeroed, and the
    transposed m = 0 solves (the (m, k) = (0, 0) system carries the log column
    of 1091-1107).  B%LN does not enter, so B_bar%LN = 0."""
    from .bandmat import band_del2h
    y = farfield_T(g, A_bar)
    g.chopdo(y)
    Bb = g.alloc(FFF)
    K = y.E.shape[2]
    n0 = g.NORM0
    for mm in range(1, y.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        band0 = band_del2h(nn, g.M[mm], g.ELL, g.LOGNORM[:, mm])
        for kk in range(K):
            band = band0.copy()
            band[:, 2] -= g.AK[mm, kk] ** 2
            Bb.E[:nn, mm, kk] = _solve_T_column(band, 2, nn, y.E[:nn, mm, kk])
    nn = int(g.NRCHOPS[0])
    d0 = band_del2h(nn + 1, g.M[0], g.ELL, g.LOGNORM[:, 0])
    x_bar = np.array(y.E[:nn, 0, :])
    x_bar[0, 0] = A_bar.LN * n0[0]            # A(1,1,1) was replaced by the log term
    for kk in range(K):
        band = d0.copy()
        band[:, 2] -= g.AK[0, kk] ** 2
        if kk == 0:
            band[0, 2] += 4.0 / 3 / g.ELL2
            band[1, 1] -= 2 * n0[0] / n0[1] / g.ELL2
            band[2, 0] += 2.0 / 3 * n0[0] / n0[2] / g.ELL2
        Bb.E[:nn, 0, kk] = _solve_T_column(band, 2, nn, x_bar[:, kk])
    g.chopdo(Bb)
    Bb.LN = 0.0
    return Bb


def idel2_T(g, A_bar):
    """Adjoint of IDEL2(B, A) without LN (mod_legops.f90:823-1010): the
    far-field fix, CHOPDO, the transposed m >= 1 penta-band solves and the
    transposed m = 0 7-band solves, where (m, k) = (0, 0) carries the log
    column and solves the right-hand side shifted down one row (917-936)."""
    from .bandmat import band_del2h
    y = farfield_T(g, A_bar)
    g.chopdo(y)
    Bb = g.alloc(FFF)
    K = y.E.shape[2]
    n0 = g.NORM0
    for mm in range(1, y.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        band0 = band_del2h(nn, g.M[mm], g.ELL, g.LOGNORM[:, mm])
        for kk in range(K):
            band = band0.copy()
            band[:, 2] -= g.AK[mm, kk] ** 2
            Bb.E[:nn, mm, kk] = _solve_T_column(band, 2, nn, y.E[:nn, mm, kk])
    nn = int(g.NRCHOPS[0])
    np_ = nn + 1
    d0 = np.zeros((np_, 7))
    d0[:, 1:6] = band_del2h(np_, g.M[0], g.ELL, g.LOGNORM[:, 0])
    for kk in range(K):
        o = d0.copy()
        o[:, 3] -= g.AK[0, kk] ** 2
        if kk == 0:
            o[0, 3] += 4.0 / 3 / g.ELL2
            o[1, 2] -= 2 * n0[0] / n0[1] / g.ELL2
            o[2, 1] += 2.0 / 3 * n0[0] / n0[2] / g.ELL2
            o[1:np_, 0:5] = o[0:np_ - 1, 1:6].copy()
            o[:, 5:7] = 0
            o[0, :] = 0
            o[0, 3] = 1
        b_bar = _solve_T_column(o, 3, nn, y.E[:nn, 0, kk])
        if kk == 0:           # the right-hand side was shifted down one row, row 0 <- 0
            shifted = np.zeros_like(b_bar)
            shifted[:nn - 1] = b_bar[1:nn]
            b_bar = shifted
        Bb.E[:nn, 0, kk] = b_bar
    g.chopdo(Bb)
    Bb.LN = 0.0
    return Bb


def _vel2pln_vectors(g):
    """VEL2PLN (2277-2339) as line -> line - v (c . Re line) on the (m, k) =
    (0, 0) PFF line: c gives PSI%LN = c . Re line, v the removed -LN (1 + x)."""
    nr, nrh = g.NR, g.NRH
    w = g.W[:nrh]
    nn = int(g.NRCHOPS[0])
    pf = g.PF[:nrh, :, 0]
    e = np.exp(g.LOGNORM[:nn, 0])
    se = pf[:, 0:nn:2] @ e[0:nn:2]
    so = pf[:, 1:nn:2] @ e[1:nn:2]
    c = np.zeros(nr)
    c[:nrh] = -0.5 * w * (se + so)
    c[nr - 1:nrh - 1:-1] = -0.5 * w * (se - so)
    v = np.zeros(nr)
    v[:nrh] = -(pf[:, 0] / g.NORM0[0] + pf[:, 1] / g.NORM0[1])
    v[nr - 1:nrh - 1:-1] = -(pf[:, 0] / g.NORM0[0] - pf[:, 1] / g.NORM0[1])
    return c, v


def vel2pln_T(g, RUP_bar):
    """Adjoint of the in-place VEL2PLN update of RUP (PFF) with LN given: only
    the real part of the (0, 0) line changes, line - v (c . Re line)."""
    c, v = _vel2pln_vectors(g)
    out = _field(RUP_bar.E, PFF)
    nr = g.NR
    y = out.E[:nr, 0, 0]
    out.E[:nr, 0, 0] = (y.real - c * np.dot(v, y.real)) + 1j * y.imag
    return out


def project_ppp_ln0_T(g, PSI_bar, W_bar):
    """Adjoint of PROJECT(ROR, ROP, OZ, PSI, W, 0.0) on PPP inputs, as
    CALC_BOUSSI_NONLIN calls it (mod_boussinesq.f90:283): PLNFFT(-1) of the
    three inputs (HORFFT(-1) then VERFFT(-1)), VEL2PLN with LN = 0 on RUP, the
    fold products and the far-field fix.  PSI%LN is set to 0, so it has no
    cotangent."""
    bars = project_T(g, PSI_bar, W_bar)
    bars[1] = vel2pln_T(g, bars[1])
    return [horfft_T(g, verfft_T(g, b, -1), -1) for b in bars]


def boussi_nonlin_vjp(g, B, RUR, RUP, UZ, ROR, ROP, OZ, BN_bar, NR_bar, NP_bar, NZ_bar):
    """Vector-Jacobian product of CALC_BOUSSI_NONLIN (mod_boussinesq.f90:235-314,
    oracle/boussinesq.calc_boussi_nonlin): inputs B and the FFF velocity and
    vorticity, outputs BN and the velocity form (NR, NP, NZ) of the projected
    u x omega.  Returns the cotangents (B, RUR, RUP, UZ, ROR, ROP, OZ), FFF with LN."""
    from .legops import grad, idel2, project, vdotpsub, vprodsub
    from .transforms import tofp
    # forward, keeping what the products need
    g.chopset(1)
    G = grad(g, B)
    g.chopset(-1)
    U = [tofp(g, F.copy()) for F in (RUR, RUP, UZ)]
    Wv = [tofp(g, F.copy()) for F in (ROR, ROP, OZ)]
    Gp = [tofp(g, F) for F in G]
    Nv = [F.copy() for F in Wv]
    vprodsub(g, *[F.copy() for F in U], *Nv)
    PSI, W = project(g, *[F.copy() for F in Nv], 0.0)
    # reverse
    g.chopset(3)
    psi_bar, chi_bar = pc2vel_T(g, NR_bar, NP_bar, NZ_bar)
    g.chopset(-3)
    w_bar = idel2_T(g, chi_bar)
    nv_bar = project_ppp_ln0_T(g, psi_bar, w_bar)
    bn_ppp_bar = toff_T(g, BN_bar)
    u_bar1, w_bar1 = vprodsub_T(g, [F.E for F in U], [F.E for F in Wv], [F.E for F in nv_bar])
    u_bar2, g_bar = vdotpsub_T(g, [F.E for F in U], [F.E for F in Gp], -bn_ppp_bar.E)
    ins = []
    for q in range(3):
        ins.append(tofp_T(g, _field(u_bar1[q] + u_bar2[q], PPP)))
    for q in range(3):
        ins.append(tofp_T(g, _field(w_bar1[q], PPP)))
    g_fff = [tofp_T(g, _field(gb, PPP)) for gb in g_bar]
    g.chopset(1)
    b_bar = grad_T(g, *g_fff)
    g.chopset(-1)
    return [b_bar] + ins


HISTORY = ("r_pi_r", "r_pi_p", "pi_z", "r_n_r", "r_n_p", "n_z", "n_b")


def etdab_cn_step_vjp(s, bars):
    """Vector-Jacobian product of one steady STEP_BOUSSI_ETDAB_CN
    (mod_march.f90:811-901, oracle Solver._step_etdab_cn with VISC%SW = 3 and
    no sponge) as the map of the state (psi, chi, b and the seven history
    fields) to the next state.  s: an oracle Solver holding the state before
    the step (not changed); bars: dict of output cotangents keyed "psi", "chi",
    "b" and HISTORY (FFF Fields; psi and chi with LN).  Returns the input
    cotangents in a dict with the same keys."""
    from .boussinesq import calc_boussi_etdab_sub, calc_boussi_nonlin, _etd_mats
    from .legops import idel2ln, pc2vel, pc2vor, project
    g, ph, dt = s.g, s.ph, s.ph.dt
    tf = 1.0
    hyp = s.hyp

    def filt(F, which):
        out = _field(F.E, FFF, F.LN)
        if hyp is not None:
            hyp._apply(g, out, hyp.hv if which == "v" else hyp.hd, tf)
        return out

    # ---- forward, keeping the intermediates
    PSI, CHI, B = s.psi, s.chi, s.b
    g.chopset(3)
    V = pc2vel(g, PSI, CHI)
    Om = pc2vor(g, PSI, CHI)
    g.chopset(-3)
    BN, NR_, NP_, NZ_ = calc_boussi_nonlin(g, B.copy(), *[F.copy() for F in V], *[F.copy() for F in Om])
    Nf = [filt(F, "v") for F in (NR_, NP_, NZ_)] + [filt(BN, "d")]
    Vw = [F.copy() for F in V]
    Bw = B.copy()
    calc_boussi_etdab_sub(s, Bw, *Vw, Nf[3], Nf[0], Nf[1], Nf[2], dt)
    Vf = [filt(F, "v") for F in Vw]
    Bf = filt(Bw, "d")
    PSI1, W = project(g, *[F.copy() for F in Vf], "psi")
    CHI1 = idel2ln(g, W)

    # ---- reverse
    psi1_bar = _field(bars["psi"].E, FFF, bars["psi"].LN)
    chi1_bar = _field(bars["chi"].E, FFF, bars["chi"].LN)
    g.chopset(3)
    p_h, c_h = pc2vel_T(g, *[_neg(bars[k]) for k in ("r_pi_r", "r_pi_p", "pi_z")])
    g.chopset(-3)
    psi1_bar = _add(psi1_bar, p_h)
    chi1_bar = _add(chi1_bar, c_h)
    w_bar = idel2ln_T(g, chi1_bar)
    pb = project_T(g, psi1_bar, w_bar)
    c, _ = _vel2pln_vectors(g)
    pb[1] = vel2pln_T(g, pb[1])
    pb[1].E[:g.NR, 0, 0] += c * psi1_bar.LN                       # PSI%LN = c . Re line
    vf_bar = [_add(_field(bars[k].E, FFF), rtran_T(g, b_, 1))
              for k, b_ in zip(("r_pi_r", "r_pi_p", "pi_z"), pb)]
    for F in vf_bar:
        F.LN = 0.0
    # the filters after the update
    vw_bar = [filt(F, "v") for F in vf_bar]
    bw_bar = filt(_field(bars["b"].E, FFF), "d")
    # CALC_BOUSSI_ETDAB_SUB: cv = Er ev + Nr av per k
    K = B.E.shape[2]
    notm0 = np.ones(B.E.shape[1])
    notm0[0] = 0.0
    ev_bar = [np.zeros_like(B.E) for _ in range(4)]
    av_bar = [np.zeros_like(B.E) for _ in range(4)]
    cvb = [vw_bar[0].E, vw_bar[1].E, vw_bar[2].E, bw_bar.E]
    for kk in range(K):
        Er, Nr = _etd_mats(s.etd_e, s.etd_nl, dt, kk == 0)
        cv = np.stack([x[:, :, kk] for x in cvb])
        e_ = np.einsum("ji,j...->i...", Er, cv)
        a_ = np.einsum("ji,j...->i...", Nr, cv)
        for q in range(4):
            ev_bar[q][:, :, kk] = e_[q]
            av_bar[q][:, :, kk] = a_[q]
    notk0 = np.ones(K)
    notk0[0] = 0.0
    out = {}
    out["r_pi_r"] = _field(-ev_bar[0], FFF)
    out["r_pi_p"] = _field(-ev_bar[1] * notm0[None, :, None], FFF)
    out["pi_z"] = _field(-ev_bar[2] * notk0[None, None, :], FFF)
    for k, q in zip(("r_n_r", "r_n_p", "n_z", "n_b"), range(4)):
        out[k] = _field(-0.5 * av_bar[q], FFF)
    v_bar = [_field(ev_bar[q], FFF) for q in range(3)]
    b_bar = _field(ev_bar[3], FFF)
    nf_bar = [_field(1.5 * av_bar[q], FFF) for q in range(4)]
    for q, k in enumerate(("r_n_r", "r_n_p", "n_z", "n_b")):
        nf_bar[q].E = nf_bar[q].E + bars[k].E
    n_bar = [filt(nf_bar[q], "v") for q in range(3)] + [filt(nf_bar[3], "d")]
    nl = boussi_nonlin_vjp(g, B, *V, *Om, n_bar[3], n_bar[0], n_bar[1], n_bar[2])
    b_bar = _add(b_bar, nl[0])
    g.chopset(3)
    p1, c1 = pc2vel_T(g, *[_add(v_bar[q], nl[1 + q]) for q in range(3)])
    p2, c2 = pc2vor_T(g, *nl[4:7])
    g.chopset(-3)
    out["psi"] = _add(p1, p2)
    out["chi"] = _add(c1, c2)
    out["b"] = b_bar
    return out


STATE = ("psi", "chi", "b") + HISTORY


def trajectory_grad(s, nsteps, objective_grad):
    """Reverse-mode gradient through nsteps steady steps (AB2-CN or ETD2AB-CN,
    as s.ph.adams says) from the oracle Solver s (not changed): forward with
    every state kept, then the step VJPs in reverse.  objective_grad(final)
    returns the cotangents of the objective with respect to the final state
    (a dict over AB2_STATE or STATE).  Returns the gradient with respect to
    the state s holds."""
    import copy
    adams = s.ph.adams
    keys = AB2_STATE if adams else STATE
    traj = [copy.deepcopy(s)]
    for _ in range(nsteps):
        nxt = copy.deepcopy(traj[-1])
        if adams:
            nxt._step_ab_cn()
        else:
            nxt._step_etdab_cn()
        traj.append(nxt)
    bars = objective_grad({k: getattr(traj[-1], k) for k in keys})
    for i in range(nsteps - 1, -1, -1):
        bars = ab_cn_step_vjp(traj[i], bars) if adams else etdab_cn_step_vjp(traj[i], bars)
    return bars


def etd_trajectory_grad(s, nsteps, objective_grad):
    """trajectory_grad for an ETD2AB-CN solver."""
    return trajectory_grad(s, nsteps, objective_grad)


# ----------------------------------------------------------------------
# AB2-CN (mod_march.f90:609-661) pieces.

def ihelm_T(g, A_bar, alp):
    """Adjoint of IHELM(B, A, ALP) (mod_legops.f90:1204-1354) as the map
    (B, B%LN) -> (A, A%LN): m >= 1 transposed penta-band solves of
    (del^2_h - k^2 - alp); m = 0 the transposed (H XM) solve on NN-1 rows and
    XM^T; the log term A%LN = -B%LN/alp whose del^2 rows move to the rhs."""
    from .bandmat import band_del2h, band_to_full, band_xm, banbanmul
    y = _field(A_bar.E, FFF, A_bar.LN)
    g.chopdo(y)
    Bb = g.alloc(FFF)
    K = y.E.shape[2]
    for mm in range(1, y.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        band0 = band_del2h(nn, g.M[mm], g.ELL, g.LOGNORM[:, mm])
        band0[:, 2] -= alp
        for kk in range(K):
            band = band0.copy()
            band[:, 2] -= g.AK[mm, kk] ** 2
            Bb.E[:nn, mm, kk] = _solve_T_column(band, 2, nn, y.E[:nn, mm, kk])
    nn = int(g.NRCHOPS[0])
    np_, nm = nn + 1, nn - 1
    xm = band_xm(np_, g.M[0], g.LOGNORM[:, 0])
    xmf = band_to_full(xm[:nn], 1, nn)
    h0 = band_del2h(np_, g.M[0], g.ELL, g.LOGNORM[:, 0])
    h0[:, 2] -= alp
    for kk in range(K):
        h = h0.copy()
        h[:, 2] -= g.AK[0, kk] ** 2
        ops, _ = banbanmul(h, 2, xm, 1)
        w_bar = xmf.T @ y.E[:nn, 0, kk]
        Bb.E[:nm, 0, kk] = _solve_T_column(ops, 3, nm, w_bar[:nm])
        Bb.E[nm:nn, 0, kk] = 0.0
    g.chopdo(Bb)
    n0 = g.NORM0
    c = np.array([4.0 / 3 / g.ELL2 / n0[0], -2.0 / n0[1] / g.ELL2, 2.0 / 3 / n0[2] / g.ELL2])
    # rhs(0..2, 0, 0) = B - A%LN c = B + (B%LN / alp) c;  A%LN = -B%LN / alp
    Bb.LN = float(-y.LN / alp + np.dot(c, Bb.E[0:3, 0, 0].real) / alp)
    return Bb


def visc2_T(g, out_bar, nu, dt):
    """Adjoint of VISC2(A, AO, NU, DT) (mod_march.f90:1579-1636):
    WK = -CHOPDO(DEL2(AO) at CHOPSET(2)) - alp A, WK%LN = -alp A%LN,
    result IHELM(WK, alp), alp = 2/(NU DT).  Returns (A_bar, AO_bar)."""
    alp = 2 / nu / dt
    wk = ihelm_T(g, out_bar, alp)
    a_bar = _field(-alp * wk.E, FFF, -alp * wk.LN)
    t = _field(-wk.E, FFF)
    g.chopdo(t)
    g.chopset(2)
    ao_bar = del2_T(g, t)
    g.chopset(-2)
    return a_bar, ao_bar


def boussi_force_vjp(g, ph, PSI, CHI, B, PSIN_bar, CHIN_bar, BN_bar):
    """Vector-Jacobian product of CALC_BOUSSI_FORCE (mod_boussinesq.f90:317-410,
    oracle calc_boussi_force): returns (PSI_bar, CHI_bar, B_bar)."""
    from .legops import grad, pc2vel, pc2vor, vprodsub
    from .transforms import tofp
    g.chopset(3)
    G = grad(g, B)
    V = pc2vel(g, PSI, CHI)
    Om = pc2vor(g, PSI, CHI)
    U = [tofp(g, F.copy()) for F in V]
    Wv = [tofp(g, F.copy()) for F in Om]
    Gp = [tofp(g, F.copy()) for F in G]
    g.chopset(-3)
    w_bar = idel2ln_T(g, CHIN_bar)
    nb = project_ppp_ln0_T(g, _field(PSIN_bar.E, FFF), w_bar)
    bn = toff_T(g, BN_bar).E
    o2, n2 = 2 * ph.omega, ph.bv0 ** 2
    # ROR = N_r + 2 Omega RUP, ROP = N_t - 2 Omega RUR, OZ = N_z - W, BN = -VDOTP + N^2 UZ
    u_lin = [-o2 * nb[1].E, o2 * nb[0].E, n2 * bn]
    W_bar = _field(-nb[2].E, PPP)
    g.chopset(3)
    u1, wb = vprodsub_T(g, [F.E for F in U], [F.E for F in Wv], [F.E for F in nb])
    u2, gb = vdotpsub_T(g, [F.E for F in U], [F.E for F in Gp], -bn)
    ub = [tofp_T(g, _field(u1[q] + u2[q] + u_lin[q], PPP)) for q in range(3)]
    wbf = [tofp_T(g, _field(wb[q], PPP)) for q in range(3)]
    gbf = [tofp_T(g, _field(gb[q], PPP)) for q in range(3)]
    p1, c1 = pc2vel_T(g, *ub)
    p2, c2 = pc2vor_T(g, *wbf)
    b1 = grad_T(g, *gbf)
    g.chopset(-3)
    b2 = tofp_T(g, W_bar)
    g.chopdo(b2)
    return _add(p1, p2), _add(c1, c2), _add(b1, b2)


AB2_STATE = ("psi", "chi", "b", "n_psi", "n_chi", "n_b")


def ab_cn_step_vjp(s, bars):
    """Vector-Jacobian product of one steady STEP_BOUSSI_AB_CN (mod_march.f90:
    609-661) with VISC%SW = 1 as the map of (psi, chi, b, n_psi, n_chi, n_b)
    to the next state; s (an oracle Solver) is not changed."""
    from .boussinesq import calc_boussi_force
    g, ph, dt = s.g, s.ph, s.ph.dt
    if ph.visc_sw != 1:
        raise ValueError("ab_cn_step_vjp: VISC%SW = 1 only")
    PSI, CHI, B = s.psi, s.chi, s.b
    out = {}
    pairs = {}
    for k, nu in (("psi", ph.nu), ("chi", ph.nu), ("b", ph.kappa)):
        yb = _field(bars[k].E, FFF, bars[k].LN if k != "b" else 0.0)
        if nu != 0.0:
            a_bar, ao_bar = visc2_T(g, yb, nu, dt)
        else:
            a_bar, ao_bar = yb, _field(np.zeros_like(yb.E), FFF)
        if k == "b":
            a_bar.LN = 0.0
            ao_bar.LN = 0.0
        pairs[k] = (a_bar, ao_bar)
    force_bar = []
    for k, nk in (("psi", "n_psi"), ("chi", "n_chi"), ("b", "n_b")):
        a_bar, _ = pairs[k]
        h = _field(bars[nk].E, FFF, bars[nk].LN if k != "b" else 0.0)
        g.chopdo(h)
        fb = _field(1.5 * dt * a_bar.E + h.E, FFF, 1.5 * dt * a_bar.LN + h.LN)
        force_bar.append(fb)
        out[nk] = _field(-0.5 * dt * a_bar.E, FFF, -0.5 * dt * a_bar.LN)
    fp, fc, fbb = boussi_force_vjp(g, ph, PSI, CHI, B, *force_bar)
    for k, f in (("psi", fp), ("chi", fc), ("b", fbb)):
        a_bar, ao_bar = pairs[k]
        ao = _field(ao_bar.E, FFF, ao_bar.LN)
        g.chopdo(ao)
        out[k] = _add(a_bar, ao, f)
    out["b"].LN = 0.0
    return out


# ----------------------------------------------------------------------
# The gradient configuration's objective: J = KE(psi - psi_bar, chi - chi_bar)
# + 1/2 int b^2 dV, psi_bar, chi_bar the (m, k) = (0, 0) parts (log term
# included), KE in the quadrature form of CALC_BOUSSI_ENERGY
# (mod_boussinesq.f90:176-206: PRODCT_MK of RTRAN'd DELSQH / DEL2 at CHOPSET(3))
# and int b^2 dV = 2 x the summed CALC_BOUSSI_PE (mod_boussinesq.f90:112-136)
# times N^2.

def _pff_weights(g, inv_om2=False):
    """Per-entry weights of the PFF quadratures, 4 pi ZLEN ELL2 w_r (/(1-x_r)^2),
    m = 0 halved: prodct_mk_allk / l2norm_mk_allk summed over (m, k)."""
    nr = g.NR
    w = g.W[:nr] / ((1 - g.X[:nr]) ** 2 if inv_om2 else 1.0)
    f = np.ones(g.NTCHOPDIM)
    f[0] = 0.5
    out = np.zeros(g.shape(PFF))
    out[:nr] = 4.0 * np.pi * g.ZLEN * g.ELL2 * w[:, None, None] * f[None, :, None]
    return out


def _fluct(F):
    out = F.copy()
    out.E[:, 0, 0] = 0.0
    out.LN = 0.0
    return out


def energy_objective(g, psi, chi, b):
    """J = KE(psi - psi_bar, chi - chi_bar) + 1/2 int b^2 dV (see above)."""
    from .diagnostics import boussi_energy
    ke, pe, _ = boussi_energy(g, _fluct(psi), _fluct(chi), _field(b.E, FFF), 1.0)
    return float(ke.sum() + pe.sum())


def energy_objective_grad(g, psi, chi, b):
    """Gradient of energy_objective with respect to (psi, chi, b) (FFF, with
    LN): the quadratic forms' symmetric parts through RTRAN(+1)^T, DELSQH^T
    and DEL2^T at CHOPSET(3)."""
    from .legops import del2, delsqh
    from .transforms import rtran
    Wt = _pff_weights(g)
    Wb = _pff_weights(g, inv_om2=True)
    p, c = _fluct(psi), _fluct(chi)
    g.chopset(3)
    try:
        def R(F):
            X = _field(F.E, FFF)
            rtran(g, X, 1)
            return X

        # KE = 1/2 [ -<R p, R Dh p>_W + <R D2 c, R Dh c>_W ]  (LN parts are zero)
        Rp, RDp = R(p), R(delsqh(g, p))
        gp = _add(rtran_T(g, _field(-0.5 * Wt * RDp.E, PFF), 1),
                  delsqh_T(g, rtran_T(g, _field(-0.5 * Wt * Rp.E, PFF), 1)))
        RD2c, RDc = R(del2(g, c)), R(delsqh(g, c))
        gc = _add(del2_T(g, rtran_T(g, _field(0.5 * Wt * RDc.E, PFF), 1)),
                  delsqh_T(g, rtran_T(g, _field(0.5 * Wt * RD2c.E, PFF), 1)))
        # 1/2 int b^2 = 1/2 <R b, R b>_{W/(1-x)^2}
        Rb = R(_field(b.E, FFF))
        gb = rtran_T(g, _field(Wb * Rb.E, PFF), 1)
    finally:
        g.chopset(-3)
    for G in (gp, gc):
        G.E[:, 0, 0] = 0.0
        G.LN = 0.0
    gb.LN = 0.0
    return gp, gc, gb


def visc1_T(g, out_bar, nu, dt):
    """Adjoint of VISC1(A, NU, DT) (mod_march.f90:1529-1576) = IHELM(-alp A, alp),
    alp = 1/(NU DT)."""
    alp = 1 / (nu * dt)
    wk = ihelm_T(g, out_bar, alp)
    return _field(-alp * wk.E, FFF, -alp * wk.LN)


def _visc_be_T(g, ph, bars, dt):
    out = []
    for k, F in zip(("psi", "chi", "b"), bars):
        nu = ph.kappa if k == "b" else ph.nu
        if nu == 0.0:
            out.append(F.copy())
        else:
            out.append(visc1_T(g, F, nu, dt))
    out[2].LN = 0.0
    return out


def rich_fe_be_vjp(s0, bars):
    """Vector-Jacobian product of RICH_BOUSSI_FE_BE (mod_march.f90:535-606,
    the AB2-CN start-up, VISC%SW = 1) as the map (psi, chi, b) -> (psi, chi,
    b, n_psi, n_chi, n_b); s0 is an oracle Solver holding (psi, chi, b)."""
    from .boussinesq import calc_boussi_force, calc_boussi_visc_be
    g, ph, dt = s0.g, s0.ph, s0.ph.dt
    hdt = 0.5 * dt
    x0 = [s0.psi.copy(), s0.chi.copy(), s0.b.copy()]

    def axpy(xs, a, fs):
        out = []
        for x, f in zip(xs, fs):
            F = x.copy()
            F.E = x.E + a * f.E
            F.LN = x.LN + a * f.LN
            out.append(F)
        out[2].LN = x0[2].LN
        return out

    F0 = calc_boussi_force(g, ph, *[F.copy() for F in x0])
    x2 = list(calc_boussi_visc_be(g, ph, *axpy(x0, hdt, F0), hdt))
    out_bar = [_field(bars[k].E, FFF, bars[k].LN if k != "b" else 0.0) for k in ("psi", "chi", "b")]
    x2pp_bar = [_field(2.0 * F.E, FFF, 2.0 * F.LN) for F in out_bar]
    x1_bar = [_field(-F.E, FFF, -F.LN) for F in out_bar]
    y1 = _visc_be_T(g, ph, x1_bar, dt)
    x2p_bar = _visc_be_T(g, ph, x2pp_bar, hdt)
    f1_bar = [_field(hdt * F.E, FFF, hdt * F.LN) for F in x2p_bar]
    fx2 = boussi_force_vjp(g, ph, *x2, *f1_bar)
    x2_bar = [_add(a, b_) for a, b_ in zip(x2p_bar, fx2)]
    z = _visc_be_T(g, ph, x2_bar, hdt)
    f0_bar = []
    for q, k in enumerate(("n_psi", "n_chi", "n_b")):
        F = _field(dt * y1[q].E + hdt * z[q].E + bars[k].E, FFF,
                   dt * y1[q].LN + hdt * z[q].LN + (bars[k].LN if k != "n_b" else 0.0))
        f0_bar.append(F)
    fx0 = boussi_force_vjp(g, ph, *x0, *f0_bar)
    res = {}
    for q, k in enumerate(("psi", "chi", "b")):
        res[k] = _add(y1[q], z[q], fx0[q])
    res["b"].LN = 0.0
    return res


def idelsqh_T(g, A_bar):
    """Adjoint of IDELSQH(B, A) (mod_legops.f90:136-241): the far-field fix,
    A = -B ELL2/(n(n+1)) for n >= 1, and A%LN = Re B(1,1,1) NORM(1,1) ELL2."""
    y = farfield_T(g, A_bar)
    Bb = g.alloc(FFF)
    for mm in range(y.E.shape[1]):
        nn = int(g.NRCHOPS[mm])
        for i in range(nn):
            n = int(g.M[mm]) + i
            if n >= 1:
                Bb.E[i, mm, :] = -y.E[i, mm, :] * (g.ELL2 / (n * (n + 1)))
    Bb.E[0, 0, 0] += A_bar.LN * g.NORM0[0] * g.ELL2
    return Bb


def initial_state_T(g, psi_bar, chi_bar, b_bar):
    """Adjoint of the seeded initial state (oracle layout.initial_state) with
    respect to the perturbation coefficients (c_psi, c_chi, c_b)."""
    out = []
    for F in (psi_bar, chi_bar):
        q = _field(F.E, FFF, F.LN)
        g.chopdo(q)
        p = idelsqh_T(g, q)
        g.chopdo(p)
        out.append(-p.E)
    # The state is zero outside the chop, so its cotangent there is dropped
    # before the far-field transpose, which would mix it into kept entries.
    bq = _field(b_bar.E, FFF)
    g.chopdo(bq)
    bb = farfield_T(g, bq)
    g.chopdo(bb)
    out.append(bb.E)
    return out


def etdfe_be_vjp(s, PSI, CHI, B, E, NL, dt, store, bars):
    """Vector-Jacobian product of STEP_BOUSSI_ETDFE_BE (mod_march.f90:664-753,
    oracle Solver._etdfe_be, no sponge) from (PSI, CHI, B) to (PSI', CHI', B')
    and, with store, the seven history fields (r_pi_* = (V - PC2VEL(PSI',
    CHI'))/2).  E, NL: the ETD matrices for dt; s supplies the filters."""
    from .boussinesq import calc_boussi_etdfe_sub, calc_boussi_nonlin, _etd_mats
    from .legops import idel2ln, pc2vel, pc2vor, project
    g, ph = s.g, s.ph
    tf = dt / ph.dt
    hyp = s.hyp

    def filt(F, which):
        out = _field(F.E, FFF, F.LN)
        if hyp is not None:
            hyp._apply(g, out, hyp.hv if which == "v" else hyp.hd, tf)
        return out

    g.chopset(3)
    V = pc2vel(g, PSI, CHI)
    Om = pc2vor(g, PSI, CHI)
    g.chopset(-3)
    BN, NR_, NP_, NZ_ = calc_boussi_nonlin(g, B.copy(), *[F.copy() for F in V], *[F.copy() for F in Om])
    Nf = [filt(F, "v") for F in (NR_, NP_, NZ_)] + [filt(BN, "d")]
    Vw = [F.copy() for F in V]
    Bw = B.copy()
    calc_boussi_etdfe_sub(E, NL, Bw, *Vw, Nf[3], Nf[0], Nf[1], Nf[2], dt)
    Vf = [filt(F, "v") for F in Vw]
    # reverse
    psi1_bar = _field(bars["psi"].E, FFF, bars["psi"].LN)
    chi1_bar = _field(bars["chi"].E, FFF, bars["chi"].LN)
    vf_bar = [_field(np.zeros_like(B.E), FFF) for _ in range(3)]
    if store:
        g.chopset(3)
        p_h, c_h = pc2vel_T(g, *[_field(-0.5 * bars[k].E, FFF) for k in ("r_pi_r", "r_pi_p", "pi_z")])
        g.chopset(-3)
        psi1_bar = _add(psi1_bar, p_h)
        chi1_bar = _add(chi1_bar, c_h)
        vf_bar = [_field(0.5 * bars[k].E, FFF) for k in ("r_pi_r", "r_pi_p", "pi_z")]
    w_bar = idel2ln_T(g, chi1_bar)
    pb = project_T(g, psi1_bar, w_bar)
    c, _ = _vel2pln_vectors(g)
    pb[1] = vel2pln_T(g, pb[1])
    pb[1].E[:g.NR, 0, 0] += c * psi1_bar.LN
    vf_bar = [_add(vf_bar[q], rtran_T(g, pb[q], 1)) for q in range(3)]
    for F in vf_bar:
        F.LN = 0.0
    vw_bar = [filt(F, "v") for F in vf_bar]
    bw_bar = filt(_field(bars["b"].E, FFF), "d")
    K = B.E.shape[2]
    ev_bar = [np.zeros_like(B.E) for _ in range(4)]
    av_bar = [np.zeros_like(B.E) for _ in range(4)]
    cvb = [vw_bar[0].E, vw_bar[1].E, vw_bar[2].E, bw_bar.E]
    for kk in range(K):
        Er, Nr = _etd_mats(E, NL, dt, kk == 0)
        cv = np.stack([x[:, :, kk] for x in cvb])
        e_ = np.einsum("ji,j...->i...", Er, cv)
        a_ = np.einsum("ji,j...->i...", Nr, cv)
        for q in range(4):
            ev_bar[q][:, :, kk] = e_[q]
            av_bar[q][:, :, kk] = a_[q]
    nf_bar = [_field(av_bar[q], FFF) for q in range(4)]
    if store:
        for q, k in enumerate(("r_n_r", "r_n_p", "n_z", "n_b")):
            nf_bar[q].E = nf_bar[q].E + bars[k].E
    n_bar = [filt(nf_bar[q], "v") for q in range(3)] + [filt(nf_bar[3], "d")]
    nl = boussi_nonlin_vjp(g, B, *V, *Om, n_bar[3], n_bar[0], n_bar[1], n_bar[2])
    b_bar = _add(_field(ev_bar[3], FFF), nl[0])
    g.chopset(3)
    p1, c1 = pc2vel_T(g, *[_add(_field(ev_bar[q], FFF), nl[1 + q]) for q in range(3)])
    p2, c2 = pc2vor_T(g, *nl[4:7])
    g.chopset(-3)
    return _add(p1, p2), _add(c1, c2), b_bar


def rich_etdfe_be_vjp(s0, bars):
    """Vector-Jacobian product of RICH_BOUSSI_ETDFE_BE (mod_march.f90:756-808,
    the ETD2AB-CN start-up, VISC%SW = 3 so the BE viscous steps are identities)
    as the map (psi, chi, b) -> (psi, chi, b and the seven history fields)."""
    from .boussinesq import calc_boussi_etd_op
    g, ph, dt = s0.g, s0.ph, s0.ph.dt
    if ph.visc_sw == 1:
        raise ValueError("rich_etdfe_be_vjp: VISC%SW = 1 not handled")
    hdt = 0.5 * dt
    he, hnl = calc_boussi_etd_op(ph.bv0, ph.omega, hdt)
    x0 = [s0.psi.copy(), s0.chi.copy(), s0.b.copy()]
    y0 = [g.copy0(F) for F in x0]
    y2 = list(s0._etdfe_be(*[F.copy() for F in y0], he, hnl, hdt, False))
    out_bar = {k: bars[k] for k in ("psi", "chi", "b")}
    z_bars = {k: _field(-bars[k].E, FFF, -bars[k].LN if k != "b" else 0.0) for k in ("psi", "chi", "b")}
    for k in HISTORY:
        z_bars[k] = bars[k]
    fe, fnl = calc_boussi_etd_op(ph.bv0, ph.omega, dt)
    zp, zc, zb = etdfe_be_vjp(s0, *x0, fe, fnl, dt, True, z_bars)
    y3_bar = {k: _field(2.0 * out_bar[k].E, FFF, 2.0 * out_bar[k].LN if k != "b" else 0.0)
              for k in ("psi", "chi", "b")}
    a = etdfe_be_vjp(s0, *y2, he, hnl, hdt, False, y3_bar)
    y1_bar = dict(zip(("psi", "chi", "b"), a))
    y0_bar = etdfe_be_vjp(s0, *y0, he, hnl, hdt, False, y1_bar)
    res = {}
    for q, (k, zq) in enumerate(zip(("psi", "chi", "b"), (zp, zc, zb))):
        y = _field(y0_bar[q].E, FFF, y0_bar[q].LN)
        g.chopdo(y)
        res[k] = _add(zq, y)
    res["b"].LN = 0.0
    return res
