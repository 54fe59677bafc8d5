"""Boussinesq right-hand sides, implicit/ETD updates and time steppers (oracle).

Restates:
  mod_boussinesq.f90:42-109   CALC_BOUSSI_DIAG
  mod_boussinesq.f90:235-314  CALC_BOUSSI_NONLIN
  mod_boussinesq.f90:317-410  CALC_BOUSSI_FORCE
  mod_march.f90:535-606       RICH_BOUSSI_FE_BE
  mod_march.f90:609-661       STEP_BOUSSI_AB_CN
  mod_march.f90:664-753       STEP_BOUSSI_ETDFE_BE
  mod_march.f90:756-808       RICH_BOUSSI_ETDFE_BE
  mod_march.f90:811-901       STEP_BOUSSI_ETDAB_CN
  mod_march.f90:906-945       CALC_BOUSSI_ETD_OP
  mod_march.f90:948-1047      CALC_BOUSSI_ETDFE_SUB
  mod_march.f90:1050-1139     CALC_BOUSSI_ETDAB_SUB
  mod_march.f90:1200-1265     CALC_BOUSSI_VISC_BE / _CN
  mod_march.f90:1305-1349     CALC_BOUSSI_HYPERV
  mod_march.f90:1352-1416     CALC_BOUSSI_ETD_HYPERV
  mod_march.f90:1529-1636     VISC1 / VISC2
  mod_march.f90:3320-3486     HYP3SET / HYP3MASK / HYP3INIT
  mod_march.f90:3521-3560     HYPERV3
Freestream/strain (NADD) and the sponge (RMV%SW = 2) are zero/off in every
configured run and are not restated; the per-step host diagnostics
(DIAGNOST, CALC_BOUSSI_ENERGY, INSPECT, MSAVE) do not modify the state.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import math
from dataclasses import dataclass

import numpy as np

from .grid import FFF, PPP
from .legops import (del2, grad, idel2, idel2ln, ihelm, pc2vel, pc2vor, project,
                     vdotpsub, vprodsub)
from .transforms import rtran, toff, tofp, verfft


@dataclass
class Physics:
    """BSNSQ / VISC / TIM parameters (mod_boussinesq.f90:16-26, mod_march.f90:48-87)."""
    dt: float
    omega: float = 1.0
    bv0: float = 1.0
    kappa: float = 0.0
    kappap: float = 0.0
    adams: bool = True
    visc_sw: int = 1
    nu: float = 0.0
    nup: float = 0.0
    p: int = 2
    rmv_sw: int = 0


# ----------------------------------------------------------------------
def calc_boussi_force(g, ph, PSI, CHI, B):
    """CALC_BOUSSI_FORCE(PSI, CHI, B, PSIN, CHIN, BN), mod_boussinesq.f90:317-410."""
    g.chopset(3)
    RBR, RBP, BZ = grad(g, B)
    RUR, RUP, UZ = pc2vel(g, PSI, CHI)
    ROR, ROP, OZ = pc2vor(g, PSI, CHI)
    for F in (RUR, RUP, UZ, ROR, ROP, OZ, RBR, RBP, BZ):
        tofp(g, F)
    vprodsub(g, RUR, RUP, UZ, ROR, ROP, OZ)
    BN = g.alloc(PPP)
    BN.E = -vdotpsub(g, RUR, RUP, UZ, RBR, RBP, BZ)
    g.chopset(-3)
    W = g.copy0(B)
    tofp(g, W)
    ROR.E = ROR.E + 2 * ph.omega * RUP.E
    ROP.E = ROP.E - 2 * ph.omega * RUR.E
    OZ.E = OZ.E - W.E
    BN.E = BN.E + ph.bv0 ** 2 * UZ.E
    PSIN, Wf = project(g, ROR, ROP, OZ, 0.0)
    CHIN = idel2ln(g, Wf)
    toff(g, BN)
    return PSIN, CHIN, BN


def calc_boussi_nonlin(g, B, RUR, RUP, UZ, ROR, ROP, OZ):
    """CALC_BOUSSI_NONLIN, mod_boussinesq.f90:235-314.

    Returns (BN, NR, NP, NZ): -(u.grad)b and the projected u x omega as a
    velocity-form FFF field (PC2VEL of its poloidal-toroidal potentials).
    """
    g.chopset(1)
    RBR, RBP, BZ = grad(g, B)
    g.chopset(-1)
    for F in (RUR, RUP, UZ, ROR, ROP, OZ, RBR, RBP, BZ):
        tofp(g, F)
    vprodsub(g, RUR, RUP, UZ, ROR, ROP, OZ)
    BN = g.alloc(PPP)
    BN.E = -vdotpsub(g, RUR, RUP, UZ, RBR, RBP, BZ)
    PSI, W = project(g, ROR, ROP, OZ, 0.0)
    CHI = idel2(g, W)
    g.chopset(3)
    NR_, NP_, NZ_ = pc2vel(g, PSI, CHI)
    g.chopset(-3)
    toff(g, BN)
    return BN, NR_, NP_, NZ_


# ----------------------------------------------------------------------
def visc1(g, A, nu, dt):
    """VISC1(A, NU, DT, WK), mod_march.f90:1529-1576 (backward Euler)."""
    if nu == 0.0:
        raise ValueError("VISC1: NU CAN'T BE ZERO")
    alp = 1 / (nu * dt)
    WK = g.alloc(FFF)
    WK.LN = -alp * A.LN
    WK.E = -alp * A.E
    return ihelm(g, WK, alp)


def visc2(g, A, AO, nu, dt):
    """VISC2(A, AO, NU, DT, WK), mod_march.f90:1579-1636 (Crank-Nicolson)."""
    if nu == 0.0:
        raise ValueError("VISC2: NU CAN'T BE ZERO")
    alp = 2 / nu / dt
    g.chopset(2)
    WK = del2(g, AO)
    g.chopset(-2)
    g.chopdo(WK)
    WK.E = -WK.E - alp * A.E
    WK.LN = -alp * A.LN
    return ihelm(g, WK, alp)


def calc_boussi_visc_be(g, ph, PSI, CHI, B, dt):
    """CALC_BOUSSI_VISC_BE, mod_march.f90:1200-1230."""
    if ph.visc_sw != 1:
        return PSI, CHI, B
    PSI = visc1(g, PSI, ph.nu, dt)
    CHI = visc1(g, CHI, ph.nu, dt)
    if ph.kappa != 0.0:
        B = visc1(g, B, ph.kappa, dt)
    return PSI, CHI, B


def calc_boussi_visc_cn(g, ph, PSI, CHI, B, PSIO, CHIO, BO):
    """CALC_BOUSSI_VISC_CN, mod_march.f90:1233-1265."""
    if ph.visc_sw != 1:
        return PSI, CHI, B
    PSI = visc2(g, PSI, PSIO, ph.nu, ph.dt)
    CHI = visc2(g, CHI, CHIO, ph.nu, ph.dt)
    if ph.kappa != 0.0:
        B = visc2(g, B, BO, ph.kappa, ph.dt)
    return PSI, CHI, B


# ----------------------------------------------------------------------
def hyp3mask(kvals, size, ratio=2.0 / 3.0, steep=3.0):
    """HYP3MASK(K_VALS, K_MASK, RATIO, STEEPNESS), mod_march.f90:3410-3461."""
    out = np.ones(size)
    kvals = np.asarray(kvals, dtype=np.float64)
    kmax = kvals.max() if kvals.size else -np.inf
    if kmax < 1e-12:
        kmax = 1.0
    ta = math.tanh(steep)
    for i, kv in enumerate(kvals):
        kn = kv / kmax
        if kn < ratio:
            out[i] = 0.0
        else:
            xr = (kn - ratio) / (1.0 - ratio)
            yr = steep * (2.0 * xr - 1.0)
            out[i] = (math.tanh(yr) + ta) / (2.0 * ta)
    return out


class Hyperv3:
    """HYP3SET / HYP3INIT (mod_march.f90:3320-3486): exponential spectral filters."""

    def __init__(self, g, ph):
        nrchop = g.NRCHOP
        self.mask_r = np.ones((nrchop, g.NTCHOPDIM))
        for mm in range(g.NTCHOPDIM):
            self.mask_r[:, mm] = hyp3mask(np.arange(int(g.NRCHOPS[mm]), dtype=float), nrchop,
                                          ratio=0.5, steep=2.0)
        self.mask_t = hyp3mask(g.M.astype(float), g.NTCHOPDIM, steep=2.0)
        self.mask_x = hyp3mask(np.abs(g.AK[0, :]), g.NXCHOPDIM, steep=2.0)
        # HYP3INIT (3464-3480): NUP_R/T/X = NUP, KAPPAP_R/T/X = KAPPAP
        self.nup = [ph.nup] * 3
        self.kappap = [ph.kappap] * 3
        self.hv = self._set(g, ph, *self.nup)
        self.hd = self._set(g, ph, *self.kappap)

    def _set(self, g, ph, nu_r, nu_t=None, nu_x=None):
        """HYP3SET(NU_R, NU_T, NU_X, ...), mod_march.f90:3320-3368 (without hyperv.dat)."""
        nu_t = nu_r if nu_t is None else nu_t
        nu_x = nu_r if nu_x is None else nu_x
        nrchop = g.NRCHOP
        ph2 = ph.p // 2
        k2r = 1.5 ** 2 * float((nrchop - 1) * nrchop) / g.ELL2
        k2t = float(np.max(g.M ** 2))
        k2x = float(np.max(g.AK[0, :] ** 2))
        ht = np.exp(-nu_t * self.mask_t * (g.M.astype(float) ** 2 / k2t) ** ph2)
        nn = np.arange(1, nrchop + 1)
        hr = np.exp(-nu_r * self.mask_r * ((1.5 ** 2 * ((nn - 1) * nn).astype(float) / g.ELL2 / k2r) ** ph2)[:, None])
        hx = np.exp(-nu_x * self.mask_x * (g.AK[0, :] ** 2 / k2x) ** ph2)
        return hr, ht, hx

    def reset(self, g, ph):
        """The two HYP3SET calls after HYP3ADJ in the stepper (mod_march.f90:286-287)."""
        self.hv = self._set(g, ph, *self.nup)
        self.hd = self._set(g, ph, *self.kappap)

    @staticmethod
    def _apply(g, A, filt, tf):
        hr, ht, hx = filt
        for mm in range(A.E.shape[1]):
            nn = int(g.NRCHOPS[mm])
            fac = (hr[:nn, mm][:, None] * ht[mm] * hx[None, :]) ** tf
            A.E[:nn, mm, :] = A.E[:nn, mm, :] * fac
        g.chopdo(A)

    def hyperv3(self, g, PSI, CHI, B, tf):
        """HYPERV3(PSI, CHI, B, DT_SCALE), mod_march.f90:3521-3560."""
        self._apply(g, PSI, self.hv, tf)
        self._apply(g, CHI, self.hv, tf)
        self._apply(g, B, self.hd, tf)

    def etd_hyperv(self, g, RUR, RUP, UZ, B, tf):
        """CALC_BOUSSI_ETD_HYPERV (SW = 3), mod_march.f90:1352-1416."""
        self._apply(g, RUR, self.hv, tf)
        self._apply(g, RUP, self.hv, tf)
        self._apply(g, UZ, self.hv, tf)
        self._apply(g, B, self.hd, tf)


def calc_boussi_diag(bv0, omega):
    """CALC_BOUSSI_DIAG(J, S, S_INV), mod_boussinesq.f90:42-109."""
    if bv0 == 0.0:
        raise ValueError("CALC_BOUSSI_DIAG: N_FREQ = 0, CANNOT DIAGONALIZE")
    iu = 1j
    J = np.zeros((4, 4), dtype=complex)
    J[0, 0] = -iu * bv0
    J[1, 1] = iu * bv0
    J[2, 2] = -2.0 * iu * omega
    J[3, 3] = 2.0 * iu * omega
    S = np.zeros((4, 4), dtype=complex)
    S[0, 2] = iu
    S[0, 3] = -iu
    S[1, 2] = 1.0
    S[1, 3] = 1.0
    S[2, 0] = -iu / bv0
    S[2, 1] = iu / bv0
    S[3, 0] = 1.0
    S[3, 1] = 1.0
    Si = np.zeros((4, 4), dtype=complex)
    Si[0, 2] = iu * bv0 / 2.0
    Si[0, 3] = 0.5
    Si[1, 2] = -iu * bv0 / 2.0
    Si[1, 3] = 0.5
    Si[2, 0] = -iu / 2.0
    Si[2, 1] = 0.5
    Si[3, 0] = iu / 2.0
    Si[3, 1] = 0.5
    return J, S, Si


def calc_boussi_etd_op(bv0, omega, dt):
    """CALC_BOUSSI_ETD_OP(ETD_E, ETD_NL, DT), mod_march.f90:906-945."""
    J, S, Si = calc_boussi_diag(bv0, omega)
    je = np.zeros((4, 4), dtype=complex)
    jp = np.zeros((4, 4), dtype=complex)
    for i in range(4):
        je[i, i] = np.exp(J[i, i] * dt)
        if abs(J[i, i]) > 1e-14:
            jp[i, i] = (je[i, i] - 1.0) / J[i, i]
        else:
            jp[i, i] = dt
    return S @ je @ Si, S @ jp @ Si


def _etd_mats(E, NL, dt, k0):
    Er = E.real.copy()
    Nr = NL.real.copy()
    if k0:
        Er[0, :] = 0
        Er[0, 0] = 1
        Er[1, :] = 0
        Er[1, 1] = 1
        Nr[0, :] = 0
        Nr[0, 0] = dt
        Nr[1, :] = 0
        Nr[1, 1] = dt
    return Er, Nr


def calc_boussi_etdfe_sub(E, NL, B, RUR, RUP, UZ, NB, RNR, RNP, NZ, dt):
    """CALC_BOUSSI_ETDFE_SUB, mod_march.f90:948-1047 (in place)."""
    K = B.E.shape[2]
    for kk in range(K):
        Er, Nr = _etd_mats(E, NL, dt, kk == 0)
        ev = np.stack([RUR.E[:, :, kk], RUP.E[:, :, kk], UZ.E[:, :, kk], B.E[:, :, kk]])
        av = np.stack([RNR.E[:, :, kk], RNP.E[:, :, kk], NZ.E[:, :, kk], NB.E[:, :, kk]])
        cv = np.einsum("ij,j...->i...", Er, ev) + np.einsum("ij,j...->i...", Nr, av)
        RUR.E[:, :, kk], RUP.E[:, :, kk], UZ.E[:, :, kk], B.E[:, :, kk] = cv


def calc_boussi_etdab_sub(st, B, RUR, RUP, UZ, NB, RNR, RNP, NZ, dt):
    """CALC_BOUSSI_ETDAB_SUB, mod_march.f90:1050-1139 (in place)."""
    K = B.E.shape[2]
    notm0 = np.ones(B.E.shape[1])
    notm0[0] = 0.0
    for kk in range(K):
        Er, Nr = _etd_mats(st.etd_e, st.etd_nl, dt, kk == 0)
        notk0 = 0.0 if kk == 0 else 1.0
        ev = np.stack([RUR.E[:, :, kk] - st.r_pi_r.E[:, :, kk],
                       RUP.E[:, :, kk] - st.r_pi_p.E[:, :, kk] * notm0[None, :],
                       UZ.E[:, :, kk] - st.pi_z.E[:, :, kk] * notk0,
                       B.E[:, :, kk]])
        av = np.stack([1.5 * RNR.E[:, :, kk] - 0.5 * st.r_n_r.E[:, :, kk],
                       1.5 * RNP.E[:, :, kk] - 0.5 * st.r_n_p.E[:, :, kk],
                       1.5 * NZ.E[:, :, kk] - 0.5 * st.n_z.E[:, :, kk],
                       1.5 * NB.E[:, :, kk] - 0.5 * st.n_b.E[:, :, kk]])
        cv = np.einsum("ij,j...->i...", Er, ev) + np.einsum("ij,j...->i...", Nr, av)
        RUR.E[:, :, kk], RUP.E[:, :, kk], UZ.E[:, :, kk], B.E[:, :, kk] = cv


# ----------------------------------------------------------------------
class Solver:
    """SOLVER_T (mod_march.f90:17-39) with INITIALIZE / TIME_STEPPING bodies.

    state: (psi, chi, b) FFF Fields, advanced in place by ``step``.
    """

    def __init__(self, g, ph, psi, chi, b):
        self.g, self.ph = g, ph
        self.psi, self.chi, self.b = psi, chi, b
        self.t = 0.0
        self.n = 0
        self.hyp = Hyperv3(g, ph) if ph.visc_sw == 3 else None

    # -- shared helpers ------------------------------------------------
    def _hyperv(self, PSI, CHI, B, dt):
        """CALC_BOUSSI_HYPERV, mod_march.f90:1305-1349 (SW 0/1 are no-ops)."""
        if self.ph.visc_sw == 3:
            self.hyp.hyperv3(self.g, PSI, CHI, B, dt / self.ph.dt)
        elif self.ph.visc_sw == 2:
            # HYPERV per field, B only when KAPPAP /= 0 (1327-1335); in place
            from .legops import hyperv
            ph, g = self.ph, self.g
            fields = [(PSI, ph.nu, ph.nup), (CHI, ph.nu, ph.nup)]
            if ph.kappap != 0.0:
                fields.append((B, ph.kappa, ph.kappap))
            for F, nu, nup in fields:
                R = hyperv(g, F, nu, nup, ph.p, dt)
                F.E, F.LN = R.E, R.LN

    def _etd_hyperv(self, RUR, RUP, UZ, B, dt):
        if self.ph.visc_sw == 3:
            self.hyp.etd_hyperv(self.g, RUR, RUP, UZ, B, dt / self.ph.dt)

    def initialize(self):
        """SOLVER_T%INITIALIZE, mod_march.f90:171-240 (Richardson start-up)."""
        if self.ph.adams:
            self._rich_fe_be()
        else:
            self.etd_e, self.etd_nl = calc_boussi_etd_op(self.ph.bv0, self.ph.omega, self.ph.dt)
            self._rich_etdfe_be()

    def step(self):
        """SOLVER_T%TIME_STEPPING state update, mod_march.f90:243-307."""
        if self.ph.adams:
            self._step_ab_cn()
        else:
            self._step_etdab_cn()

    # -- AB2-CN -------------------------------------------------------
    def _rich_fe_be(self):
        """RICH_BOUSSI_FE_BE, mod_march.f90:535-606."""
        g, ph = self.g, self.ph
        dt = ph.dt
        hdt = dt * 0.5
        self.t += dt
        self.n += 1
        PSI, CHI, B = self.psi, self.chi, self.b
        self.n_psi, self.n_chi, self.n_b = calc_boussi_force(g, ph, PSI, CHI, B)
        PSI2 = g.alloc(FFF)
        CHI2 = g.alloc(FFF)
        B2 = g.alloc(FFF)
        PSI2.E = PSI.E + hdt * self.n_psi.E
        PSI2.LN = PSI.LN + hdt * self.n_psi.LN
        CHI2.E = CHI.E + hdt * self.n_chi.E
        CHI2.LN = CHI.LN + hdt * self.n_chi.LN
        B2.E = B.E + hdt * self.n_b.E
        PSI2, CHI2, B2 = calc_boussi_visc_be(g, ph, PSI2, CHI2, B2, hdt)
        self._hyperv(PSI2, CHI2, B2, hdt)
        P_N, C_N, B_N = calc_boussi_force(g, ph, PSI2, CHI2, B2)
        PSI2.E = PSI2.E + hdt * P_N.E
        PSI2.LN = PSI2.LN + hdt * P_N.LN
        CHI2.E = CHI2.E + hdt * C_N.E
        CHI2.LN = CHI2.LN + hdt * C_N.LN
        B2.E = B2.E + hdt * B_N.E
        PSI2, CHI2, B2 = calc_boussi_visc_be(g, ph, PSI2, CHI2, B2, hdt)
        self._hyperv(PSI2, CHI2, B2, hdt)
        PSI.E = PSI.E + dt * self.n_psi.E
        PSI.LN = PSI.LN + dt * self.n_psi.LN
        CHI.E = CHI.E + dt * self.n_chi.E
        CHI.LN = CHI.LN + dt * self.n_chi.LN
        B.E = B.E + dt * self.n_b.E
        PSI, CHI, B = calc_boussi_visc_be(g, ph, PSI, CHI, B, dt)
        self._hyperv(PSI, CHI, B, dt)
        PSI.E = 2.0 * PSI2.E - PSI.E
        PSI.LN = 2.0 * PSI2.LN - PSI.LN
        CHI.E = 2.0 * CHI2.E - CHI.E
        CHI.LN = 2.0 * CHI2.LN - CHI.LN
        B.E = 2.0 * B2.E - B.E
        self.psi, self.chi, self.b = PSI, CHI, B

    def _step_ab_cn(self):
        """STEP_BOUSSI_AB_CN, mod_march.f90:609-661."""
        g, ph = self.g, self.ph
        dt = ph.dt
        self.t += dt
        self.n += 1
        PSI, CHI, B = self.psi, self.chi, self.b
        PSIN, CHIN, BN = calc_boussi_force(g, ph, PSI, CHI, B)
        PSI0, CHI0, B0 = g.copy0(PSI), g.copy0(CHI), g.copy0(B)
        PSI.E = PSI.E + dt * (1.5 * PSIN.E - 0.5 * self.n_psi.E)
        PSI.LN = PSI.LN + dt * (1.5 * PSIN.LN - 0.5 * self.n_psi.LN)
        CHI.E = CHI.E + dt * (1.5 * CHIN.E - 0.5 * self.n_chi.E)
        CHI.LN = CHI.LN + dt * (1.5 * CHIN.LN - 0.5 * self.n_chi.LN)
        B.E = B.E + dt * (1.5 * BN.E - 0.5 * self.n_b.E)
        self.n_psi, self.n_chi, self.n_b = g.copy0(PSIN), g.copy0(CHIN), g.copy0(BN)
        PSI, CHI, B = calc_boussi_visc_cn(g, ph, PSI, CHI, B, PSI0, CHI0, B0)
        self._hyperv(PSI, CHI, B, dt)
        self.psi, self.chi, self.b = PSI, CHI, B

    # -- ETD2AB-CN ----------------------------------------------------
    def _etd_sponge(self, UZ, B, dt):
        """CALC_BOUSSI_ETD_SPONGE(UZ, B, DT), mod_march.f90:1436-1469, with the
        SPNGINIT profile (2292-2323): N_TAU = 10, RATIO_L = 0.86, RATIO_S = 0.04;
        each z-plane of UZ and B in PFP is scaled by exp(-(1 - T(z))/TAU DT),
        T = TOPHAT(Z - ZLEN/2, ZLEN RATIO_L/2, ZLEN RATIO_S) (3704-3712); the
        m = 0 modes are made real; both go back to FFF."""
        if self.ph.rmv_sw != 2:
            return
        g = self.g
        z = g.Z[:g.NX] - g.ZLEN / 2.0
        hw, st = g.ZLEN * 0.86 / 2.0, g.ZLEN * 0.04
        tophat = 0.5 * (np.tanh((z + hw) / st) - np.tanh((z - hw) / st))
        tau = 10 * self.ph.dt
        damp = np.exp(-(1.0 - tophat) / tau * dt)
        for F in (UZ, B):
            rtran(g, F, 1)
            verfft(g, F, 1)
            F.E[:, :, :g.NX] *= damp[None, None, :]
            F.E[:, 0, :] = F.E[:, 0, :].real
            toff(g, F)

    def _etdfe_be(self, PSI, CHI, B, E, NL, dt, store):
        """STEP_BOUSSI_ETDFE_BE, mod_march.f90:664-753 (returns new PSI, CHI)."""
        g = self.g
        g.chopset(3)
        RURN, RUPN, UZN = pc2vel(g, PSI, CHI)
        RORN, ROPN, OZN = pc2vor(g, PSI, CHI)
        g.chopset(-3)
        BN, RORN, ROPN, OZN = calc_boussi_nonlin(g, B, RURN, RUPN, UZN, RORN, ROPN, OZN)
        self._etd_hyperv(RORN, ROPN, OZN, BN, dt)
        g.chopset(3)
        RURN, RUPN, UZN = pc2vel(g, PSI, CHI)
        g.chopset(-3)
        calc_boussi_etdfe_sub(E, NL, B, RURN, RUPN, UZN, BN, RORN, ROPN, OZN, dt)
        self._etd_sponge(UZN, B, dt)
        self._etd_hyperv(RURN, RUPN, UZN, B, dt)
        if store:
            self.n_b = BN.copy()
            self.r_n_r, self.r_n_p, self.n_z = RORN.copy(), ROPN.copy(), OZN.copy()
            self.r_pi_r, self.r_pi_p, self.pi_z = RURN.copy(), RUPN.copy(), UZN.copy()
        PSI_new, W = project(g, RURN, RUPN, UZN, "psi")
        CHI_new = idel2ln(g, W)
        if store:
            g.chopset(3)
            r1, r2, r3 = pc2vel(g, PSI_new, CHI_new)
            g.chopset(-3)
            self.r_pi_r.E = 0.5 * (self.r_pi_r.E - r1.E)
            self.r_pi_p.E = 0.5 * (self.r_pi_p.E - r2.E)
            self.pi_z.E = 0.5 * (self.pi_z.E - r3.E)
        return PSI_new, CHI_new, B

    def _rich_etdfe_be(self):
        """RICH_BOUSSI_ETDFE_BE, mod_march.f90:756-808."""
        g, ph = self.g, self.ph
        dt = ph.dt
        hdt = dt * 0.5
        he, hnl = calc_boussi_etd_op(ph.bv0, ph.omega, hdt)
        self.t += dt
        self.n += 1
        PSI2, CHI2, B2 = g.copy0(self.psi), g.copy0(self.chi), g.copy0(self.b)
        PSI2, CHI2, B2 = self._etdfe_be(PSI2, CHI2, B2, he, hnl, hdt, False)
        PSI2, CHI2, B2 = calc_boussi_visc_be(g, ph, PSI2, CHI2, B2, hdt)
        PSI2, CHI2, B2 = self._etdfe_be(PSI2, CHI2, B2, he, hnl, hdt, False)
        PSI2, CHI2, B2 = calc_boussi_visc_be(g, ph, PSI2, CHI2, B2, hdt)
        PSI, CHI, B = self._etdfe_be(self.psi, self.chi, self.b, self.etd_e, self.etd_nl, dt, True)
        PSI, CHI, B = calc_boussi_visc_be(g, ph, PSI, CHI, B, dt)
        PSI.E = 2.0 * PSI2.E - PSI.E
        PSI.LN = 2.0 * PSI2.LN - PSI.LN
        CHI.E = 2.0 * CHI2.E - CHI.E
        CHI.LN = 2.0 * CHI2.LN - CHI.LN
        B.E = 2.0 * B2.E - B.E
        self.psi, self.chi, self.b = PSI, CHI, B

    def _step_etdab_cn(self):
        """STEP_BOUSSI_ETDAB_CN, mod_march.f90:811-901."""
        g, ph = self.g, self.ph
        dt = ph.dt
        self.t += dt
        self.n += 1
        PSI, CHI, B = self.psi, self.chi, self.b
        g.chopset(3)
        RURN, RUPN, UZN = pc2vel(g, PSI, CHI)
        RORN, ROPN, OZN = pc2vor(g, PSI, CHI)
        g.chopset(-3)
        BN, RORN, ROPN, OZN = calc_boussi_nonlin(g, B, RURN, RUPN, UZN, RORN, ROPN, OZN)
        self._etd_hyperv(RORN, ROPN, OZN, BN, dt)
        B0 = g.copy0(B)
        g.chopset(3)
        RURN, RUPN, UZN = pc2vel(g, PSI, CHI)
        g.chopset(-3)
        calc_boussi_etdab_sub(self, B, RURN, RUPN, UZN, BN, RORN, ROPN, OZN, dt)
        self.n_b = BN.copy()
        self.r_n_r, self.r_n_p, self.n_z = RORN.copy(), ROPN.copy(), OZN.copy()
        self._etd_sponge(UZN, B, dt)
        self._etd_hyperv(RURN, RUPN, UZN, B, dt)
        self.r_pi_r, self.r_pi_p, self.pi_z = RURN.copy(), RUPN.copy(), UZN.copy()
        PSI0, CHI0 = g.copy0(PSI), g.copy0(CHI)
        PSI, W = project(g, RURN, RUPN, UZN, "psi")
        CHI = idel2ln(g, W)
        g.chopset(3)
        r1, r2, r3 = pc2vel(g, PSI, CHI)
        g.chopset(-3)
        self.r_pi_r.E = self.r_pi_r.E - r1.E
        self.r_pi_p.E = self.r_pi_p.E - r2.E
        self.pi_z.E = self.pi_z.E - r3.E
        PSI, CHI, B = calc_boussi_visc_cn(g, ph, PSI, CHI, B, PSI0, CHI0, B0)
        self.psi, self.chi, self.b = PSI, CHI, B
