"""Adaptive hyperviscosity (oracle).

Restates mod_march.f90:
  2585-2617  ENEMON(PSI, CHI, EM, EK)       kinetic-energy spectra E(m), E(k)
  2619-2698  SPECURV(ESPEC, USE_RATIO)      Legendre P2 curvature of log10 E
  2700-2774  SPESLOP(ESPEC, RATIO)          Legendre P1 slope of log10 E over log10 k
  2776-2812  PDAJUST(COEFF, ...)            proportional-derivative coefficient update
  3000-3182  HYP3ADJ(PSI, CHI, B)           the dual curvature / slope controller
with mod_scalar3.f90:556-599 (PRODCT_M, PRODCT_K) and mod_boussinesq.f90:112-136
(CALC_BOUSSI_PE), for one process, without the printing.  Indices in the
spectrum helpers stay 1-based as in the reference (IS, IE, K_START).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import math

import numpy as np

from .diagnostics import boussi_pe, halfk, prodct_mk_allk
from .legops import del2, delsqh
from .transforms import rtran

CURV_PARAMS = (2.0, 1.0, 0.05, 0.8)      # [KP, KD, OFFSET, SCALE], 3019
SLOPE_PARAMS = (1.5, 0.5, 1.5, 1.0)      # 3023
BASELINE_NUP = 0.8                       # 3013


def enemon(g, PSI, CHI, with_k=True):
    """ENEMON at the current chop: EM(NTCHOP), EK(NXCHOP) (sums of PRODCT_MK_HALFK)."""
    W1 = g.copy0(PSI)
    W1.LN = 2.0 * PSI.LN
    W2 = delsqh(g, W1)
    rtran(g, W2, 1)
    W1 = g.copy0(PSI)
    W1.LN = 0.0
    rtran(g, W1, 1)
    tor = halfk(g, prodct_mk_allk(g, W2, W1))
    W1 = del2(g, CHI)
    rtran(g, W1, 1)
    W2 = delsqh(g, CHI)
    rtran(g, W2, 1)
    pol = halfk(g, prodct_mk_allk(g, W2, W1))
    em = -tor.sum(axis=1) + pol.sum(axis=1)
    ek = -tor.sum(axis=0) + pol.sum(axis=0)
    return em, (ek if with_k else None)


def specurv(espec, use_ratio=1.0 / 3.0):
    """SPECURV: trapezoidal P2 projection of log10 E over the top USE_RATIO of the spectrum."""
    floor, target = 1.0e-22, -0.05
    e = np.asarray(espec, dtype=np.float64)
    ie = e.size
    is_ = ie - max(1, int(ie * use_ratio))
    while ie > is_ and e[ie - 1] < floor:
        ie -= 1
    r_trunc = 1.0 - float(ie - is_) / float(e.size - is_)
    n = ie - is_ + 1
    if n < 10 or r_trunc > 0.2:
        return target
    logsp = np.log10(e[is_ - 1:ie])
    dx = 2.0 / (n - 1)
    curv = 0.0
    for i in range(1, n + 1):
        x = -1.0 + 2.0 * (i - 1) / (n - 1)
        fac = 0.5 if i in (1, n) else 1.0
        curv += fac * logsp[i - 1] * dx * math.sqrt(5.0 / 8.0) * (3.0 * x ** 2 - 1.0)
    return min(10.0, max(-10.0, curv))


def speslop(espec, ratio=1.0 / 3.0):
    """SPESLOP: trapezoidal P1 projection of log10 E against log10 k, as a slope."""
    floor, drop = 1.0e-24, 1.0e10
    e = np.asarray(espec, dtype=np.float64)
    ie = e.size
    is_ = ie - max(1, int(ie * ratio))
    k_start = is_
    rel_floor = e[is_ - 1:ie].max() / drop
    while ie > is_ and (e[ie - 1] < floor or e[ie - 1] < rel_floor):
        ie -= 1
    n = ie - is_ + 1
    if n < 3:
        return -3.0
    logsp = np.log10(e[is_ - 1:ie])
    logk = np.log10(np.arange(k_start, k_start + n, dtype=np.float64))
    xi_min, xi_max = logk[0], logk[n - 1]
    dx = 2.0 / (n - 1)
    slope = 0.0
    for i in range(1, n + 1):
        x = -1.0 + 2.0 * (logk[i - 1] - xi_min) / (xi_max - xi_min)
        fac = 0.5 if i in (1, n) else 1.0
        slope += fac * logsp[i - 1] * dx * math.sqrt(3.0 / 2.0) * x
    slope = slope * 2.0 / (xi_max - xi_min)
    return min(5.0, max(-15.0, slope))


def pdajust(coeff, current, previous, baseline, params, overdamp_threshold=None):
    """PDAJUST: returns the updated COEFF."""
    kp, kd, offset, scale = params
    control = kp * (current - previous) + kd * current + offset
    if overdamp_threshold is not None and current < overdamp_threshold and previous < overdamp_threshold:
        severity = min(5.0, abs(current - overdamp_threshold))
        control = -(0.1 + 0.05 * severity)
    control = min(1.0, max(-0.4, scale * control))
    coeff = (1.0 + control) * coeff
    return baseline if coeff < baseline else coeff


def _radial(mc, kc, mo, ko):
    if mc > kc:
        return (3.0 * mc + kc) / 4.0, (3.0 * mo + ko) / 4.0
    return (mc + 3.0 * kc) / 4.0, (mo + 3.0 * ko) / 4.0


class Hyp3Adj:
    """VISC's HYP3ADJ state (CURVMO ... KAPPAPB, mod_march.f90:74-78) and the controller."""

    def __init__(self):
        self.nupb = -1.0
        self.kappapb = -1.0
        self.hist = [0.0] * 4     # CURVMO CURVKO SLOPMO SLOPKO
        self.phist = [0.0] * 4    # PCURVMO PCURVKO PSLOPMO PSLOPKO

    @staticmethod
    def _metrics(em, ek):
        return (specurv(em, 0.25), specurv(ek, 0.25), speslop(em), speslop(ek))

    @staticmethod
    def _control(coef, met, old, base):
        """Returns (R, T, X) after the T/X and radial curvature + slope controllers."""
        mc, kc, ms, ks = met
        cmo, cko, smo, sko = old
        r, t, x = coef
        t_c = pdajust(t, mc, cmo, base, CURV_PARAMS, -1.0)
        x_c = pdajust(x, kc, cko, base, CURV_PARAMS, -1.0)
        t_s = pdajust(t, ms, smo, base, SLOPE_PARAMS)
        x_s = pdajust(x, ks, sko, base, SLOPE_PARAMS)
        t_new, x_new = max(t_c, t_s), max(x_c, x_s)
        cur, old_r = _radial(mc, kc, cmo, cko)
        r_c = pdajust(r, cur, old_r, base, CURV_PARAMS, -1.0)
        cur, old_r = _radial(ms, ks, smo, sko)
        r_s = pdajust(r, cur, old_r, base, SLOPE_PARAMS)
        return [min(max(r_c, r_s), 2.0), t_new, x_new]

    def adjust(self, g, ph, hyp, PSI, CHI, B=None):
        """HYP3ADJ(PSI, CHI, B) then the two HYP3SET (mod_march.f90:283-288)."""
        g.chopset(2)
        try:
            em, ek = enemon(g, PSI, CHI)
        finally:
            g.chopset(-2)
        met = self._metrics(em[:em.size - 2], ek)
        if self.nupb < 0.0:
            self.hist = list(met)
            self.nupb = BASELINE_NUP
        hyp.nup = self._control(hyp.nup, met, self.hist, self.nupb)
        self.hist = list(met)
        if B is not None:
            pemk = boussi_pe(g, B, ph.bv0)
            nt = g.NTCHOP
            pm = pemk[:nt - 2, :].sum(axis=1)
            pk = pemk.sum(axis=0)
            met = self._metrics(pm, pk)
            if self.kappapb < 0.0:
                self.phist = list(met)
                self.kappapb = self.nupb
            hyp.kappap = self._control(hyp.kappap, met, self.phist, self.kappapb)
            self.phist = list(met)
        hyp.reset(g, ph)
        return em, ek
