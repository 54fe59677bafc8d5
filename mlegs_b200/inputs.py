"""Benchmark configurations and seeded synthetic inputs (host-side numpy).

The reference publishes no dataset; every run here starts from the same
construction the reference's drivers use (f90/bsnsq_test.f90:39-41):
one Gaussian q-vortex (QVORTEX, mod_layout.f90:449-609, core radius 1,
Q = 1, H = 0, at the origin) and b = 0, plus a seeded spectral perturbation.

The perturbation is built like QVORTEX builds the vortex itself: random
FFF coefficients stand for (1-x)^-2 omega_z' and (1-x)^-2 u_z' and are
turned into psi', chi' by the inverse horizontal Laplacian (IDELSQH,
mod_legops.f90:136-241) -- i.e. psi' = -IDELSQH(c_psi), chi' = -IDELSQH(c_chi)
-- while b' takes the coefficients directly with its far-field value
removed (the CALCAT1 fix the reference applies, mod_legops.f90:2540).
Coefficient envelope: amp * exp(-n/decay) for |m| <= mmax, |k| <= kmax,
Gaussian real/imaginary parts from numpy's Philox generator seeded with
seed + field id (0 = psi, 1 = chi, 2 = b); m = 0 is made Hermitian in k
(coef(-k) = conj coef(k), real at k = 0) like f90/bsnsq_gauss.f90:177-210.
The (n, m, k) = (0, 0, 0) entry is zero so the vortex keeps its log term.
"""

import math
from dataclasses import dataclass, field


@dataclass
class Config:
    """One benchmark / parity configuration (grid, physics, run length)."""
    name: str
    nr: int
    nth: int
    nx: int
    nrchop: int
    ntchop: int
    nxchop: int
    ell: float = 1.0
    zlen: float = 2 * math.pi
    dt: float = 1e-3
    nsteps: int = 100
    adams: bool = True
    omega: float = 1.0
    bv0: float = 1.0
    visc_sw: int = 1
    nu: float = 1e-3
    kappa: float = 1e-3
    nup: float = 0.0
    kappap: float = 0.0
    p: int = 2
    rmv_sw: int = 0          # REMOVE SW (2: axial sponge in the ETD steps)
    amp: float = 1e-3
    mmax: int = 4
    kmax: int = 4
    decay: float = 8.0
    seed: int = 1234
    notes: list = field(default_factory=list)


def chops(nr, nth, nx):
    """2/3 dealiasing rule with the reference's limits (NRCHOP <= NR-6 so that
    CHOPSET(3) cannot stop, 2*NXCHOP <= NX): mod_fft.f90:231-243."""
    return min(2 * nr // 3, nr - 6), 2 * nth // 3, nx // 3


CONFIGS = {
    # AB2-CN IVP as the reference runs it; NRCHOP 64 -> 58 (= NR-6), see notes.
    "ab2_64x32x32": Config(
        "ab2_64x32x32", 64, 32, 32, 58, 16, 16, dt=1e-3, nsteps=100, adams=True,
        omega=1.0, bv0=1.0, visc_sw=1, nu=1e-3, kappa=1e-3, amp=1e-3, mmax=4, kmax=4, decay=8.0,
        notes=["NRCHOP=64=NR makes CHOPSET(3) stop (mod_scalar3.f90:192-200); run with 58 = NR-6",
               "KAPPA unspecified: Pr = 1 (KAPPA = NU)"]),
    # Mixed-precision ETD timestep (the headline workload).
    "etd_192x128x256": Config(
        "etd_192x128x256", 192, 128, 256, 128, 85, 85, dt=5e-4, nsteps=100, adams=False,
        omega=1.0, bv0=2.0, visc_sw=3, nu=1.0 / 5000, kappa=0.0, nup=1e-10, kappap=1e-10, p=2,
        amp=1e-2, mmax=8, kmax=16, decay=10.0,
        notes=["VISC%SW=3: Re=5000 has no effect (CALC_BOUSSI_VISC_CN returns, mod_march.f90:1251)"]),
    # Transform round trips at 256^3 (batch of 8 fields; chi, psi, b coefficients).
    "roundtrip_256": Config("roundtrip_256", 256, 256, 256, 170, 170, 85, decay=10.0),
    # Gradient of the final fluctuation KE + buoyancy variance after the
    # start-up and 200 AB2-CN steps w.r.t. the perturbation coefficients
    # (checkpoints every 20 steps).
    "grad_96x64x64": Config(
        "grad_96x64x64", 96, 64, 64, 64, 42, 21, dt=1e-3, nsteps=200, adams=True,
        omega=1.0, bv0=1.0, visc_sw=1, nu=1.0 / 2000, kappa=1.0 / 2000, amp=1e-4, mmax=4, kmax=4, decay=8.0,
        notes=["Re = 2000: NU = 1/2000; KAPPA unspecified: Pr = 1 (KAPPA = NU)",
               "checkpoint every 20 steps with recomputation"]),
}


def small_config(name, nr, nth, nx, adams=True, **kw):
    """A reduced-size configuration with the same physics as the named one."""
    base = CONFIGS["ab2_64x32x32" if adams else "etd_192x128x256"]
    nrc, ntc, nxc = chops(nr, nth, nx)
    d = dict(base.__dict__)
    d.update(name=name, nr=nr, nth=nth, nx=nx, nrchop=nrc, ntchop=ntc, nxchop=nxc)
    d.update(kw)
    d["notes"] = list(base.notes)
    return Config(**d)


def fff_shape(cfg):
    nrchopdim = min(cfg.nrchop + 6, cfg.nr)
    return (nrchopdim, min(cfg.ntchop, cfg.nth), 2 * cfg.nxchop - 1)


def perturbation_coefficients(cfg, fid, amp=None):
    """Random FFF coefficients E[n, m, k] (before IDELSQH / far-field fix)."""
    import numpy as np

    amp = cfg.amp if amp is None else amp
    shape = fff_shape(cfg)
    rng = np.random.Generator(np.random.Philox(cfg.seed + fid))
    e = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    n = np.arange(shape[0])[:, None, None]
    m = np.arange(shape[1])[None, :, None]
    kk = np.arange(shape[2])
    kv = np.where(kk + 1 > cfg.nxchop, -(shape[2] - kk), kk)
    mask = (m <= cfg.mmax) & (np.abs(kv)[None, None, :] <= cfg.kmax)
    e = e * amp * np.exp(-n / cfg.decay) * mask
    neg = np.r_[0, np.arange(shape[2] - 1, 0, -1)]
    e[:, 0, :] = 0.5 * (e[:, 0, :] + np.conj(e[:, 0, neg]))
    e[0, 0, 0] = 0.0
    return e


def buoyancy_perturbation(cfg):
    """b' = c_b chopped at NRCHOPS(m) = NRCHOP - m, with the m = 0 far-field value
    removed: E(1,1,:) -= sum_{n < NRCHOP} AT1(n) E(n,1,:) / AT1(1), AT1(n) = sqrt((2n+1)/2)
    (the CALCAT1 fix of mod_legops.f90:2540 / mod_scalar3.f90:286-310)."""
    import numpy as np

    e = perturbation_coefficients(cfg, 2)
    nrcd, ntcd, _ = e.shape
    for m in range(ntcd):
        e[max(cfg.nrchop - m, 0):, m, :] = 0.0
    at1 = np.sqrt((2 * np.arange(cfg.nrchop) + 1) / 2.0)
    e[0, 0, :] -= (at1 @ e[:cfg.nrchop, 0, :]) / at1[0]
    return e


def roundtrip_coefficients(cfg, fid):
    """Spectral coefficients of the transform round-trip workload: E[n, m, k]
    with amplitude exp(-(n + |m| + |k|) / decay) and Gaussian real and
    imaginary parts (numpy Philox, seed + fid; fid 0 chi, 1 psi, 2 b, further
    ids for the rest of a batch), chopped at NRCHOPS(m) = NRCHOP - m, Hermitian
    in k at m = 0 (coef(-k) = conj coef(k), real at k = 0)."""
    import numpy as np

    shape = fff_shape(cfg)
    rng = np.random.Generator(np.random.Philox(cfg.seed + 100 + fid))
    e = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    n = np.arange(shape[0])[:, None, None]
    m = np.arange(shape[1])[None, :, None]
    kk = np.arange(shape[2])
    kv = np.where(kk + 1 > cfg.nxchop, -(shape[2] - kk), kk)
    e = e * np.exp(-(n + m + np.abs(kv)[None, None, :]) / cfg.decay)
    neg = np.r_[0, np.arange(shape[2] - 1, 0, -1)]
    e[:, 0, :] = 0.5 * (e[:, 0, :] + np.conj(e[:, 0, neg]))
    for mm in range(shape[1]):
        e[max(cfg.nrchop - mm, 0):, mm, :] = 0.0
    return e


ENSEMBLE_NR = (48, 64, 96, 128, 192)
ENSEMBLE_NTH = (32, 64, 128)
ENSEMBLE_NX = (32, 64, 128, 256)


def ensemble_configs(n=64, seed=2024, nrs=ENSEMBLE_NR, nths=ENSEMBLE_NTH, nxs=ENSEMBLE_NX):
    """The batched-run configuration: n independent AB2-CN runs with (NR, NTH,
    NX) drawn uniformly from nrs x nths x nxs, Re uniform in [500, 5000] (NU =
    KAPPA = 1/Re), N uniform in [0.5, 4], dt = 1e-3, the AB2-CN IVP physics
    otherwise (Omega = 1, VISC%SW = 1) and its initial condition (q-vortex plus
    a perturbation of amplitude 1e-3 in |m|, |k| <= 4 decaying as exp(-n/8)),
    seeded per instance; chops by the 2/3 rule (chops())."""
    import numpy as np

    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(n):
        nr = int(rng.choice(nrs))
        nth = int(rng.choice(nths))
        nx = int(rng.choice(nxs))
        re = float(rng.uniform(500.0, 5000.0))
        bv0 = float(rng.uniform(0.5, 4.0))
        nrc, ntc, nxc = chops(nr, nth, nx)
        out.append(Config("ens%02d_%dx%dx%d" % (i, nr, nth, nx), nr, nth, nx, nrc, ntc, nxc, dt=1e-3, nsteps=50,
                          adams=True, omega=1.0, bv0=bv0, visc_sw=1, nu=1.0 / re, kappa=1.0 / re, amp=1e-3,
                          mmax=4, kmax=4, decay=8.0, seed=1234 + 7 * i,
                          notes=["Re = %.1f, N = %.3f" % (re, bv0)]))
    return out
