"""B200-native MLegS transform-and-step library: Python host binding.

The compute path is the CUDA library ``libmlegs_b200.so`` (C ABI in
include/mlegs_b200.h).  This module mirrors the reference's Fortran module
interface for the hot path -- TYPE(SCALAR) fields with space tags and log
terms, RTRAN/HORFFT/VERFFT/TOFF/TOFP, the mod_legops operators,
CALC_BOUSSI_FORCE and the SOLVER_T stepping -- over ctypes.  Arrays cross
the boundary in the reference's own layouts (Fortran index order (n|r, m|j,
k|z), complex128).  There is no CPU fallback: if the library cannot be
loaded, construction fails.
"""

import ctypes
import os

import numpy as np

from . import _lib
from .inputs import CONFIGS, Config, buoyancy_perturbation, perturbation_coefficients  # noqa: F401

PPP, FFF, PFP, PFF = 0, 1, 2, 3
PREC_FP64, PREC_SPLIT = 0, 1


class MlegsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("mlegs error %d: %s" % (code, msg))
        self.code = code


class Field:
    """TYPE(SCALAR) (mod_scalar3.f90:41-47) living on the device."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    @property
    def space(self):
        return self.ctx.lib.mlegs_field_space(self.h)

    def upload(self, E, ln=0.0, space=None):
        """Copy a reference-layout complex array (shape of ``space``) to the device."""
        space = self.ctx.space_of(E.shape) if space is None else space
        want = self.ctx.shape(space)
        if tuple(E.shape) != want:
            raise ValueError("shape %s does not match space %d %s" % (E.shape, space, want))
        buf = np.asfortranarray(E, dtype=np.complex128)
        self.ctx._ck(self.ctx.lib.mlegs_field_upload(self.ctx.c, self.h, space,
                                                     buf.ctypes.data_as(ctypes.c_void_p), float(ln)))
        return self

    def download(self, out=None):
        """Return (E, LN) in the reference layout of the field's current space.

        ``out``: optional preallocated Fortran-ordered complex128 array of that
        shape (e.g. in pinned host memory); it is filled and returned as is."""
        shape = self.ctx.shape(self.space)
        if out is None:
            E = np.empty(shape, dtype=np.complex128, order="F")
        else:
            if tuple(out.shape) != shape or out.dtype != np.complex128 or not out.flags.f_contiguous:
                raise ValueError("out must be a Fortran-ordered complex128 array of shape %s" % (shape,))
            E = out
        ln = ctypes.c_double(0.0)
        self.ctx._ck(self.ctx.lib.mlegs_field_download(self.ctx.c, self.h,
                                                       E.ctypes.data_as(ctypes.c_void_p),
                                                       ctypes.byref(ln)))
        return (np.ascontiguousarray(E) if out is None else E), ln.value


def params_of(cfg, precision=PREC_FP64, split_slices=0, device=0):
    """mlegs_params of a configuration."""
    p = _lib.Params()
    p.nr, p.nth, p.nx = cfg.nr, cfg.nth, cfg.nx
    p.nrchop, p.ntchop, p.nxchop = cfg.nrchop, cfg.ntchop, cfg.nxchop
    p.ell, p.zlen, p.dt = cfg.ell, cfg.zlen, cfg.dt
    p.adams = 1 if cfg.adams else 0
    p.omega, p.bv0, p.kappa, p.kappap = cfg.omega, cfg.bv0, cfg.kappa, cfg.kappap
    p.visc_sw, p.visc_p = cfg.visc_sw, cfg.p
    p.nu, p.nup = cfg.nu, cfg.nup
    p.precision, p.split_slices, p.device = precision, split_slices, device
    p.rmv_sw = int(getattr(cfg, "rmv_sw", 0))
    return p


class Context:
    """One grid + solver on one GPU (LEGINIT, mod_fft.f90:180-367)."""

    def __init__(self, cfg, precision=PREC_FP64, split_slices=0, device=0):
        self.lib = _lib.load()
        self.cfg = cfg
        self._owned = True
        self.device = int(device)
        p = params_of(cfg, precision, split_slices, device)
        h = ctypes.c_void_p()
        rc = self.lib.mlegs_create(ctypes.byref(p), ctypes.byref(h))
        if rc != 0:
            raise MlegsError(rc, "mlegs_create failed")
        self._attach(h)

    @classmethod
    def _wrap(cls, handle, cfg):
        """A context owned by someone else (an ensemble instance): not destroyed here."""
        self = cls.__new__(cls)
        self.lib = _lib.load()
        self.cfg = cfg
        self._owned = False
        self._attach(ctypes.c_void_p(handle))
        return self

    def _attach(self, h):
        self.c = h
        d = (ctypes.c_int32 * 9)()
        self.lib.mlegs_dims(self.c, d)
        (self.NDIMR, self.NDIMTH, self.NX, self.NRCHOPDIM, self.NTCHOPDIM, self.NXCHOPDIM,
         self.NRH, self.NR, self.NTH) = list(d)
        self.NTCHOP, self.NXCHOP = int(self.cfg.ntchop), int(self.cfg.nxchop)

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "c", None):
            if getattr(self, "_owned", True):
                self.lib.mlegs_destroy(self.c)
            self.c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != 0:
            msg = self.lib.mlegs_last_error(self.c)
            raise MlegsError(rc, msg.decode() if msg else "")
        return rc

    def shape(self, space):
        if space == FFF:
            return (self.NRCHOPDIM, self.NTCHOPDIM, self.NXCHOPDIM)
        if space == PFF:
            return (self.NDIMR, self.NTCHOPDIM, self.NXCHOPDIM)
        return (self.NDIMR, self.NDIMTH, self.NX)

    def space_of(self, shape):
        for sp in (FFF, PFF):
            if tuple(shape) == self.shape(sp):
                return sp
        raise ValueError("ambiguous space for shape %s; pass space=" % (shape,))

    def field(self, space=FFF, E=None, ln=0.0):
        h = ctypes.c_void_p()
        self._ck(self.lib.mlegs_field_alloc(self.c, space, ctypes.byref(h)))
        f = Field(self, h)
        if E is not None:
            f.upload(E, ln, space)
        return f

    def grid(self):
        n = self.NR
        x, w, r = (np.empty(n) for _ in range(3))
        dp = ctypes.POINTER(ctypes.c_double)
        self.lib.mlegs_grid(self.c, x.ctypes.data_as(dp), w.ctypes.data_as(dp), r.ctypes.data_as(dp))
        return x, w, r

    def sync(self):
        self._ck(self.lib.mlegs_sync(self.c))

    def launches(self):
        return self.lib.mlegs_launch_count(self.c)

    def reset_launches(self):
        self.lib.mlegs_reset_launch_count(self.c)

    # ------------------------------------------------------- transforms
    def RTRAN(self, f, IS, pad=0):
        self._ck(self.lib.mlegs_rtran(self.c, f.h, IS, pad))

    def HORFFT(self, f, IS):
        self._ck(self.lib.mlegs_horfft(self.c, f.h, IS))

    def VERFFT(self, f, IS):
        self._ck(self.lib.mlegs_verfft(self.c, f.h, IS))

    def PLNFFT(self, f, IS):
        self._ck(self.lib.mlegs_plnfft(self.c, f.h, IS))

    def TOFF(self, f, pad=0):
        self._ck(self.lib.mlegs_toff(self.c, f.h, pad))

    def TOFP(self, f, pad=0):
        self._ck(self.lib.mlegs_tofp(self.c, f.h, pad))

    def CHOPDO(self, f, pad=0):
        self._ck(self.lib.mlegs_chopdo(self.c, f.h, pad))

    def COPY(self, dst, src, pad=0):
        self._ck(self.lib.mlegs_field_copy(self.c, dst.h, src.h, pad))

    def AXPBY(self, y, a, x1, b=0.0, x2=None, c=0.0):
        self._ck(self.lib.mlegs_field_axpby(self.c, y.h, a, x1.h if x1 else None, b,
                                            x2.h if x2 else None, c))

    def SET_LN(self, f, ln):
        self._ck(self.lib.mlegs_field_set_ln(self.c, f.h, ln))

    # -------------------------------------------------------- operators
    def _unary(self, name, a, b, pad):
        self._ck(getattr(self.lib, name)(self.c, a.h, b.h, pad))
        return b

    def DELSQH(self, a, b, pad=0):
        return self._unary("mlegs_delsqh", a, b, pad)

    def IDELSQH(self, b, a, pad=0):
        return self._unary("mlegs_idelsqh", b, a, pad)

    def MULXM(self, a, b, pad=0):
        return self._unary("mlegs_mulxm", a, b, pad)

    def XXDX(self, a, b, pad=0):
        return self._unary("mlegs_xxdx", a, b, pad)

    def DEL2(self, a, b, pad=0):
        return self._unary("mlegs_del2", a, b, pad)

    def IDEL2LN(self, b, a, pad=0):
        return self._unary("mlegs_idel2ln", b, a, pad)

    def IDEL2(self, b, a, LN=None, pad=0):
        self._ck(self.lib.mlegs_idel2(self.c, b.h, a.h, 0 if LN is None else 1,
                                      0.0 if LN is None else float(LN), pad))
        return a

    def IHELM(self, b, a, alp, pad=0):
        self._ck(self.lib.mlegs_ihelm(self.c, b.h, a.h, float(alp), pad))
        return a

    def IHELMP(self, P, b, a, alp, NU=0.0, pad=0):
        """IHELMP(P, B, A, ALP, NUIN) (mod_legops.f90:1409-1592)."""
        self._ck(self.lib.mlegs_ihelmp(self.c, b.h, a.h, int(P), float(alp), float(NU), pad))
        return a

    def HYPERV(self, a, NU, NUP, P, DT):
        """HYPERV(A, NU, NUP, P, DT, WK) (mod_march.f90:1639-1686), A in place."""
        self._ck(self.lib.mlegs_hyperv(self.c, a.h, float(NU), float(NUP), int(P), float(DT)))
        return a

    def GRAD(self, a, rr, rp, gz, pad=0):
        self._ck(self.lib.mlegs_grad(self.c, a.h, rr.h, rp.h, gz.h, pad))

    def PC2VEL(self, psi, chi, rur, rup, uz, pad=0):
        self._ck(self.lib.mlegs_pc2vel(self.c, psi.h, chi.h, rur.h, rup.h, uz.h, pad))

    def PC2VOR(self, psi, chi, ror, rop, oz, pad=0):
        self._ck(self.lib.mlegs_pc2vor(self.c, psi.h, chi.h, ror.h, rop.h, oz.h, pad))

    def PROJECT(self, rur, rup, uz, psi, chi, LN=None):
        """LN: None, a number, or "psi" (the steppers' PSI%LN-by-reference form)."""
        if LN is None:
            mode, v = 0, 0.0
        elif isinstance(LN, str):
            mode, v = 2, 0.0
        else:
            mode, v = 1, float(LN)
        self._ck(self.lib.mlegs_project(self.c, rur.h, rup.h, uz.h, psi.h, chi.h, mode, v))

    def CALC_BOUSSI_FORCE(self, psi, chi, b, psin, chin, bn):
        self._ck(self.lib.mlegs_boussi_force(self.c, psi.h, chi.h, b.h, psin.h, chin.h, bn.h))

    def CALC_BOUSSI_NONLIN(self, b, rur, rup, uz, bn, ror, rop, oz):
        """CALC_BOUSSI_NONLIN(B, RUR, RUP, UZ, BN, ROR, ROP, OZ) (mod_boussinesq.f90:235-314):
        ROR, ROP, OZ become the velocity form of the projected u x omega, BN the
        FFF -(u.grad)b; RUR, RUP, UZ are consumed (left in PFP)."""
        self._ck(self.lib.mlegs_boussi_nonlin(self.c, b.h, rur.h, rup.h, uz.h, bn.h, ror.h, rop.h, oz.h))

    def legendre_table(self):
        """TFM%PF (mod_fft.f90:297) as built on the device: (NRH, NRCHOPDIM+1, NTCHOPDIM)."""
        out = np.empty((self.NRH, self.NRCHOPDIM + 1, self.NTCHOPDIM), dtype=np.float64, order="F")
        self._ck(self.lib.mlegs_legendre_table(self.c, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    # ------------------------------------------------------------ adjoint
    # Transposes and VJPs of the AB2-CN path (include/mlegs_b200.h, MLEGS_T_*);
    # cotangents are fields like any other, LN included where the map uses it.
    T_OPS = {"RTRAN+1": 0, "RTRAN-1": 1, "VERFFT+1": 2, "VERFFT-1": 3, "HORFFT+1": 4, "HORFFT-1": 5,
             "TOFP": 6, "TOFF": 7, "XXDX": 8, "MULXM": 9, "DELSQH": 10, "DEL2": 11, "GRAD": 12,
             "PC2VEL": 13, "PC2VOR": 14, "IDEL2LN": 15, "IHELM": 16, "PROJECT_PPP": 17, "VISC2": 18,
             "IDELSQH": 19, "FARFIELD": 20}

    @staticmethod
    def _handles(fields):
        arr = (ctypes.c_void_p * len(fields))(*[f.h for f in fields])
        return arr, ctypes.cast(arr, ctypes.c_void_p)

    def TRANSPOSE(self, op, ys, xs, pad=0, p1=0.0):
        """Transpose of one operator (name in T_OPS) at CHOPSET(pad): ys, the
        cotangents of its outputs -> xs, those of its inputs."""
        ya, yp = self._handles(list(ys))
        xa, xp = self._handles(list(xs))
        self._ck(self.lib.mlegs_transpose(self.c, self.T_OPS[op], yp, xp, int(pad), float(p1)))

    def CALC_BOUSSI_FORCE_VJP(self, psi, chi, b, psin_bar, chin_bar, bn_bar, psi_bar, chi_bar, b_bar):
        self._ck(self.lib.mlegs_boussi_force_vjp(self.c, psi.h, chi.h, b.h, psin_bar.h, chin_bar.h, bn_bar.h,
                                                 psi_bar.h, chi_bar.h, b_bar.h))

    def AB2_STEP_MAP(self, ins, outs):
        """One steady STEP_BOUSSI_AB_CN of (psi, chi, b, n_psi, n_chi, n_b)."""
        ia, ip = self._handles(list(ins))
        oa, op = self._handles(list(outs))
        self._ck(self.lib.mlegs_ab2_step_map(self.c, ip, op))

    def AB2_STEP_VJP(self, state, bars, outs):
        sa, sp = self._handles(list(state))
        ba, bp = self._handles(list(bars))
        oa, op = self._handles(list(outs))
        self._ck(self.lib.mlegs_ab2_step_vjp(self.c, sp, bp, op))

    def AB2_STARTUP_MAP(self, ins, outs):
        """RICH_BOUSSI_FE_BE of (psi, chi, b) -> (psi, chi, b, n_psi, n_chi, n_b)."""
        ia, ip = self._handles(list(ins))
        oa, op = self._handles(list(outs))
        self._ck(self.lib.mlegs_ab2_startup_map(self.c, ip, op))

    def AB2_STARTUP_VJP(self, state, bars, outs):
        sa, sp = self._handles(list(state))
        ba, bp = self._handles(list(bars))
        oa, op = self._handles(list(outs))
        self._ck(self.lib.mlegs_ab2_startup_vjp(self.c, sp, bp, op))

    def INITIAL_STATE_T(self, state_bar, coef_bar):
        sa, sp = self._handles(list(state_bar))
        ca, cp = self._handles(list(coef_bar))
        self._ck(self.lib.mlegs_initial_state_T(self.c, sp, cp))

    def ENERGY_OBJECTIVE(self, psi, chi, b, gpsi, gchi, gb):
        """J = fluctuation KE + 1/2 int b^2 dV; its gradient into (gpsi, gchi, gb)."""
        J = ctypes.c_double()
        self._ck(self.lib.mlegs_energy_objective(self.c, psi.h, chi.h, b.h, ctypes.byref(J), gpsi.h, gchi.h, gb.h))
        return J.value

    def DEVICE_COPY(self, f, to_field, space, ptr, ln_ptr=None):
        """Device-to-device copy between field f and a device buffer (device layout)."""
        self._ck(self.lib.mlegs_field_device_copy(self.c, f.h, 1 if to_field else 0, int(space),
                                                  ctypes.c_void_p(int(ptr)),
                                                  None if ln_ptr is None else ctypes.c_void_p(int(ln_ptr))))

    # ------------------------------------------------------------ diagnostics
    def _mk_array(self):
        return np.zeros((self.NXCHOP, self.NTCHOP), dtype=np.float64)  # Fortran order (NTCHOP, NXCHOP)

    def CALC_BOUSSI_ENERGY(self, psi, chi, b):
        """CALC_BOUSSI_ENERGY (mod_boussinesq.f90:139-232) without the file
        output: (KE, PE, DKE), each an (NTCHOP, NXCHOP) array over m >= 0,
        k >= 0.  The reference's especData_M / especData_K lines are
        KE.sum(axis=1) / KE.sum(axis=0) (likewise PE, DKE)."""
        ke, pe, dke = self._mk_array(), self._mk_array(), self._mk_array()
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self._ck(self.lib.mlegs_boussi_energy(self.c, psi.h, chi.h, b.h, ptr(ke), ptr(pe), ptr(dke)))
        return ke.T.copy(), pe.T.copy(), dke.T.copy()

    DIAGNOST_KEYS = ("VALVOR", "VALZMO", "VALANG", "VALENE", "VALHEL", "PAT1_SPREAD", "CAT1_SPREAD", "NORM_CHECK",
                     "VALX", "VALY", "VALR")

    def DIAGNOST(self, psi, chi):
        """DIAGNOST(PSI, CHI) (mod_march.f90:1689-1917) values as a dict (see
        mlegs_diagnost); raises MlegsError 11 / 12 on the dealiasing /
        divergence checks."""
        out = np.zeros(len(self.DIAGNOST_KEYS))
        self._ck(self.lib.mlegs_diagnost(self.c, psi.h, chi.h, out.ctypes.data_as(ctypes.c_void_p)))
        return dict(zip(self.DIAGNOST_KEYS, out.tolist()))

    def ENEMON(self, psi, chi, pad=0):
        """ENEMON(PSI, CHI, EM, EK) (mod_march.f90:2585-2617) at CHOPSET(pad): (EM, EK)."""
        em, ek = np.zeros(self.NTCHOP), np.zeros(self.NXCHOP)
        self._ck(self.lib.mlegs_enemon(self.c, psi.h, chi.h, pad, em.ctypes.data_as(ctypes.c_void_p),
                                       ek.ctypes.data_as(ctypes.c_void_p)))
        return em, ek

    def HYP3ADJ(self, psi, chi, b=None):
        """HYP3ADJ(PSI, CHI[, B]) and the stepper's two HYP3SET (mod_march.f90:283-288)."""
        self._ck(self.lib.mlegs_hyp3adj(self.c, psi.h, chi.h, b.h if b is not None else None))

    def hyp3_coeffs(self):
        """(NUP_R, NUP_T, NUP_X), (KAPPAP_R, KAPPAP_T, KAPPAP_X)."""
        out = np.zeros(6)
        self._ck(self.lib.mlegs_hyp3_coeffs(self.c, out.ctypes.data_as(ctypes.c_void_p)))
        return tuple(out[:3]), tuple(out[3:])

    def CALC_BOUSSI_PE(self, b):
        """CALC_BOUSSI_PE (mod_boussinesq.f90:112-136): (NTCHOP, NXCHOP) array."""
        pe = self._mk_array()
        self._ck(self.lib.mlegs_boussi_pe(self.c, b.h, pe.ctypes.data_as(ctypes.c_void_p)))
        return pe.T.copy()

    # ------------------------------------------------------------ snapshots
    def MSAVE(self, f, path, glb=True):
        """MSAVE0(A, FN, GLB) (mod_fft.f90:2224-2301): glb=True writes the global
        MSAVEX file, glb=False the MPISAVEX pair FN.info + FN (one process)."""
        self._ck(self.lib.mlegs_msave(self.c, f.h, os.fsencode(path), 1 if glb else 0))

    def MLOAD(self, path, f, glb=True):
        """MLOAD0(FN, A, GLB) (mod_fft.f90:2390-2633): loads E, SPACE and LN into f."""
        self._ck(self.lib.mlegs_mload(self.c, os.fsencode(path), f.h, 1 if glb else 0))

    # ------------------------------------------------------------ solver
    def initialize(self, psi, chi, b):
        """SOLVER_T%INITIALIZE: Richardson start-up step (mod_march.f90:171-240)."""
        self.state = (psi, chi, b)
        self._ck(self.lib.mlegs_solver_init(self.c, psi.h, chi.h, b.h))

    def step(self, n=1, graph=False):
        """n steady-state steps (STEP_BOUSSI_AB_CN / STEP_BOUSSI_ETDAB_CN)."""
        fn = self.lib.mlegs_step_graph if graph else self.lib.mlegs_step
        self._ck(fn(self.c, int(n)))

    def run_host(self, hosts, lns, n=1):
        """n graph-replayed steps with the state streamed through host memory
        (mlegs_run_host): per step psi, chi, b are uploaded from ``hosts`` (FFF,
        Fortran-ordered complex128, page-locked for overlapped copies) with LN
        ``lns`` and downloaded back into them.  Returns the last LN values."""
        if len(hosts) != 3 or len(lns) != 3:
            raise ValueError("run_host streams the three state fields psi, chi, b")
        want = self.shape(FFF)
        for h in hosts:
            if tuple(h.shape) != want or h.dtype != np.complex128 or not h.flags.f_contiguous:
                raise ValueError("hosts must be Fortran-ordered complex128 arrays of shape %s" % (want,))
        ptrs = (ctypes.c_void_p * 3)(*[h.ctypes.data for h in hosts])
        ln = (ctypes.c_double * 3)(*[float(v) for v in lns])
        self._ck(self.lib.mlegs_run_host(self.c, int(n), ctypes.cast(ptrs, ctypes.c_void_p), ln))
        return [ln[0], ln[1], ln[2]]

    def time(self):
        t = ctypes.c_double()
        n = ctypes.c_int32()
        self.lib.mlegs_time(self.c, ctypes.byref(t), ctypes.byref(n))
        return t.value, n.value

    def check_finite(self):
        self._ck(self.lib.mlegs_check_finite(self.c))

    def stream(self):
        return self.lib.mlegs_stream(self.c)

    KERNELS = {"rtran_b2p": 0, "rtran_p2b": 1, "verfft_b": 2, "verfft_f": 3, "horfft_b": 4,
               "horfft_f": 5, "pointwise": 6, "solve": 7, "phys": 8,
               "horfft_wb": 9, "horfft_wf": 10, "split_b2p": 11,
               "split_p2b": 12, "project": 13,
               "project_fff": 14, "phys_nonlin": 15, "roundtrip": 16, "dmma_peak": 17}

    def kernel_time(self, name, reps=20):
        """Mean device ms per launch of one internal kernel (CUDA events on the
        library's stream) and its algorithmic HBM bytes per launch."""
        ms, by = ctypes.c_double(), ctypes.c_double()
        self._ck(self.lib.mlegs_kernel_time(self.c, self.KERNELS[name], reps, ctypes.byref(ms),
                                            ctypes.byref(by)))
        return ms.value, by.value


class Ensemble:
    """Independent AB2-CN runs of different grids advanced in lock-step on one
    GPU with grouped launches (mlegs_ensemble_*, include/mlegs_b200.h); no
    counterpart in the reference.  ``contexts[i]`` is instance i's Context
    (fields, uploads, ``initialize``), owned by the ensemble."""

    def __init__(self, cfgs, device=0):
        self.lib = _lib.load()
        self.cfgs = list(cfgs)
        arr = (_lib.Params * len(self.cfgs))(*[params_of(c, device=device) for c in self.cfgs])
        h = ctypes.c_void_p()
        rc = self.lib.mlegs_ensemble_create(arr, len(self.cfgs), ctypes.byref(h))
        if rc != 0:
            raise MlegsError(rc, "mlegs_ensemble_create failed")
        self.e = h
        self.contexts = [Context._wrap(self.lib.mlegs_ensemble_context(self.e, i), c)
                         for i, c in enumerate(self.cfgs)]

    def _ck(self, rc):
        if rc != 0:
            msg = self.lib.mlegs_ensemble_last_error(self.e)
            raise MlegsError(rc, msg.decode() if msg else "")

    def step(self, n=1, graph=True):
        self._ck(self.lib.mlegs_ensemble_step(self.e, int(n), 1 if graph else 0))

    def tune(self):
        self._ck(self.lib.mlegs_ensemble_tune(self.e))

    def tuning(self):
        """(rows, ctas): rows of (transform 0 RTRAN(+1) / 1 fold, NRH, NRCHOP,
        tile columns) chosen by the autotuner; CTAs per SM per transform."""
        buf = (ctypes.c_int32 * 512)()
        n = self.lib.mlegs_ensemble_tuning(self.e, buf, 128)
        rows = [tuple(buf[4 * i:4 * i + 4]) for i in range(max(n, 0))]
        c = (ctypes.c_int32 * 2)()
        self._ck(self.lib.mlegs_ensemble_ctas(self.e, c))
        return rows, (c[0], c[1])

    def sync(self):
        self._ck(self.lib.mlegs_ensemble_sync(self.e))

    def stream(self):
        return self.lib.mlegs_ensemble_stream(self.e)

    def launches(self):
        return self.lib.mlegs_ensemble_launch_count(self.e)

    def close(self):
        if getattr(self, "e", None):
            for c in self.contexts:
                c.c = None
            self.lib.mlegs_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _spectrum_call(name, espec, ratio):
    e = np.ascontiguousarray(espec, dtype=np.float64)
    out = ctypes.c_double(0.0)
    rc = getattr(_lib.load(), name)(e.ctypes.data_as(ctypes.c_void_p), e.size, float(ratio), ctypes.byref(out))
    if rc != 0:
        raise MlegsError(rc, name)
    return out.value


def SPECURV(espec, use_ratio=1.0 / 3.0):
    """SPECURV(ESPEC, USE_RATIO), mod_march.f90:2619-2698 (host code, no device)."""
    return _spectrum_call("mlegs_specurv", espec, use_ratio)


def SPESLOP(espec, ratio=1.0 / 3.0):
    """SPESLOP(ESPEC, RATIO), mod_march.f90:2700-2774 (host code, no device)."""
    return _spectrum_call("mlegs_speslop", espec, ratio)


def PDAJUST(coeff, current, previous, baseline, params, overdamp_threshold=None):
    """PDAJUST(COEFF, CURRENT, PREVIOUS, BASELINE, PARAMS[, OVERDAMP_THRESHOLD]),
    mod_march.f90:2776-2812; returns the updated COEFF (host code, no device)."""
    c = ctypes.c_double(coeff)
    prm = np.ascontiguousarray(params, dtype=np.float64)
    rc = _lib.load().mlegs_pdajust(ctypes.byref(c), float(current), float(previous), float(baseline),
                                   prm.ctypes.data_as(ctypes.c_void_p), int(overdamp_threshold is not None),
                                   float(overdamp_threshold or 0.0))
    if rc != 0:
        raise MlegsError(rc, "mlegs_pdajust")
    return c.value


VORTEX_DEFAULTS = dict(x=0.0, y=0.0, q=1.0, h=0.0, b=1.0, dx=0.0, dy=0.0, k=0.0, dp=0.0,
                       r=1.0, dr=0.0, rk=0.0, rp=0.0)


def QVORTEX(ctx, vortices, noise_seeds=None):
    """QVORTEX(PSI, CHI) (mod_layout.f90:449-609) on the device for a QPAIR
    list: each entry a dict with any of the keys of VORTEX_DEFAULTS (X, Y, Q, H,
    B, DX, DY, K, DP, R, DR, RK, RP in lower case).  noise_seeds: None for
    NOISE = 0, or the two RAN0 seeds (PSI, CHI) of NOISE = 1.  Returns (psi, chi)."""
    arr = (_lib.Vortex * len(vortices))()
    for i, v in enumerate(vortices):
        unknown = set(v) - set(VORTEX_DEFAULTS)
        if unknown:
            raise ValueError("unknown vortex keys %s" % sorted(unknown))
        full = dict(VORTEX_DEFAULTS, **v)
        for key, val in full.items():
            setattr(arr[i], key, float(val))
    psi, chi = ctx.field(FFF), ctx.field(FFF)
    seeds = None
    if noise_seeds is not None:
        seeds = (ctypes.c_int32 * 2)(*[int(x) for x in noise_seeds])
    ctx._ck(ctx.lib.mlegs_qvortex(ctx.c, arr, len(vortices), seeds, psi.h, chi.h))
    return psi, chi


def HYP3_CONTROLLER(em, ek, state, coef):
    """One field's HYP3ADJ controller (mod_march.f90:3025-3101) on given spectra
    (host code, no device).  state: [NUPB, CURVMO, CURVKO, SLOPMO, SLOPKO]
    (NUPB < 0 before the first call); coef: [R, T, X].  Returns the updated
    (state, coef) as new arrays."""
    e_m = np.ascontiguousarray(em, dtype=np.float64)
    e_k = np.ascontiguousarray(ek, dtype=np.float64)
    st = np.array(state, dtype=np.float64)
    cf = np.array(coef, dtype=np.float64)
    rc = _lib.load().mlegs_hyp3_controller(e_m.ctypes.data_as(ctypes.c_void_p), e_m.size,
                                           e_k.ctypes.data_as(ctypes.c_void_p), e_k.size,
                                           st.ctypes.data_as(ctypes.c_void_p), cf.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise MlegsError(rc, "mlegs_hyp3_controller")
    return st, cf


def qvortex(ctx, q=1.0, r0=1.0, xc=0.0, yc=0.0, h=0.0, b=1.0):
    """One Gaussian q-vortex (QVORTEX with a single QPAIR entry) on the device."""
    return QVORTEX(ctx, [dict(q=q, r=r0, x=xc, y=yc, h=h, b=b)])


def initial_state(ctx, cfg=None):
    """Vortex + seeded perturbation (construction in mlegs_b200.inputs), on the device."""
    cfg = ctx.cfg if cfg is None else cfg
    psi, chi = qvortex(ctx)
    b = ctx.field(FFF)
    tmp = ctx.field(FFF)
    out = ctx.field(FFF)
    for F, fid in ((psi, 0), (chi, 1)):
        c = perturbation_coefficients(cfg, fid)
        tmp.upload(-c, 0.0, FFF)
        ctx.CHOPDO(tmp)
        ctx.IDELSQH(tmp, out)
        ctx.AXPBY(F, 1.0, out, 0.0, None, 1.0)
        ctx.CHOPDO(F)
    b.upload(buoyancy_perturbation(cfg), 0.0, FFF)
    return psi, chi, b


__all__ = ["Context", "Ensemble", "params_of", "Field", "MlegsError", "qvortex", "QVORTEX", "initial_state", "CONFIGS", "Config",
           "SPECURV", "SPESLOP", "PDAJUST", "HYP3_CONTROLLER",
           "PPP", "FFF", "PFP", "PFF", "PREC_FP64", "PREC_SPLIT"]
