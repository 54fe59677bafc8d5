"""CPU tests of the oracle against the reference's known answers and golden vectors.

Known answers restated from the reference's own tests and notes:
  * divxm analytic case (tests/mlegs/divxm_test.f90:79-86): (1-x) Pbar_2 has
    normalised coefficients (-2/5 N3/N2, 1, -3/5 N3/N4) -> MULXM KAT;
  * one Gaussian q-vortex has psi log term -0.5 wherever it sits (notes:3-8);
  * PF is orthonormal under the Gauss weights (RTRAN +-1 symmetry,
    mod_fft.f90:1230-1243 vs 1284-1292; tests/mlegs/test_prodct.f90:41-45);
  * FFF -> PPP -> FFF is the identity for band-limited fields;
  * ETD_E / ETD_NL against a dense matrix exponential (the reference echoes
    S S^-1 and S J S^-1 for this check, mod_boussinesq.f90:92-105);
  * the golden 50-digit tables of tests/golden/legendre_golden.npz.
"""

import math
import os

import numpy as np
import pytest
import scipy.linalg as sl

from conftest import oracle_grid, oracle_physics, random_fff, rel, small_cfg

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "legendre_golden.npz")


def test_gauss_legendre_golden():
    from oracle.grid import gauss_legendre
    z = np.load(GOLDEN)
    for ci in range(4):
        nr = int(z["c%d_nr" % ci])
        x, w = gauss_legendre(nr)
        assert np.abs(x - z["c%d_x" % ci]).max() < 5e-15
        assert rel(w, z["c%d_w" % ci]) < 5e-14


def test_legendre_table_golden():
    from oracle.grid import gauss_legendre, leg_log_norm, leg_table
    z = np.load(GOLDEN)
    for ci in range(4):
        nr = int(z["c%d_nr" % ci])
        ms = list(z["c%d_ms" % ci])
        gold = z["c%d_pf" % ci]
        ne = gold.shape[1]
        x = z["c%d_x" % ci][: nr // 2]
        pf = leg_table(x, ne, ms)
        # relative to each (m) slice's scale; entries that underflow stay zero
        for j in range(len(ms)):
            assert rel(pf[:, :, j], gold[:, :, j]) < 1e-12, (ci, ms[j])
            assert np.array_equal(pf[:, :, j] == 0.0, gold[:, :, j] == 0.0)
        ln = leg_log_norm(ne + 14, ms)
        assert rel(ln, z["c%d_lognorm" % ci]) < 1e-14
        # the nodes the oracle itself produces give the same table to roundoff
        xo, _ = gauss_legendre(nr)
        assert rel(leg_table(xo[: nr // 2], ne, ms), gold) < 1e-11


def test_pf_orthonormal():
    g = oracle_grid(small_cfg(64, 32, 32))
    for mm in (0, 3, 15):
        pf = g.PF[:, :30, mm]
        G = 2 * (pf.T * g.W[: g.NRH]) @ pf
        par = (np.arange(30)[:, None] + np.arange(30)[None, :]) % 2
        G[par == 1] = 0
        assert np.abs(G - np.eye(30)).max() < 1e-13


def test_roundtrip_identity():
    from oracle import transforms as T
    g = oracle_grid(small_cfg(64, 32, 32))
    A = random_fff(g, 0)
    B = A.copy()
    T.tofp(g, B)
    T.toff(g, B)
    assert rel(B.E, A.E) < 1e-13


def test_mulxm_divxm_kat():
    from oracle import legops as L
    from oracle.grid import FFF
    g = oracle_grid(small_cfg(64, 32, 32))
    A = g.alloc(FFF)
    A.E[2, 0, :] = 1.0
    B = L.mulxm(g, A)
    n0 = g.NORM0
    assert abs(B.E[1, 0, 0] - (-2.0 / 5.0 * n0[2] / n0[1])) < 1e-15
    assert abs(B.E[2, 0, 0] - 1.0) < 1e-15
    assert abs(B.E[3, 0, 0] - (-3.0 / 5.0 * n0[2] / n0[3])) < 1e-15


@pytest.mark.parametrize("xc", [0.0, 0.7])
def test_qvortex_logterm(xc):
    from oracle import layout
    g = oracle_grid(small_cfg(64, 32, 32))
    psi, chi = layout.qvortex(g, xc=xc)
    assert abs(psi.LN + 0.5) < 1e-12
    assert chi.LN == 0.0


def test_gaus_matches_reference_notebook():
    """The oracle's GAUS against the reference's own Python restatement of it
    (tests/init/visualize_gaussian.ipynb), golden values from
    tests/golden/make_gaus_golden.py, with the waviness and core modulation."""
    import os
    from oracle import layout
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "gaus_golden.npz"))
    keys = [str(k) for k in d["keys"]]
    for prm, ref in zip(d["params"], d["vals"]):
        p = dict(zip(keys, prm))
        v = layout.vortex(x=p["XC"], y=p["YC"], dx=p["DX"], dy=p["DY"], k=p["K"], dp=p["DP"], r=p["R"],
                          dr=p["DR"], rk=p["RK"], rp=p["RP"])
        got = layout.gaus_value(v, p["Q"], p["B"], d["x"], d["y"], d["z"], p["ZLEN"])
        assert np.abs(got - ref).max() <= 1e-15 * max(1.0, np.abs(ref).max())


def test_qvortex_list_logterms():
    """QVORTEX over a QPAIR list: PSI%LN = -sum(Q)/2 and CHI%LN = -sum(H/B)/4
    (the circulations 2 pi Q and pi H / B of the Gaussians over 4 pi), with the
    z-waviness and core modulation in use; a one-entry list equals the
    single-vortex form."""
    from oracle import layout
    g = oracle_grid(small_cfg(64, 32, 32))
    vs = [layout.vortex(x=0.4, y=-0.2, q=1.0, h=0.3, b=1.5, dx=0.05, dy=-0.03, k=1.0, dp=30.0, dr=0.1,
                        rk=2.0, rp=-45.0),
          layout.vortex(x=-0.5, y=0.6, q=-0.7, h=-0.2, b=0.8, r=0.8)]
    psi, chi = layout.qvortex_list(g, vs)
    assert abs(psi.LN + 0.5 * 0.3) < 1e-12
    assert abs(chi.LN + (0.3 / 1.5 - 0.2 / 0.8) / 4.0) < 1e-12
    p1, c1 = layout.qvortex(g, q=1.0, h=0.5, b=2.0, r0=1.2, xc=0.3, yc=-0.1)
    p2, c2 = layout.qvortex_list(g, [layout.vortex(q=1.0, h=0.5, b=2.0, r=1.2, x=0.3, y=-0.1)])
    assert np.array_equal(p1.E, p2.E) and np.array_equal(c1.E, c2.E) and p1.LN == p2.LN


def test_ran0_and_noise():
    """RAN0 is the Park-Miller minimal standard behind an XOR mask: from state 1
    the 10000th state is 1043618065 (Park & Miller's check value).  NOISE touches
    only n < NRCHOPS(m), m < NTCHOP, with |dE| <= 0.1 ALEVEL max|A| per part;
    FLATTEN keeps B where B is zero and A where |B| is large."""
    from oracle import layout
    r = layout.Ran0(1 ^ layout.Ran0.MASK)
    for _ in range(10000):
        r()
    assert r.idum ^ layout.Ran0.MASK == 1043618065
    g = oracle_grid(small_cfg(32, 16, 16))
    psi, _ = layout.qvortex(g)
    A = g.copy0(psi)
    A0 = A.E.copy()
    layout.noise(g, A, 0.02, 4242)
    d = A.E - A0
    ref = 0.02 * np.abs(A0).max()
    assert np.abs(d.real).max() <= 0.1 * ref and np.abs(d.imag).max() <= 0.1 * ref and np.abs(d).max() > 0
    for mm in range(g.NTCHOPDIM):
        assert not np.any(d[int(g.NRCHOPS[mm]):, mm, :])
    from oracle.grid import PPP
    B = g.alloc(PPP)
    B.E[:g.NR, :g.NTH, :] = 1.0 + 1.0j
    B.E[0, 0, 0] = 0.0
    C = g.alloc(PPP)
    C.E[:] = 0.5
    layout.flatten(g, C, B)
    # REFVAL = max |Re A| = 0.5: where B = 0 the result is B; where B = 1 + i it is
    # B + (A - B) tanh(20 / 0.5)^2 per part
    t2 = np.tanh(40.0) ** 2
    expect = (1.0 + (0.5 - 1.0) * t2) + 1j * (1.0 + (0.0 - 1.0) * t2)
    assert C.E[0, 0, 0] == 0.0 and abs(C.E[1, 1, 1] - expect) < 1e-15


def test_etd_matches_expm():
    from oracle.boussinesq import calc_boussi_diag, calc_boussi_etd_op
    J, S, Si = calc_boussi_diag(2.0, 1.0)
    L = S @ J @ Si
    E, NL = calc_boussi_etd_op(2.0, 1.0, 5e-4)
    assert np.abs(E - sl.expm(L * 5e-4)).max() < 1e-14
    # phi_1(L dt) dt = L^-1 (e^{L dt} - I)
    assert np.abs(NL - np.linalg.solve(L, sl.expm(L * 5e-4) - np.eye(4))).max() < 1e-14


def test_band_lu_matches_dense():
    from oracle.bandmat import band_del2h, band_lu_solve, band_to_full
    g = oracle_grid(small_cfg(32, 16, 16))
    b = band_del2h(20, 3, 1.0, g.LOGNORM[:, 3])
    b[:, 2] -= 2.5
    rhs = np.random.default_rng(1).standard_normal(20) + 0j
    x = band_lu_solve(b[None], 2, rhs[None])[0]
    full = band_to_full(b, 2)
    assert rel(full @ x, rhs) < 1e-12


def test_projection_identity_physical():
    """PC2VEL -> TOFP (CHOPSET(3)) -> PROJECT -> IDEL2LN recovers (psi, chi)."""
    from oracle import legops as L
    from oracle import transforms as T
    g = oracle_grid(small_cfg(64, 32, 32))
    psi = random_fff(g, 1, decay=4.0)
    chi = random_fff(g, 2, decay=4.0)
    for F in (psi, chi):
        F.E[0, 0, :] -= g.calcat1(F) / g.AT1[0]
    g.chopset(3)
    U = L.pc2vel(g, psi, chi)
    for u in U:
        T.tofp(g, u)
    g.chopset(-3)
    P2, W2 = L.project(g, *U, None)
    C2 = L.idel2ln(g, W2)
    assert rel(P2.E, psi.E) < 1e-11
    assert rel(C2.E, chi.E) < 1e-9


def test_buoyancy_column_accelerates():
    """z-uniform axisymmetric b accelerates u_z = -b t (no pressure gradient at k = 0)."""
    from oracle import boussinesq as BQ
    from oracle import legops as L
    from oracle import transforms as T
    from oracle.grid import FFF
    from conftest import oracle_physics
    cfg = small_cfg(64, 32, 32)
    g = oracle_grid(cfg)
    b = random_fff(g, 3, decay=4.0)
    b.E[:, 1:, :] = 0
    b.E[:, :, 1:] = 0
    b.E *= 1e-3
    b.E[0, 0, 0] -= g.calcat1(b)[0] / g.AT1[0]
    b0 = b.copy()
    s = BQ.Solver(g, oracle_physics(cfg), g.alloc(FFF), g.alloc(FFF), b)
    s.initialize()
    for _ in range(9):
        s.step()
    g.chopset(3)
    uz = L.pc2vel(g, s.psi, s.chi)[2]
    g.chopset(-3)
    T.tofp(g, uz)
    T.tofp(g, b0)
    want = -b0.E[: g.NR, 0, 0].real * s.t
    assert rel(uz.E[: g.NR, 0, 0].real, want) < 5e-3


def test_inputs_deterministic():
    from mlegs_b200.inputs import CONFIGS, perturbation_coefficients
    cfg = CONFIGS["ab2_64x32x32"]
    a = perturbation_coefficients(cfg, 0)
    b = perturbation_coefficients(cfg, 0)
    assert np.array_equal(a, b)
    neg = np.r_[0, np.arange(a.shape[2] - 1, 0, -1)]
    assert np.allclose(a[:, 0, :], np.conj(a[:, 0, neg]))
    assert a[0, 0, 0] == 0


def test_pe_matches_physical_integral():
    """L2NORM_MK_HALFK / CALC_BOUSSI_PE summed over (m, k) equals the
    physical-space integral of b^2 / (2 N^2) on the collocation grid
    (Gauss weights with r dr = ELL^2 dx / (1 - x)^2, uniform theta and z)."""
    from oracle import diagnostics as D
    from oracle import transforms as T
    cfg = small_cfg(32, 16, 16, adams=False)
    g = oracle_grid(cfg)
    B = random_fff(g, 5, decay=3.0)
    bv0 = 2.0
    pe = D.boussi_pe(g, B, bv0)
    P = B.copy()
    T.tofp(g, P)
    f = T.physical_samples(g, P)
    wr = g.ELL2 * g.W[:g.NR] / (1 - g.X[:g.NR]) ** 2
    integ = np.einsum("i,isl->", wr, f * f) * (math.pi / g.NTH) * (g.ZLEN / g.NX)
    assert abs(pe.sum() - integ / 2 / bv0 ** 2) < 1e-13 * integ
    assert pe.shape == (g.NTCHOP, g.NXCHOP) and (pe >= 0).all()


def test_diagnost_known_answers():
    """DIAGNOST restated: the n = 0 row of DELSQH is the log term alone, so
    VALVOR = -4 pi ZLEN PSI%LN and VALZMO = -4 pi ZLEN CHI%LN; VALENE is twice
    the kinetic energy that CALC_BOUSSI_ENERGY sums over (m, k); the
    dealiasing and divergence checks raise the reference's abort codes; CALCXY
    finds the centre of an off-axis q-vortex."""
    from oracle import diagnostics as D
    cfg = small_cfg(32, 16, 16, adams=False)
    g = oracle_grid(cfg)
    PSI, CHI, B = (random_fff(g, 60 + i, decay=4.0) for i in range(3))
    PSI.LN, CHI.LN = 0.3, -0.2
    v = D.diagnost(g, PSI, CHI)
    assert abs(v["VALVOR"] + 4 * math.pi * g.ZLEN * PSI.LN) < 1e-13
    assert abs(v["VALZMO"] + 4 * math.pi * g.ZLEN * CHI.LN) < 1e-13
    ke, _, _ = D.boussi_energy(g, PSI, CHI, B, 1.0)
    assert abs(v["VALENE"] - 2 * ke.sum()) < 1e-12 * abs(v["VALENE"])
    assert v["NORM_CHECK"] == abs(PSI.E[1, 0, 0].imag + CHI.E[1, 0, 0].imag)
    assert g.NRCHOP == cfg.nrchop  # CHOPSET(3) undone
    bad = PSI.copy()
    bad.E[g.NRCHOPS[1], 1, 2] = 1e-9
    with pytest.raises(D.DiagnostError) as ei:
        D.diagnost(g, bad, CHI)
    assert ei.value.code == 11
    bad = PSI.copy()
    bad.E[3, 2, 1] = 150.0
    with pytest.raises(D.DiagnostError) as ei:
        D.diagnost(g, bad, CHI)
    assert ei.value.code == 12
    # CALCXY: the enstrophy of a Gaussian q-vortex at (xc, yc) with core R0 is
    # a Gaussian of variance R0^2/4 per axis, so <X> = xc, <Y> = yc and
    # <R>^2 = xc^2 + yc^2 + R0^2/2.
    from oracle import layout
    g = oracle_grid(small_cfg(64, 32, 32))
    psi, chi = layout.qvortex(g, xc=0.4, yc=-0.3)
    v = D.diagnost(g, psi, chi)
    assert abs(v["VALX"] - 0.4) < 1e-10 and abs(v["VALY"] + 0.3) < 1e-10
    assert abs(v["VALR"] - math.sqrt(0.4 ** 2 + 0.3 ** 2 + 0.5)) < 1e-10
    # two equal, well separated vortices: the enstrophy-weighted centre is their midpoint
    psi, chi = layout.qvortex_list(g, [layout.vortex(x=1.5, y=0.5), layout.vortex(x=-1.0, y=-0.5)])
    v = D.diagnost(g, psi, chi)
    assert abs(v["VALX"] - 0.25) < 1e-8 and abs(v["VALY"]) < 1e-8


def test_snapshot_record_layout(tmp_path):
    """MSAVEX / MPISAVEX restated: the record list and byte layout the
    reference's reader (tests/postproc/read_binary_info.ipynb) expects, and a
    round trip of both forms."""
    import struct
    from oracle import snapshot as S
    cfg = small_cfg(32, 16, 16)
    g = oracle_grid(cfg)
    A = random_fff(g, 9)
    A.LN = 0.125
    p = str(tmp_path / "a.dat")
    S.msave(p, g, A, glb=True)
    raw = open(p, "rb").read()
    assert struct.unpack("<iiiii", raw[:20]) == (12, g.NR, g.NTH, g.NX, 12)
    off = 20 + 20  # second record: chops
    assert struct.unpack("<iiiii", raw[20:40]) == (12, g.NRCHOP, g.NTCHOP, g.NXCHOP, 12)
    assert struct.unpack("<iidi", raw[off:off + 20]) == (12, A.space, A.LN, 12)
    E, sp, ln, hdr = S.mload(p, glb=True)
    assert sp == A.space and ln == A.LN and np.array_equal(E, A.E)
    assert hdr["minc"] == 1 and hdr["mklink"] == 0 and hdr["zlen"] == g.ZLEN
    q = str(tmp_path / "b.dat")
    S.msave(q, g, A, glb=False)
    assert len(open(q, "rb").read()) == A.E.size * 16
    E2, sp2, ln2, hdr2 = S.mload(q, glb=False, shape=A.E.shape)
    assert np.array_equal(E2, A.E) and sp2 == A.space and ln2 == A.LN
    assert hdr2["dims"] == (g.NDIMR, g.NDIMTH, g.NDIMX)


def test_sponge_profile_and_k0_kat():
    """CALC_BOUSSI_ETD_SPONGE restated: the damping is 1 in the middle of the
    axial domain, symmetric, and between exp(-DT/TAU) = exp(-0.1) and 1
    (TAU = 10 DT), strongest at the ends; a
    field with only k = 0 content keeps its k = 0 coefficients scaled by the
    z-average of the damping (the m = 0 modes real)."""
    from oracle import boussinesq as BQ
    cfg = small_cfg(32, 16, 16, adams=False, rmv_sw=2)
    g = oracle_grid(cfg)
    ph = oracle_physics(cfg)
    s = BQ.Solver.__new__(BQ.Solver)
    s.g, s.ph = g, ph
    z = g.Z[:g.NX] - g.ZLEN / 2.0
    hw, st = g.ZLEN * 0.86 / 2.0, g.ZLEN * 0.04
    damp = np.exp(-(1.0 - 0.5 * (np.tanh((z + hw) / st) - np.tanh((z - hw) / st))) / (10 * ph.dt) * ph.dt)
    assert abs(damp[g.NX // 2] - 1.0) < 1e-9
    assert (damp >= math.exp(-0.1)).all() and (damp <= 1.0).all()
    assert np.abs(damp[1:] - damp[1:][::-1]).max() < 1e-15      # symmetric about ZLEN/2
    assert damp[0] < 0.91                                        # damped at the ends
    B = random_fff(g, 12)
    B.E[:, :, 1:] = 0.0
    B.E[:, 0, 0] = B.E[:, 0, 0].real
    U = g.alloc()
    ref = B.E[:, :, 0].copy()
    s._etd_sponge(U, B, ph.dt)
    assert np.abs(B.E[:, :, 0] - damp.mean() * ref).max() < 1e-12 * np.abs(ref).max()
    assert np.abs(U.E).max() == 0.0


@pytest.mark.parametrize("P,nu,alp,fwd", [(4, 0.0, 3.0, 2e-9), (4, 0.7, -2.5, 5e-10), (6, 0.3, 5.0, 2e-7),
                                           (8, 0.0, -7.0, 5e-5), (8, 1e-3, 2e4, 1e-6)])
def test_ihelmp_known_answer(P, nu, alp, fwd):
    """IHELMP (mod_legops.f90:1409-1592) recovers a field from its image under
    (DEL^P + NU DEL^2 - ALP), the image formed independently with dense
    matrices: (D - k^2)^(P/2) + NU (D - k^2) - ALP for D the DEL2H band
    (mod_lin_legendre.f90:1986-2092) as a dense matrix, per (m, k), applied to
    coefficients supported on rows < NRCHOPS(m) - P (so the truncated band
    system reproduces them exactly), with the log term LN (-log(1-x)) whose
    DEL2 image is AL2 and whose DEL^P image is DEL2H^(P/2-1) AL2, and with
    CALCAT1 = 0 at m = 0 (the far-field fix then leaves row 0 alone).

    The unpivoted band LU is backward stable here: the residual of every
    (m, k) system is below 1e-14 of |H| |A|.  The forward error follows the
    conditioning of DEL^P - ALP (DEL2H's entries reach n^2 / ELL^2, so
    DEL^P's reach n^(2P)): bounded per case, from 2e-9 at P = 4 to 5e-5 at
    P = 8 with |ALP| of order one (1e-6 with ALP = 2e4, still far below
    DEL^8's largest entries)."""
    from oracle import legops as L
    from oracle.bandmat import band_del2h, band_to_full
    from oracle.grid import FFF
    g = oracle_grid(small_cfg(48, 16, 16))
    rng = np.random.default_rng(P)
    A0 = g.alloc(FFF)
    for mm in range(g.NTCHOPDIM):
        nn = int(g.NRCHOPS[mm])
        if nn - P > 0:
            sh = (nn - P, g.NXCHOPDIM)
            A0.E[: nn - P, mm, :] = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    A0.E[0, 0, :] -= g.calcat1(A0) / g.AT1[0]
    A0.LN = 0.3
    B = g.alloc(FFF)
    B.LN = -alp * A0.LN
    hp = P // 2
    H = {}
    for mm in range(g.NTCHOPDIM):
        nn = int(g.NRCHOPS[mm])
        if nn < 1:
            continue
        big = nn + 2 * P
        D = band_to_full(band_del2h(big, g.M[mm], g.ELL, g.LOGNORM[:, mm]), 2, big)
        for kk in range(g.NXCHOPDIM):
            k2 = g.AK[mm, kk] ** 2
            Dk = D - k2 * np.eye(big)
            H[mm, kk] = np.linalg.matrix_power(Dk, hp) + nu * Dk - alp * np.eye(big)
            x = np.zeros(big, dtype=complex)
            x[:nn] = A0.E[:nn, mm, kk]
            B.E[:nn, mm, kk] = (H[mm, kk] @ x)[:nn]
    n0 = g.NORM0
    al2 = np.zeros(g.NRCHOP)
    al2[:3] = A0.LN * np.array([(4.0 / 3 / g.ELL2) / n0[0], -2 / n0[1] / g.ELL2, (2.0 / 3) / n0[2] / g.ELL2])
    D0 = band_to_full(band_del2h(g.NRCHOP, g.M[0], g.ELL, g.LOGNORM[:, 0]), 2, g.NRCHOP)
    logpart = np.linalg.matrix_power(D0, hp - 1) @ al2 + nu * al2
    B.E[: g.NRCHOP, 0, 0] += logpart
    A = L.ihelmp(g, B, P, alp, nu)
    assert abs(A.LN - A0.LN) < 1e-14
    worst = 0.0
    for (mm, kk), Hm in H.items():
        nn = int(g.NRCHOPS[mm])
        rhs = B.E[:nn, mm, kk].copy()
        if mm == 0 and kk == 0:
            rhs -= logpart[:nn]
        a = A.E[:nn, mm, kk]
        Ht = Hm[:nn, :nn]
        res = np.abs(Ht @ a - rhs).max() / (np.abs(Ht).sum(axis=1).max() * np.abs(a).max())
        worst = max(worst, res)
    assert worst < 1e-14, worst
    assert rel(A.E, A0.E) < fwd
    # HYPERV is IHELMP(P, ALP A, A, -ALP, BET) with ALP = (-1)^(P/2)/(DT NUP)
    dt, nup = 1e-3, 0.05
    Hv = L.hyperv(g, A0.copy(), 1e-3, nup, P, dt)
    a = (-1) ** hp / dt / nup
    W = A0.copy()
    W.E, W.LN = a * A0.E, a * A0.LN
    R = L.ihelmp(g, W, P, -a, -(-1) ** hp * 1e-3 / nup)
    assert np.array_equal(Hv.E, R.E) and Hv.LN == R.LN
