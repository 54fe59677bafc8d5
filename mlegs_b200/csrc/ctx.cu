// Context, fields, operator composition, Boussinesq steppers and the C ABI.
//
// Host-side composition follows the reference routine by routine (file:line
// in each method's comment); the arithmetic runs in the kernels of
// tables.cu / kernels.cu / fft.cu / gemm.cu / solve.cu on one CUDA stream.
// Nothing here computes on the CPU except the FP64 set-up tables that the
// reference also builds once (LOGNORM, band-operator coefficients, ETD 4x4
// matrices, hyperviscosity masks).
#include "ctx_internal.h"

thread_local std::vector<void*>* mlegs_host::g_allocs = nullptr;

// ====================================================================== set-up
namespace {

// LEG_LOG_NORMT (mod_lin_legendre.f90:306-377) for MS = (0..ntchopdim-1).
std::vector<double> leg_log_norm(int ndim, int ntchopdim) {
    int me = ntchopdim - 1;
    std::vector<double> wk(me + 1);
    wk[0] = std::log(0.5);
    for (int m = 1; m <= me; ++m) wk[m] = wk[m - 1] + std::log(2 * m + 1.0) - std::log(2 * m * std::pow(2 * m - 1.0, 2));
    std::vector<double> out((size_t)ntchopdim * ndim);
    for (int m = 0; m < ntchopdim; ++m) {
        double* o = &out[(size_t)m * ndim];
        o[0] = wk[m];
        for (int nn = 2; nn <= ndim; ++nn) {
            int n = m + (nn - 1);
            o[nn - 1] = o[nn - 2] + std::log(2 * n + 1.0) - std::log(2 * n - 1.0) + std::log(1.0 * (n - m)) -
                        std::log(1.0 * (n + m));
        }
        for (int nn = 0; nn < ndim; ++nn) o[nn] = 0.5 * o[nn];
    }
    return out;
}

}  // namespace

// Band x band product in BANBANMUL's order (mod_bandmat.f90:1288-1345): C(r, k)
// accumulates A(r, i) B(r + i - ac, k - i) over i ascending; rows and columns
// outside [0, nn) are skipped.  Widths aw, bw; centres ac, bc (0-based).
static std::vector<double> banbanmul(const std::vector<double>& A, int aw, int ac, const std::vector<double>& B,
                                     int bw, int bc, int nn) {
    const int cw = aw + bw - 1;
    std::vector<double> C((size_t)nn * cw, 0.0);
    for (int i = 0; i < aw; ++i) {
        const int as = i - ac;
        for (int j = 0; j < bw; ++j) {
            const int k = i + j, bs = j - bc;
            for (int r = 0; r < nn; ++r) {
                const int rb = r + as;  // row of B = column of A
                if (rb < 0 || rb >= nn || rb + bs < 0 || rb + bs >= nn) continue;
                C[(size_t)r * cw + k] += A[(size_t)r * aw + i] * B[(size_t)rb * bw + j];
            }
        }
    }
    return C;
}

const double* mlegs_ctx::helmp_tables(int P) {
    for (const auto& t : helmp_tab)
        if (t.first == P) return t.second;
    no_capture("IHELMP");
    const int HP = P / 2, rows = helmp_rows();
    // DEL2H rows i < rows + P - 2 (BAND_LOGLEG_RAT_DEL2H with S = 0, mod_lin_legendre.f90:1986-2092):
    // the powers' rows below `rows` are then those of the untruncated operator
    const int nd = std::min(rows + P - 2, d.NLN - 2);
    const size_t per_m = (size_t)rows * HP * (2 * HP + 3);  // rows * sum_{q <= HP} (4q + 1)
    std::vector<double> h((size_t)d.NTCHOPDIM * per_m, 0.0);
    for (int m = 0; m < d.NTCHOPDIM; ++m) {
        const double* ln = &h_lognorm[(size_t)m * d.NLN];
        const double am = m, e2 = d.ELL2;
        auto ex = [&](int a, int b2) { return std::exp(ln[a] - ln[b2]); };
        std::vector<double> D((size_t)nd * 5, 0.0);
        for (int nn = 0; nn < nd; ++nn) {
            const double N = am + nn;
            double* db = &D[(size_t)nn * 5];
            if (nn >= 2)
                db[0] = -(N - am - 1.0) * (N - am) * (N - 2) * (N - 1) / (2 * N - 3.) / (2 * N - 1.0) / e2 *
                        ex(nn - 2, nn);
            if (nn >= 1) db[1] = 2.0 * N * (N - am) * (N - 1) / (2 * N - 1.0) / e2 * ex(nn - 1, nn);
            db[2] = (-2.0 * N * (N + 1.0) * (3.0 * N * N + 3 * N - am * am - 2)) / (2 * N - 1.0) / (2 * N + 3.0) / e2;
            db[3] = 2.0 * (N + 1) * (N + am + 1.0) * (N + 2) / (2 * N + 3.0) / e2 * ex(nn + 1, nn);
            db[4] = -(N + am + 1.0) * (N + am + 2.0) * (N + 3) * (N + 2) / (2 * N + 3.0) / (2 * N + 5.0) / e2 *
                    ex(nn + 2, nn);
        }
        std::vector<double> Dq = D;
        for (int q = 1; q <= HP; ++q) {
            const int w = 4 * q + 1;
            if (q > 1) Dq = banbanmul(Dq, 4 * q - 3, 2 * q - 2, D, 5, 2, nd);  // D^q = D^(q-1) D
            double* out = &h[(size_t)m * per_m + (size_t)rows * (q - 1) * (2 * q + 1)];
            for (int r = 0; r < rows && r < nd; ++r)
                for (int e = 0; e < w; ++e) out[(size_t)r * w + e] = Dq[(size_t)r * w + e];
        }
    }
    double* dp = dalloc<double>(h.size());
    CK(cudaMemcpyAsync(dp, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    helmp_tab.emplace_back(P, dp);
    return dp;
}

void mlegs_ctx::init(const mlegs_params& prm) {
    p = prm;
    if (p.nr < 4 || p.nth < 2 || p.nx < 2 || p.nrchop < 1 || p.ntchop < 1 || p.nxchop < 1)
        throw ApiError(MLEGS_ERR_ARG, "bad dimensions");
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    if (!pow2(p.nth) || !pow2(p.nx)) throw ApiError(MLEGS_ERR_ARG, "NTH and NX must be powers of two");
    if (p.nr % 2) throw ApiError(MLEGS_ERR_ARG, "NR must be even");
    if (2 * p.nxchop > p.nx) throw ApiError(MLEGS_ERR_ARG, "NXCHOP MUST BE < NX/2");  // mod_fft.f90:237-243
    dev = p.device;
    CK(cudaSetDevice(dev));
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    for (cudaEvent_t& e : evs) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    g_launch_counter = &launches;
    fft_set_attributes();
    phys_set_attributes();

    d.NR = p.nr;
    d.NRH = p.nr / 2;
    d.NTH = p.nth;
    d.NX = p.nx;
    d.NRCHOP = p.nrchop;
    d.NTCHOP = p.ntchop;
    d.NXCHOP = p.nxchop;
    d.NDIMR = p.nr + 3;
    d.NDIMTH = p.nth + 1;
    d.NRCHOPDIM = std::min(p.nrchop + 6, p.nr);
    d.NTCHOPDIM = std::min(p.ntchop, p.nth);
    d.NXCHOPDIM = 2 * p.nxchop - 1;
    d.NXCHOPH = p.nx - p.nxchop + 2;
    d.NLN = d.NRCHOPDIM + 14;
    d.ELL = p.ell;
    d.ELL2 = std::pow(p.ell, 2.0);
    d.ZLEN = p.zlen;
    if (d.NRCHOP > d.NRCHOPDIM) throw ApiError(MLEGS_ERR_ARG, "NRCHOP > NRCHOPDIM");
    const int NB = d.NRCHOPDIM + 2;

    // --- Gauss-Legendre nodes and weights on the device (FP64 Newton)
    x = dalloc<double>(d.NR);
    w = dalloc<double>(d.NR);
    k_tables_gauss(x, w, d.NR, s);
    h_x.resize(d.NR);
    h_w.resize(d.NR);
    CK(cudaMemcpyAsync(h_x.data(), x, d.NR * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h_w.data(), w, d.NR * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<double> h_r(d.NR), h_lnx(d.NR);
    for (int i = 0; i < d.NR; ++i) {
        h_r[i] = d.ELL * std::sqrt((1 + h_x[i]) / (1 - h_x[i]));  // LEG_ZERO, mod_lin_legendre.f90:172
        h_lnx[i] = -std::log(1 - h_x[i]);                          // TFM%LN, mod_fft.f90:287
    }
    r = dalloc<double>(d.NR);
    lnx = dalloc<double>(d.NR);
    CK(cudaMemcpyAsync(r, h_r.data(), d.NR * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(lnx, h_lnx.data(), d.NR * sizeof(double), cudaMemcpyHostToDevice, s));

    // --- orthonormal P^m_n table on the device
    const int ne = d.NRCHOPDIM + 1;
    pf = dalloc<double>((size_t)d.NTCHOPDIM * ne * d.NRH);
    k_tables_pf(x, pf, d.NRH, ne, d.NTCHOPDIM, s);

    // --- LOGNORM, NORM(:,m=0), AT1, AK, band coefficients (host FP64)
    h_lognorm = leg_log_norm(d.NLN, d.NTCHOPDIM);
    std::vector<double> h_norm0(d.NLN), h_explog0(d.NLN), h_at1(d.NRCHOPDIM), h_ak(d.NXCHOPDIM);
    {
        double v = 0.5;  // LEG_NORMT, m = 0 (mod_lin_legendre.f90:246-270)
        h_norm0[0] = std::sqrt(v);
        for (int nn = 2; nn <= d.NLN; ++nn) {
            int nv = nn - 1;
            v = v * (2 * nv + 1.0) / (2 * nv - 1.0) * nv / nv;
            h_norm0[nn - 1] = std::sqrt(v);
        }
    }
    for (int nn = 0; nn < d.NLN; ++nn) h_explog0[nn] = std::exp(h_lognorm[nn]);
    for (int nn = 0; nn < d.NRCHOPDIM; ++nn) h_at1[nn] = std::sqrt((2 * nn + 1) / 2.0);
    for (int kk = 0; kk < d.NXCHOPDIM; ++kk) {
        int kv = kk;
        if (kk + 1 > d.NXCHOP) kv = -(d.NXCHOPDIM - (kk + 1) + 1);
        h_ak[kk] = 2 * M_PI / d.ZLEN * kv;  // mod_fft.f90:255-263
    }
    std::vector<double> h_xxdx((size_t)d.NTCHOPDIM * NB * 2, 0.0), h_xm((size_t)d.NTCHOPDIM * NB * 2, 0.0),
        h_del2h((size_t)d.NTCHOPDIM * NB * 5, 0.0);
    for (int m = 0; m < d.NTCHOPDIM; ++m) {
        const double* ln = &h_lognorm[(size_t)m * d.NLN];
        const double am = m;
        for (int nn = 0; nn < NB; ++nn) {
            const double N = am + nn;
            auto ex = [&](int a, int b2) { return std::exp(ln[a] - ln[b2]); };
            double* xb = &h_xxdx[((size_t)m * NB + nn) * 2];
            double* mb = &h_xm[((size_t)m * NB + nn) * 2];
            double* db = &h_del2h[((size_t)m * NB + nn) * 5];
            // BAND_LOGLEG_XXDX (1683-1757) and BAND_LOGLEG_XM (910-981)
            if (nn >= 1) {
                xb[0] = -(N - 1.0) * (N - am) / (2 * N - 1.0) * ex(nn - 1, nn);
                mb[0] = -(N - am) / (2 * N - 1.0) * ex(nn - 1, nn);
            }
            xb[1] = (N + 2.0) * (N + am + 1.0) / (2 * N + 3.0) * ex(nn + 1, nn);
            mb[1] = -(N + am + 1.0) / (2 * N + 3.0) * ex(nn + 1, nn);
            // BAND_LOGLEG_RAT_DEL2H with S = 0 (1986-2092)
            const double e2 = d.ELL2;
            if (nn >= 2)
                db[0] = -(N - am - 1.0) * (N - am) * (N - 2) * (N - 1) / (2 * N - 3.) / (2 * N - 1.0) / e2 *
                        ex(nn - 2, nn);
            if (nn >= 1) db[1] = 2.0 * N * (N - am) * (N - 1) / (2 * N - 1.0) / e2 * ex(nn - 1, nn);
            db[2] = (-2.0 * N * (N + 1.0) * (3.0 * N * N + 3 * N - am * am - 2)) / (2 * N - 1.0) / (2 * N + 3.0) / e2;
            db[3] = 2.0 * (N + 1) * (N + am + 1.0) * (N + 2) / (2 * N + 3.0) / e2 * ex(nn + 1, nn);
            db[4] = -(N + am + 1.0) * (N + am + 2.0) * (N + 3) * (N + 2) / (2 * N + 3.0) / (2 * N + 5.0) / e2 *
                    ex(nn + 2, nn);
        }
    }
    auto up = [&](const std::vector<double>& h) {
        double* dp = dalloc<double>(h.size());
        CK(cudaMemcpyAsync(dp, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        return dp;
    };
    norm0 = up(h_norm0);
    explog0 = up(h_explog0);
    at1 = up(h_at1);
    ak = up(h_ak);
    tb_xxdx = up(h_xxdx);
    tb_xm = up(h_xm);
    tb_del2h = up(h_del2h);

    g.NR = d.NR;
    g.NRH = d.NRH;
    g.NTH = d.NTH;
    g.NX = d.NX;
    g.NRCHOP = d.NRCHOP;
    g.NTCHOP = d.NTCHOP;
    g.NXCHOP = d.NXCHOP;
    g.NRCHOPDIM = d.NRCHOPDIM;
    g.NTCHOPDIM = d.NTCHOPDIM;
    g.NXCHOPDIM = d.NXCHOPDIM;
    g.NLN = d.NLN;
    g.ELL2 = d.ELL2;
    g.x = x;
    g.w = w;
    g.r = r;
    g.lnx = lnx;
    g.pf = pf;
    g.ak = ak;
    g.norm0 = norm0;
    g.at1 = at1;
    g.xxdx = tb_xxdx;
    g.xm = tb_xm;
    g.del2h = tb_del2h;
    g.NB = NB;

    // --- PROJECT weights (device, from PF)
    size_t vsz = (size_t)d.NTCHOPDIM * d.NRCHOPDIM * d.NRH;
    V = dalloc<double>(vsz);
    D = dalloc<double>(vsz);
    T = dalloc<double>(vsz);
    k_tables_project(g, V, D, T, 0, s);
    diag = dalloc<double>((size_t)4 * d.NTCHOPDIM * d.NXCHOPDIM);
    if (p.rmv_sw == 2 && !p.adams) {
        // SPNGINIT (mod_march.f90:2292-2323): N_TAU = 10, RATIO_L = 0.86,
        // RATIO_S = 0.04; T(z) = TOPHAT(Z - ZLEN/2, ZLEN RATIO_L/2, ZLEN RATIO_S)
        // (3704-3712); the damping over DT is exp(-(1 - T(z))/TAU DT), TAU = N_TAU DT
        const double hw = p.zlen * 0.86 / 2.0, st = p.zlen * 0.04, tau = 10 * p.dt;
        auto damp = [&](double dt) {
            std::vector<double> h(d.NX);
            for (int q = 0; q < d.NX; ++q) {
                const double z = p.zlen * q / d.NX - p.zlen / 2.0;
                const double th = 0.5 * (std::tanh((z + hw) / st) - std::tanh((z - hw) / st));
                h[q] = std::exp(-(1.0 - th) / tau * dt);
            }
            return up(h);
        };
        sp_damp = damp(p.dt);
        sp_damp_h = damp(p.dt * 0.5);
    }
    v2p_pff = dalloc<double>(d.NR);
    v2p_fff = dalloc<double>(std::max(d.NRCHOP, 1));
    k_vel2pln_coef(g, explog0, d.NRCHOP, v2p_pff, v2p_fff, s);
    if (p.precision == MLEGS_PREC_FP64 && dmma_supported(g)) {
        const size_t nc = proj_comp_doubles(g);
        compV = dalloc<double>(nc);
        compD = dalloc<double>(nc);
        compT = dalloc<double>(nc);
        k_proj_comp(g, V, 0, compV, s);
        k_proj_comp(g, D, 1, compD, s);
        k_proj_comp(g, T, 0, compT, s);
    }
    if (p.precision == MLEGS_PREC_FP64 && fold_bulk_supported(g, d.NRCHOPDIM + 1)) {
        fc_pf = dalloc<double>(fold_table_doubles(g, d.NRCHOPDIM + 1));
        k_fold_table(g, pf, d.NRCHOPDIM + 1, 1, fc_pf, s);
        double** fcs[3] = {&fc_V, &fc_D, &fc_T};
        const double* W[3] = {V, D, T};
        for (int q = 0; q < 3; ++q) {
            *fcs[q] = dalloc<double>(fold_table_doubles(g, d.NRCHOPDIM));
            k_fold_table(g, W[q], d.NRCHOPDIM, 0, *fcs[q], s);
        }
    }

    // --- FFT twiddles (host long double, rounded once)
    auto lg2 = [](int v) { int l = 0; while ((1 << l) < v) ++l; return l; };
    fft.lx = lg2(d.NX);
    fft.lt = lg2(d.NTH);
    auto twid = [&](int N, double scale) {
        std::vector<double2> h(N + 1);
        for (int q = 0; q <= N; ++q) {
            long double a = -(long double)scale * 3.141592653589793238462643383279502884L * q / N;
            h[q] = make_double2((double)std::cos(a), (double)std::sin(a));
        }
        double2* dp = dalloc<double2>(N + 1);
        CK(cudaMemcpyAsync(dp, h.data(), (N + 1) * sizeof(double2), cudaMemcpyHostToDevice, s));
        return dp;
    };
    fft.tw_x = twid(d.NX, 2.0);
    fft.tw_t = twid(d.NTH, 2.0);
    fft.tw_h = twid(d.NTH, 1.0);

    // --- VISC%SW = 2: HYPERV / IHELMP (AB2-CN only; SOLVER_T%INITIALIZE aborts for ETD,
    //     mod_march.f90:189-201)
    if (p.visc_sw == 2) {
        if (!p.adams)
            throw ApiError(MLEGS_ERR_SOLVER, "SOLVER: ETD scheme MUST use velocity-based hyperviscosity.");
        if (p.visc_p < 4 || p.visc_p > 14 || p.visc_p % 2)
            throw ApiError(MLEGS_ERR_ARG, "HYPERV: VISC%P must be even, 4..14, for VISC%SW = 2");
        if (p.nup == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "HYPERV: NUP CAN'T BE ZERO");
    }
    // --- hyperviscosity (HYP3SET, mod_march.f90:3320-3408)
    if (p.visc_sw == 3) {
        auto mask = [](const std::vector<double>& kv, size_t size, double ratio, double steep) {
            std::vector<double> out(size, 1.0);
            double kmax = -1e300;
            for (double v : kv) kmax = std::max(kmax, v);
            if (kv.empty() || kmax < 1e-12) kmax = 1.0;
            double ta = std::tanh(steep);
            for (size_t i = 0; i < kv.size(); ++i) {
                double kn = kv[i] / kmax;
                if (kn < ratio) out[i] = 0.0;
                else {
                    double xr = (kn - ratio) / (1.0 - ratio), yr = steep * (2.0 * xr - 1.0);
                    out[i] = (std::tanh(yr) + ta) / (2.0 * ta);
                }
            }
            return out;
        };
        const int nrc = d.NRCHOP;
        std::vector<double> mr((size_t)nrc * d.NTCHOPDIM), mt, mx;
        for (int m = 0; m < d.NTCHOPDIM; ++m) {
            int nrs = std::max(d.NRCHOP - m, 0);
            std::vector<double> kv(nrs);
            for (int q = 0; q < nrs; ++q) kv[q] = q;
            auto mm = mask(kv, nrc, 0.5, 2.0);
            for (int q = 0; q < nrc; ++q) mr[(size_t)m * nrc + q] = mm[q];
        }
        {
            std::vector<double> kv(d.NTCHOPDIM);
            for (int m = 0; m < d.NTCHOPDIM; ++m) kv[m] = m;
            mt = mask(kv, d.NTCHOPDIM, 2.0 / 3.0, 2.0);
            std::vector<double> kx(d.NXCHOPDIM);
            for (int q = 0; q < d.NXCHOPDIM; ++q) kx[q] = std::fabs(h_ak[q]);
            mx = mask(kx, d.NXCHOPDIM, 2.0 / 3.0, 2.0);
        }
        h3_mr = mr;
        h3_mt = mt;
        h3_mx = mx;
        h3_ak = h_ak;
        // HYP3INIT (3464-3480)
        for (int q = 0; q < 3; ++q) {
            nup3[q] = p.nup;
            kap3[q] = p.kappap;
        }
        hyp3set(nup3, hv);
        hyp3set(kap3, hd);
    }

    // --- ETD operators (CALC_BOUSSI_ETD_OP, mod_march.f90:906-945; host FP64)
    if (!p.adams) {
        if (p.bv0 == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "CALC_BOUSSI_DIAG: N_FREQ = 0, CANNOT DIAGONALIZE");
        typedef std::complex<double> C;
        const C I(0.0, 1.0);
        auto etd = [&](double dt, double** Eo, double** No) {
            C J[4] = {-I * p.bv0, I * p.bv0, -2.0 * I * p.omega, 2.0 * I * p.omega};
            C S[4][4] = {}, Si[4][4] = {};
            S[0][2] = I; S[0][3] = -I; S[1][2] = 1.0; S[1][3] = 1.0;
            S[2][0] = -I / p.bv0; S[2][1] = I / p.bv0; S[3][0] = 1.0; S[3][1] = 1.0;
            Si[0][2] = I * p.bv0 / 2.0; Si[0][3] = 0.5; Si[1][2] = -I * p.bv0 / 2.0; Si[1][3] = 0.5;
            Si[2][0] = -I / 2.0; Si[2][1] = 0.5; Si[3][0] = I / 2.0; Si[3][1] = 0.5;
            C je[4], jp[4];
            for (int q = 0; q < 4; ++q) {
                je[q] = std::exp(J[q] * dt);
                jp[q] = (std::abs(J[q]) > 1e-14) ? (je[q] - 1.0) / J[q] : C(dt);
            }
            std::vector<double> e(16), nl(16);
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) {
                    C a = 0.0, b2 = 0.0;
                    for (int q = 0; q < 4; ++q) {
                        a += S[i][q] * je[q] * Si[q][j];
                        b2 += S[i][q] * jp[q] * Si[q][j];
                    }
                    e[i * 4 + j] = a.real();
                    nl[i * 4 + j] = b2.real();
                }
            *Eo = up(e);
            *No = up(nl);
        };
        etd(p.dt, &etdE, &etdN);
        etd(p.dt * 0.5, &hetdE, &hetdN);
    }

    // --- memory: LN slots, scratch buffers, temporaries, history
    nslots = 512;
    lnslots = dalloc<double>(nslots);
    CK(cudaMemsetAsync(lnslots, 0, nslots * sizeof(double), s));
    scratch = dalloc<double2>(d.cap());
    for (double2*& q : pbuf) q = dalloc<double2>(d.cap());
    size_t nsys = (size_t)d.NTCHOPDIM * d.NXCHOPDIM;
    solve_scr = dalloc<double>((size_t)d.NRCHOPDIM * 4 * nsys);
    size_t ref_max = (size_t)d.NDIMR * d.NDIMTH * d.NX;
    size_t ref_fff = (size_t)d.NRCHOPDIM * d.NTCHOPDIM * d.NXCHOPDIM;
    size_t ref_pff = (size_t)d.NDIMR * d.NTCHOPDIM * d.NXCHOPDIM;
    staging = dalloc<double2>(std::max(ref_max, std::max(ref_fff, ref_pff)));
    dflag = dalloc<int>(1);
    split_err = dalloc<int>(1);
    CK(cudaMemsetAsync(split_err, 0, sizeof(int), s));
    if (p.precision == MLEGS_PREC_SPLIT) {
        const int S = p.split_slices > 0 ? p.split_slices : 6;
        if (!split_supported(g, S, d.NRCHOPDIM + 1))
            throw ApiError(MLEGS_ERR_ARG, "MLEGS_PREC_SPLIT: needs 3 <= split_slices <= 6, NR <= 256 and the "
                                          "slice stages within 227 KB of shared memory");
        split_S = S;
        split_img = dalloc<uint8_t>(split_image_bytes(g, S, 0, 0));
        split_eA = dalloc<int>((size_t)d.NTCHOPDIM * 2 * 128);
        k_split_prepare(g, S, 0, pf, 0, split_img, split_eA, s);
        const double* W[4] = {pf, V, D, T};
        const int rows[4] = {d.NRCHOPDIM + 1, d.NRCHOPDIM, d.NRCHOPDIM, d.NRCHOPDIM};
        for (int q = 0; q < 4; ++q) {
            fimg[q] = dalloc<uint8_t>(split_image_bytes(g, S, 1, rows[q]));
            feA[q] = dalloc<int>((size_t)d.NTCHOPDIM * 2 * 128);
            k_split_prepare(g, S, 1, W[q], rows[q], fimg[q], feA[q], s);
        }
    } else if (p.precision != MLEGS_PREC_FP64) {
        throw ApiError(MLEGS_ERR_ARG, "unknown precision");
    }
    for (int q = 0; q < 24; ++q) {
        Field* f = new_field(MLEGS_FFF, false);
        temps.push_back(f);
        pool.push_back(f);
    }
    for (int q = 0; q < 7; ++q) hist[q] = new_field(MLEGS_FFF, true);
    if (p.visc_sw == 2) {  // IHELMP tables and scratch before any step graph is captured
        helmp_tables(p.visc_p);
        helmp_scratch(p.visc_p);
    }
    CK(cudaStreamSynchronize(s));
}

void mlegs_ctx::destroy() {
    if (gexec) cudaGraphExecDestroy(gexec);
    for (AdjGraph& a : adj_g)
        if (a.exec) cudaGraphExecDestroy(a.exec);
    if (graph) cudaGraphDestroy(graph);
    for (void* q : allocs) cudaFree(q);
    allocs.clear();
    for (cudaEvent_t& e : evs)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : io_ev)
        if (e) cudaEventDestroy(e);
    if (io_ln) cudaFreeHost(io_ln);
    io_ln = nullptr;
    if (s_up) cudaStreamDestroy(s_up);
    if (s_down) cudaStreamDestroy(s_down);
    s_up = s_down = nullptr;
    if (s2) cudaStreamDestroy(s2);
    s2 = nullptr;
    if (s) cudaStreamDestroy(s);
    s = nullptr;
}

__global__ void ln_from_coef_kernel(double* ln, const double2* data, double n0, double scale) {
    *ln = data[0].x * n0 * scale;
}
void mlegs_ctx::ln_from_coef(double* ln, const double2* data, double scale) {
    // IDELSQH: A%LN = B%E(1,1,1) * NORM(1,1) * ELL2  (mod_legops.f90:207)
    double v0 = std::sqrt(0.5);
    ln_from_coef_kernel<<<1, 1, 0, s>>>(ln, data, v0, scale);
    count_launch();
}

// ====================================================================== physics
// CALC_BOUSSI_FORCE(PSI, CHI, B, PSIN, CHIN, BN), mod_boussinesq.f90:317-410.
void mlegs_ctx::force(const Field* PSI, const Field* CHI, const Field* B, Field* PSIN, Field* CHIN, Field* BNout) {
    Field *RUR = tmp(), *RUP = tmp(), *UZ = tmp(), *ROR = tmp(), *ROP = tmp(), *OZ = tmp(), *RBR = tmp(),
          *RBP = tmp(), *BZ = tmp(), *W = tmp();
    const int P3 = 3;  // CHOPSET(3) ... CHOPSET(-3)
    grad(B, RBR, RBP, BZ, P3);
    pc2vel(PSI, CHI, RUR, RUP, UZ, P3);
    pc2vor(PSI, CHI, ROR, ROP, OZ, P3);
    copy0(W, B, 0);  // W = B; TOFP(W) after CHOPSET(-3)
    // TOFP up to PFP; the HORFFT(+1) of each field happens inside the fused kernel
    {
        Field* const fs[10] = {RUR, RUP, UZ, ROR, ROP, OZ, RBR, RBP, BZ, W};
        const int pads[10] = {P3, P3, P3, P3, P3, P3, P3, P3, P3, 0};
        tofp_pipe(fs, pads, 10);
    }
    // VPRODSUB + VDOTPSUB + the linear terms (385-391), then HORFFT(-1) of the results
    Field *NR = tmp(), *NP = tmp(), *NZ = tmp(), *BN = tmp();
    const double2* in[10] = {RUR->data, RUP->data, UZ->data, ROR->data, ROP->data,
                             OZ->data,  RBR->data, RBP->data, BZ->data,  W->data};
    double2* out[4] = {NR->data, NP->data, NZ->data, BN->data};
    k_theta_fused(g, fft, in, out, p.omega, p.bv0, 1, s);
    for (Field* f : {NR, NP, NZ, BN}) {
        f->space = MLEGS_PFP;
        ln_zero(f);
    }
    for (Field* f : {RUR, RUP, UZ, ROR, ROP, OZ, RBR, RBP, BZ, W}) rel(f);
    Field* Wf = tmp();  // W = DEL2(CHIN) in FFF
    project(NR, NP, NZ, PSIN, Wf, 1, 0.0);
    idel2ln(Wf, CHIN, 0);
    toff(BN, 0);
    copy0(BNout, BN, 0);
    for (Field* f : {Wf, NR, NP, NZ, BN}) rel(f);
}

// *_MK_HALFK (mod_scalar3.f90:528-554, 808-841) of an [m][k] quadrature array:
// the m = 0 row halved (the ALLK forms, 523 and 803), then k and -k folded into
// out(m, k), k < NXCHOP, Fortran order (NTCHOP x NXCHOP); out (+)= sign * that.
void mlegs_ctx::halfk(const double* all, double sign, double* out, bool accumulate) const {
    const int nt = d.NTCHOPDIM, nk = d.NXCHOPDIM;
    for (int kk = 0; kk < d.NXCHOP; ++kk)
        for (int mm = 0; mm < d.NTCHOP; ++mm) {
            double v = 0.0;
            if (mm < nt) {
                const double h = mm == 0 ? 0.5 : 1.0;
                const double a = h * all[(size_t)mm * nk + kk];
                v = kk == 0 ? a : h * all[(size_t)mm * nk + (nk - kk)] + a;
            }
            double& o = out[(size_t)kk * d.NTCHOP + mm];
            o = accumulate ? o + sign * v : sign * v;
        }
}

// CALC_BOUSSI_ENERGY(PSI, CHI, B), mod_boussinesq.f90:139-232, without the
// file output: KE, PE and DKE per (m >= 0, k >= 0), NTCHOP x NXCHOP each
// (Fortran order); the driver's especData sums are their row / column sums.
void mlegs_ctx::energy(const Field* PSI, const Field* CHI, const Field* B, double* ke, double* pe, double* dke) {
    require(PSI, MLEGS_FFF, "CALC_BOUSSI_ENERGY");
    require(CHI, MLEGS_FFF, "CALC_BOUSSI_ENERGY");
    require(B, MLEGS_FFF, "CALC_BOUSSI_ENERGY");
    double bln = 0.0;
    CK(cudaMemcpyAsync(&bln, B->ln, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (bln != 0.0)
        throw ApiError(MLEGS_ERR_LOGTERM, "B has non-zero LN, this is not expected in Boussinesq");
    if (p.bv0 == 0.0) throw ApiError(MLEGS_ERR_ARG, "CALC_BOUSSI_ENERGY: BV0 = 0");
    const int P3 = 3;  // CHOPSET(3) ... CHOPSET(-3)
    const size_t nmk = (size_t)d.NTCHOPDIM * d.NXCHOPDIM;
    const double scale = 4.0 * 3.141592653589793238462643383279502884 * p.zlen * d.ELL2;
    Field *W1 = tmp(), *W2 = tmp(), *W3 = tmp();
    // toroidal: W1 = PSI (LN doubled), W2 = DELSQH(W1); -PRODCT(RTRAN W1, RTRAN W2)
    copy0(W1, PSI, P3);
    k_ln_copy(W1->ln, PSI->ln, 2.0, s);
    delsqh(W1, W2, P3);
    ln_zero(W1);
    ln_zero(W2);
    rtran(W1, 1, P3);
    rtran(W2, 1, P3);
    k_prodct_mk(g, W1->data, W2->data, 0, scale, diag, s);
    // poloidal: W1 = DEL2(CHI), W2 = DELSQH(CHI)
    del2(CHI, W1, P3);
    delsqh(CHI, W2, P3);
    ln_zero(W1);
    ln_zero(W2);
    rtran(W1, 1, P3);
    rtran(W2, 1, P3);
    k_prodct_mk(g, W1->data, W2->data, 0, scale, diag + nmk, s);
    // exchange and potential energy from W3 = B
    copy0(W3, B, P3);
    ln_zero(W3);
    rtran(W3, 1, P3);
    k_prodct_mk(g, W3->data, W2->data, 0, scale, diag + 2 * nmk, s);
    k_prodct_mk(g, W3->data, nullptr, 1, scale, diag + 3 * nmk, s);
    rel(W3);
    rel(W2);
    rel(W1);
    std::vector<double> h(4 * nmk);
    CK(cudaMemcpyAsync(h.data(), diag, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const size_t nout = (size_t)d.NTCHOP * d.NXCHOP;
    std::vector<double> kev(nout);
    halfk(h.data(), -1.0, kev.data(), false);
    halfk(h.data() + nmk, 1.0, kev.data(), true);
    for (double& v : kev) v /= 2.0;
    if (ke) std::copy(kev.begin(), kev.end(), ke);
    if (dke) halfk(h.data() + 2 * nmk, 1.0, dke, false);
    if (pe) {
        halfk(h.data() + 3 * nmk, 1.0, pe, false);
        for (size_t q = 0; q < nout; ++q) pe[q] = pe[q] / 2.0 / (p.bv0 * p.bv0);
    }
}

// DIAGNOST(PSI, CHI), mod_march.f90:1689-1966, without the printing and the
// stored initial values: the norm, dealiasing and divergence checks
// (1726-1787) and, under CHOPSET(3), VALVOR = INTEG(OZH), VALZMO = INTEG(UZH)
// (OZH, UZH the 'H' forms -DELSQH(PSI), -DELSQH(CHI) of PC2VOR/PC2VEL),
// VALANG = -INTEG_P(XXDX(PSI with LN 0)), VALENE = -ENE1 + ENE2, VALHEL, the
// spread of CALCAT1(PSI), CALCAT1(CHI) over k, and CALCXY's enstrophy-weighted
// <X>, <Y>, <R>.  INTEG_P (3649-3682) reads F%E(:NR,1,1) of its FFF argument,
// whose first dimension is NRCHOPDIM < NR; the RTRAN(+1) image F_COPY that it
// forms is used here instead.
// out: VALVOR, VALZMO, VALANG, VALENE, VALHEL, PAT1MAX-PAT1MIN, CAT1MAX-CAT1MIN,
// |Im PSI(2,1,1) + Im CHI(2,1,1)| (the norm check's quantity), <X>, <Y>, <R>.
void mlegs_ctx::diagnost(const Field* PSI, const Field* CHI, double out[11]) {
    require(PSI, MLEGS_FFF, "DIAGNOST");
    require(CHI, MLEGS_FFF, "DIAGNOST");
    const int nk = d.NXCHOPDIM, nrd = d.NRCHOPDIM;
    const size_t slab = (size_t)nrd * nk;
    const int mm6 = std::min(6, d.NTCHOPDIM);
    std::vector<double2> ps((size_t)mm6 * slab), cs(slab);
    double lnp = 0.0, lnc = 0.0;
    CK(cudaMemcpyAsync(ps.data(), PSI->data, ps.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(cs.data(), CHI->data, cs.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&lnp, PSI->ln, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&lnc, CHI->ln, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    auto at = [&](const std::vector<double2>& v, int m, int n, int k) { return v[((size_t)m * nrd + n) * nk + k]; };
    auto nrchops = [&](int m, int pad) { return std::max(std::min(d.NRCHOP + pad, d.NRCHOP + pad - m), 0); };
    out[7] = (nrd > 1) ? std::fabs(at(ps, 0, 1, 0).y + at(cs, 0, 1, 0).y) : 0.0;
    // dealiasing check: radial modes past NRCHOPS of m = 0, 1 must be zero
    double chk = 0.0;
    for (int mm = 0; mm < std::min(2, d.NTCHOPDIM); ++mm) {
        double mx = 0.0;
        for (int n = nrchops(mm, 0); n < nrd; ++n)
            for (int k = 0; k < nk; ++k) mx = std::max(mx, std::hypot(at(ps, mm, n, k).x, at(ps, mm, n, k).y));
        chk += mx;
    }
    if (chk > 1.0e-12) throw ApiError(MLEGS_ERR_DEALIASING, "DIAG: DEALIASING INCOMPLETE");
    // divergence check on the first coefficients
    for (int kk = 0; kk < std::min(5, nk); ++kk)
        for (int mm = 1; mm < mm6; ++mm)
            for (int n = 0; n < std::min(5, d.NRCHOP); ++n)
                if (std::hypot(at(ps, mm, n, kk).x, at(ps, mm, n, kk).y) > 100.0)
                    throw ApiError(MLEGS_ERR_DIVERGENCE, "DIAG: DIVERGENCE");
    const int P3 = 3;  // CHOPSET(3) ... CHOPSET(-3)
    const double pi = 3.141592653589793238462643383279502884;
    const double n00 = std::sqrt(0.5);  // TFM%NORM(1,1)
    auto coef000 = [&](const Field* f) {
        double2 v;
        CK(cudaMemcpyAsync(&v, f->data, sizeof(double2), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return v.x;
    };
    const size_t nmk = (size_t)d.NTCHOPDIM * nk;
    const double scale = 4.0 * pi * p.zlen * d.ELL2;
    auto prodct = [&](const Field* A, const Field* B) {  // PRODCT: the sum of the halved ALLK array
        k_prodct_mk(g, A->data, B->data, 0, scale, diag, s);
        std::vector<double> h(nmk);
        CK(cudaMemcpyAsync(h.data(), diag, nmk * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double sum = 0.0;
        for (size_t q = 0; q < nmk; ++q) sum += (q < (size_t)nk ? 0.5 : 1.0) * h[q];
        return sum;
    };
    Field *W1 = tmp(), *W2 = tmp(), *W3 = tmp();
    // VALVOR = INTEG(-DELSQH(PSI)), VALZMO = INTEG(-DELSQH(CHI)) (INTEG, mod_scalar3.f90:312-353)
    delsqh(PSI, W1, P3);
    out[0] = 4.0 * pi * p.zlen * d.ELL2 * (-coef000(W1)) * n00;
    delsqh(CHI, W1, P3);
    out[1] = 4.0 * pi * p.zlen * d.ELL2 * (-coef000(W1)) * n00;
    // VALANG = -INTEG_P(XXDX(PSI with LN 0))
    copy0(W1, PSI, P3);
    ln_zero(W1);
    xxdx(W1, W2, P3);
    rtran(W2, 1, P3);
    {
        std::vector<double2> line(d.NR);
        CK(cudaMemcpy2DAsync(line.data(), sizeof(double2), W2->data, (size_t)nk * sizeof(double2), sizeof(double2),
                             d.NR, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double acc = 0.0;
        for (int r = 0; r < d.NR; ++r) {
            const double om = 1.0 - h_x[r];
            acc += line[r].x / (om * om) * h_w[r];
        }
        out[2] = -(2.0 * pi * p.zlen * d.ELL2 * acc);
    }
    // ENE1 = PRODCT(RTRAN DELSQH(PSI with LN doubled), RTRAN(PSI with LN 0))
    copy0(W1, PSI, P3);
    k_ln_copy(W1->ln, PSI->ln, 2.0, s);
    delsqh(W1, W2, P3);
    rtran(W2, 1, P3);
    copy0(W1, PSI, P3);
    ln_zero(W1);
    rtran(W1, 1, P3);
    const double ene1 = prodct(W2, W1);
    // ENE2 = PRODCT(RTRAN DELSQH(CHI), RTRAN DEL2(CHI)); HEL1 = PRODCT(RTRAN DELSQH(PSI), RTRAN DEL2(CHI))
    del2(CHI, W3, P3);
    ln_zero(W3);
    rtran(W3, 1, P3);
    delsqh(CHI, W1, P3);
    rtran(W1, 1, P3);
    const double ene2 = prodct(W1, W3);
    out[3] = -ene1 + ene2;
    delsqh(PSI, W1, P3);
    rtran(W1, 1, P3);
    out[4] = 2.0 * prodct(W1, W3);
    // CALCXY(ROR, ROP, OZ) (1967-2047): OZH times (1-x)^2 by the two MULXM of
    // 1953-1955 is PC2VOR's OZ; TOFP, ABSVEC2 into OZ, then INTEG(TOFF(.)) of
    // the enstrophy weighted by 1, R cos(th), R sin(th), R^2.
    Field* W4 = tmp();
    pc2vor(PSI, CHI, W1, W2, W3, P3);
    tofp(W1, P3);
    tofp(W2, P3);
    tofp(W3, P3);
    k_absvec2(g, W1->data, W2->data, W3->data, W3->data, s);
    double mom[4];
    for (int mode = 0; mode < 4; ++mode) {
        k_mulr(g, W3->data, W4->data, mode, s);
        W4->space = MLEGS_PPP;
        ln_zero(W4);
        toff(W4, P3);
        mom[mode] = 4.0 * pi * p.zlen * d.ELL2 * coef000(W4) * n00;
    }
    out[8] = mom[1] / mom[0];
    out[9] = mom[2] / mom[0];
    out[10] = std::sqrt(mom[3] / mom[0]);
    rel(W4);
    rel(W3);
    rel(W2);
    rel(W1);
    // CALCAT1 (mod_scalar3.f90:286-310) of PSI and CHI per k, at CHOPSET(3)
    auto at1range = [&](const std::vector<double2>& v) {
        double mx = 0.0, mn = 1e300;
        const int nsum = std::min(d.NRCHOP + P3, nrd);
        for (int k = 0; k < nk; ++k) {
            double sx = 0.0, sy = 0.0;
            for (int n = 0; n < nsum; ++n) {
                const double a1 = std::sqrt((2 * n + 1) / 2.0);
                sx += a1 * at(v, 0, n, k).x;
                sy += a1 * at(v, 0, n, k).y;
            }
            const double av = std::hypot(sx, sy);
            mx = std::max(mx, av);
            mn = std::min(mn, av);
        }
        return mx - mn;
    };
    out[5] = at1range(ps);
    out[6] = at1range(cs);
}

// QVORTEX(PSI, CHI), mod_layout.f90:449-609: for PSI, LAY with GAUSDATA%Q =
// 2 QPAIR%Q and B = 1 for every vortex; for CHI, Q = QPAIR%H and B = QPAIR%B;
// each then TOFF, negated with LN 0, and inverted by IDELSQH.  With seeds (the
// NOISE = 1 path, 550-559 / 585-594), before IDELSQH: B = A, NOISE(A, 0.02)
// with ISEED = seeds[field], TOFP of both, FLATTEN(A, B), TOFF(A).
void mlegs_ctx::qvortex(const mlegs_vortex* v, int n, const int32_t* seeds, Field* PSI, Field* CHI) {
    if (!v || n < 1) throw ApiError(MLEGS_ERR_ARG, "QVORTEX: no vortices");
    for (int i = 0; i < n; ++i)  // R0 = R + DR sin(.) must stay positive on every plane
        if (!(v[i].r > std::fabs(v[i].dr)))
            throw ApiError(MLEGS_ERR_ARG, "QVORTEX: the core radius R must be larger than |DR|");
    // vortex list and per-field strengths / decays in one device buffer
    const size_t vb = (size_t)n * sizeof(mlegs_vortex);
    std::vector<double> qb(4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        qb[i] = 2.0 * v[i].q;
        qb[n + i] = 1.0;
        qb[2 * n + i] = v[i].h;
        qb[3 * n + i] = v[i].b;
    }
    uint8_t* dbuf = nullptr;
    CK(cudaMallocAsync((void**)&dbuf, vb + qb.size() * sizeof(double), s));
    CK(cudaMemcpyAsync(dbuf, v, vb, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dbuf + vb, qb.data(), qb.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    const mlegs_vortex* dv = (const mlegs_vortex*)dbuf;
    const double* dq = (const double*)(dbuf + vb);
    Field* A = tmp(MLEGS_PPP);
    Field* out[2] = {PSI, CHI};
    for (int f = 0; f < 2; ++f) {
        A->space = MLEGS_PPP;
        k_fill(A->data, d.ppp(), s);
        k_lay_gaus(g, p.zlen, dv, n, dq + 2 * f * n, dq + (2 * f + 1) * n, A->data, s);
        toff(A, 0);
        k_axpby(A->data, -1.0, A->data, 0.0, nullptr, 0.0, fff(), s);
        ln_zero(A);
        if (seeds) {
            Field* Bc = tmp();
            copy0(Bc, A, 0);
            const double akmax0 = 2.0 * 3.141592653589793238462643383279502884 / p.zlen * (d.NXCHOP - 1);
            k_maxabs(A->data, fff(), 0, diag, s);
            k_noise(g, A->data, diag, 0.02, akmax0 == 0.0 ? 1.0 : akmax0,
                    (long long)(((uint32_t)seeds[f]) ^ 123459876u), s);
            chopdo(A, 0);
            tofp(A, 0);
            tofp(Bc, 0);
            k_maxabs(A->data, d.ppp(), 1, diag, s);
            k_flatten(g, A->data, Bc->data, diag, s);
            toff(A, 0);
            rel(Bc);
        }
        idelsqh(A, out[f], 0);
    }
    rel(A);
    CK(cudaFreeAsync(dbuf, s));
    CK(cudaStreamSynchronize(s));
}

// CALC_BOUSSI_PE(B), mod_boussinesq.f90:112-136: WK = B, LN 0, RTRAN at the
// current chop (pad 0), L2NORM_MK_HALFK / 2 / BV0^2 into pe (NTCHOP x NXCHOP).
void mlegs_ctx::boussi_pe(const Field* B, double* pe) {
    require(B, MLEGS_FFF, "CALC_BOUSSI_PE");
    if (p.bv0 == 0.0) throw ApiError(MLEGS_ERR_ARG, "CALC_BOUSSI_PE: BV0 = 0");
    const size_t nmk = (size_t)d.NTCHOPDIM * d.NXCHOPDIM;
    Field* W = tmp();
    copy0(W, B, 0);
    ln_zero(W);
    rtran(W, 1, 0);
    k_prodct_mk(g, W->data, nullptr, 1, 4.0 * 3.141592653589793238462643383279502884 * p.zlen * d.ELL2, diag, s);
    rel(W);
    std::vector<double> h(nmk);
    CK(cudaMemcpyAsync(h.data(), diag, nmk * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    halfk(h.data(), 1.0, pe, false);
    const size_t nout = (size_t)d.NTCHOP * d.NXCHOP;
    for (size_t q = 0; q < nout; ++q) pe[q] = pe[q] / 2.0 / (p.bv0 * p.bv0);
}

// HYP3SET(NU_R, NU_T, NU_X, HYPER_R, HYPER_T, HYPER_X), mod_march.f90:3320-3368
// (without hyperv.dat): exp(-NU * MASK * (k^2 / K2MAX)^(P/2)) per direction, with
// the masks of the first call.  The device tables are allocated once and
// rewritten in place afterwards, so captured step graphs read the new values.
void mlegs_ctx::hyp3set(const double nu[3], double** tables) {
    const int nrc = d.NRCHOP, ph2 = p.visc_p / 2;
    auto ipow = [](double v, int e) { double r2 = 1.0; for (int q = 0; q < e; ++q) r2 *= v; return r2; };
    const double k2r = 1.5 * 1.5 * (double)((nrc - 1) * nrc) / d.ELL2;
    const double k2t = (double)((d.NTCHOPDIM - 1) * (d.NTCHOPDIM - 1));
    double k2x = 0.0;
    for (double v : h3_ak) k2x = std::max(k2x, v * v);
    std::vector<double> hr((size_t)nrc * d.NTCHOPDIM), ht(d.NTCHOPDIM), hx(d.NXCHOPDIM);
    for (int m = 0; m < d.NTCHOPDIM; ++m) {
        ht[m] = std::exp(-nu[1] * h3_mt[m] * ipow((double)(m * m) / k2t, ph2));
        for (int nn = 1; nn <= nrc; ++nn)
            hr[(size_t)m * nrc + nn - 1] = std::exp(-nu[0] * h3_mr[(size_t)m * nrc + nn - 1] *
                                                    ipow(1.5 * 1.5 * (double)((nn - 1) * nn) / d.ELL2 / k2r, ph2));
    }
    for (int q = 0; q < d.NXCHOPDIM; ++q) hx[q] = std::exp(-nu[2] * h3_mx[q] * ipow(h3_ak[q] * h3_ak[q] / k2x, ph2));
    const std::vector<double>* hs[3] = {&hr, &ht, &hx};
    for (int q = 0; q < 3; ++q) {
        if (!tables[q]) tables[q] = dalloc<double>(hs[q]->size());
        CK(cudaMemcpyAsync(tables[q], hs[q]->data(), hs[q]->size() * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
}

// ENEMON(PSI, CHI, EM, EK), mod_march.f90:2585-2617, at CHOPSET(pad):
// EM(m) = sum_k, EK(k) = sum_m of -PRODCT_MK_HALFK(RTRAN DELSQH(PSI, 2 LN),
// RTRAN(PSI, LN 0)) + PRODCT_MK_HALFK(RTRAN DELSQH(CHI), RTRAN DEL2(CHI)).
void mlegs_ctx::enemon(const Field* PSI, const Field* CHI, int pad, double* em, double* ek) {
    require(PSI, MLEGS_FFF, "ENEMON");
    require(CHI, MLEGS_FFF, "ENEMON");
    const size_t nmk = (size_t)d.NTCHOPDIM * d.NXCHOPDIM;
    const double scale = 4.0 * 3.141592653589793238462643383279502884 * p.zlen * d.ELL2;
    Field *W1 = tmp(), *W2 = tmp();
    copy0(W1, PSI, pad);
    k_ln_copy(W1->ln, PSI->ln, 2.0, s);
    delsqh(W1, W2, pad);
    rtran(W2, 1, pad);
    copy0(W1, PSI, pad);
    ln_zero(W1);
    rtran(W1, 1, pad);
    k_prodct_mk(g, W2->data, W1->data, 0, scale, diag, s);
    del2(CHI, W1, pad);
    rtran(W1, 1, pad);
    delsqh(CHI, W2, pad);
    rtran(W2, 1, pad);
    k_prodct_mk(g, W2->data, W1->data, 0, scale, diag + nmk, s);
    rel(W2);
    rel(W1);
    std::vector<double> h(2 * nmk);
    CK(cudaMemcpyAsync(h.data(), diag, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int nt = d.NTCHOP, nx = d.NXCHOP;
    std::vector<double> mk((size_t)nt * nx);  // (NTCHOP, NXCHOP), m fastest
    halfk(h.data(), -1.0, mk.data(), false);
    halfk(h.data() + nmk, 1.0, mk.data(), true);
    for (int m = 0; m < nt; ++m) {
        double a = 0.0;
        for (int k = 0; k < nx; ++k) a += mk[(size_t)k * nt + m];
        if (em) em[m] = a;
    }
    for (int k = 0; k < nx; ++k) {
        double a = 0.0;
        for (int m = 0; m < nt; ++m) a += mk[(size_t)k * nt + m];
        if (ek) ek[k] = a;
    }
}

// HYP3ADJ(PSI, CHI, B), mod_march.f90:3000-3182, then the two HYP3SET of the
// stepper (283-288).  ENEMON at CHOPSET(2); the spectra metrics and the
// controllers are host code (hyperadj.cu); B (optional) adds the
// hyperdiffusivity controller from CALC_BOUSSI_PE at the current chop.
void mlegs_ctx::hyp3adj(const Field* PSI, const Field* CHI, const Field* B) {
    const int nt = d.NTCHOP, nx = d.NXCHOP;
    std::vector<double> em(nt), ek(nx);
    enemon(PSI, CHI, 2, em.data(), ek.data());
    std::vector<double> pm, pk;
    if (B) {
        require(B, MLEGS_FFF, "HYP3ADJ");
        if (p.bv0 == 0.0) throw ApiError(MLEGS_ERR_ARG, "CALC_BOUSSI_PE: BV0 = 0");
        std::vector<double> pe((size_t)nt * nx);
        boussi_pe(B, pe.data());
        pm.assign(std::max(nt - 2, 0), 0.0);
        pk.assign(nx, 0.0);
        for (int m = 0; m < nt; ++m)  // pe is (NTCHOP, NXCHOP), m fastest
            for (int k = 0; k < nx; ++k) {
                if (m < nt - 2) pm[m] += pe[(size_t)k * nt + m];
                pk[k] += pe[(size_t)k * nt + m];
            }
    }
    hyp3adj_update(adj, em.data(), std::max(nt - 2, 0), ek.data(), nx, nup3, B ? pm.data() : nullptr,
                   (int)pm.size(), B ? pk.data() : nullptr, (int)pk.size(), kap3);
    if (p.visc_sw == 3) {
        hyp3set(nup3, hv);
        hyp3set(kap3, hd);
    }
}

// CALC_BOUSSI_NONLIN(B, RUR, RUP, UZ, BN, ROR, ROP, OZ), mod_boussinesq.f90:235-314.
// On exit ROR, ROP, OZ hold the projected u x omega in velocity form (FFF).
void mlegs_ctx::nonlin(const Field* B, Field* RUR, Field* RUP, Field* UZ, Field* ROR, Field* ROP, Field* OZ,
                       Field* BN, cudaEvent_t vor_ready, Field* PSIN, Field* CHIN) {
    Field *RBR = tmp(), *RBP = tmp(), *BZ = tmp();
    // GRAD(B) on s2, beside the first RTRAN(+1) GEMMs on s; ROR, ROP, OZ may
    // still be in the making on s2 (vor_ready)
    cudaEvent_t ef = next_event();
    CK(cudaEventRecord(ef, s));
    CK(cudaStreamWaitEvent(s2, ef, 0));
    grad(B, RBR, RBP, BZ, 1, s2);
    cudaEvent_t eg = next_event();
    CK(cudaEventRecord(eg, s2));
    {
        Field* const fs[9] = {RUR, RUP, UZ, ROR, ROP, OZ, RBR, RBP, BZ};
        const int pads[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const cudaEvent_t ready[9] = {nullptr, nullptr, nullptr, vor_ready, vor_ready, vor_ready, eg, eg, eg};
        tofp_pipe(fs, pads, 9, ready);
    }
    Field *NR = tmp(), *NP = tmp(), *NZ = tmp();
    const double2* in[10] = {RUR->data, RUP->data, UZ->data, ROR->data, ROP->data,
                             OZ->data,  RBR->data, RBP->data, BZ->data,  nullptr};
    double2* out[4] = {NR->data, NP->data, NZ->data, BN->data};
    k_theta_fused(g, fft, in, out, 0.0, 0.0, 0, s);
    rel(RBR);
    rel(RBP);
    rel(BZ);
    // TOFF(BN) (VERFFT(-1), RTRAN(-1)) on s2 beside PROJECT, IDEL2 and PC2VEL on s;
    // the zero LN of the four results is set there too (nothing on s reads it)
    cudaEvent_t et = next_event();
    CK(cudaEventRecord(et, s));
    CK(cudaStreamWaitEvent(s2, et, 0));
    for (Field* f : {NR, NP, NZ, BN}) {
        f->space = MLEGS_PFP;
        CK(cudaMemsetAsync(f->ln, 0, sizeof(double), s2));
    }
    if (!k_verfft4(g, fft, BN->data, pbuf[0], -1, s2)) k_verfft_f(g, fft, BN->data, pbuf[0], s2);
    fold(0, pf, d.NRCHOPDIM + 1, pbuf[0], BN->data, 0 | 2, 0, 0, 0, s2);
    CK(cudaMemsetAsync(BN->ln, 0, sizeof(double), s2));
    BN->space = MLEGS_FFF;
    cudaEvent_t eb = next_event();
    CK(cudaEventRecord(eb, s2));
    // PSIN, CHIN given: the projected (PSI, CHI) are returned there and the
    // final PC2VEL into (ROR, ROP, OZ) is left to the caller's ETD kernel
    Field *PSI = PSIN ? PSIN : tmp(), *W = tmp(), *CHI = CHIN ? CHIN : tmp();
    project(NR, NP, NZ, PSI, W, 1, 0.0);
    idel2(W, CHI, 0, 0.0, 0);
    if (!PSIN) pc2vel(PSI, CHI, ROR, ROP, OZ, 3);
    for (Field* f : {W, NR, NP, NZ}) rel(f);
    if (!PSIN) rel(PSI);
    if (!CHIN) rel(CHI);
    CK(cudaStreamWaitEvent(s, eb, 0));
}

// VISC1 (mod_march.f90:1529-1576): A <- IHELM(-ALP A, ALP), ALP = 1/(NU DT).
void mlegs_ctx::visc1(Field* A, double nu, double dt) {
    if (nu == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "VISC1: NU CAN'T BE ZERO");
    double alp = 1 / (nu * dt);
    Field* WK = tmp();
    k_axpby_ln(WK->data, -alp, A->data, 0.0, nullptr, 0.0, fff(), WK->ln, -alp, A->ln, 0.0, nullptr, 0.0, s);
    WK->space = MLEGS_FFF;
    ihelm(WK, A, alp, 0);
    rel(WK);
}
// VISC2 (mod_march.f90:1579-1636): A <- IHELM(-DEL2(AO) - ALP A, ALP), ALP = 2/(NU DT).
void mlegs_ctx::visc2(Field* A, const Field* AO, double nu, double dt) {
    if (nu == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "VISC2: NU CAN'T BE ZERO");
    double alp = 2 / nu / dt;
    Field* WK = tmp();
    del2(AO, WK, 2);
    chopdo(WK, 0);
    k_axpby_ln(WK->data, -alp, A->data, 0.0, nullptr, -1.0, fff(), WK->ln, -alp, A->ln, 0.0, nullptr, 0.0, s);
    ihelm(WK, A, alp, 0);
    rel(WK);
}
void mlegs_ctx::visc_be(Field* P, Field* C, Field* B, double dt) {  // 1200-1230
    if (p.visc_sw != 1) return;
    visc1(P, p.nu, dt);
    visc1(C, p.nu, dt);
    if (p.kappa != 0.0) visc1(B, p.kappa, dt);
}
void mlegs_ctx::visc_cn(Field* P, Field* C, Field* B, const Field* PO, const Field* CO, const Field* BO) {
    if (p.visc_sw != 1) return;  // 1233-1265
    visc2(P, PO, p.nu, p.dt);
    visc2(C, CO, p.nu, p.dt);
    if (p.kappa != 0.0) visc2(B, BO, p.kappa, p.dt);
}
void mlegs_ctx::hyperv3(Field* P, Field* C, Field* B, double tf) {  // CALC_BOUSSI_HYPERV 1305-1349
    if (p.visc_sw == 2) {  // HYPERV per field, B only when KAPPAP /= 0 (1327-1335)
        const double dt = tf * p.dt;
        hyperv2(P, p.nu, p.nup, p.visc_p, dt);
        hyperv2(C, p.nu, p.nup, p.visc_p, dt);
        if (p.kappap != 0.0) hyperv2(B, p.kappa, p.kappap, p.visc_p, dt);
        return;
    }
    if (p.visc_sw != 3) return;
    k_hyperv(g, P->data, hv[0], hv[1], hv[2], tf, 0, s);
    k_hyperv(g, C->data, hv[0], hv[1], hv[2], tf, 0, s);
    k_hyperv(g, B->data, hd[0], hd[1], hd[2], tf, 0, s);
}
void mlegs_ctx::etd_hyperv(Field* R, Field* Pp, Field* Z, Field* B, double tf) {  // 1352-1416
    if (p.visc_sw != 3) return;
    k_hyperv(g, R->data, hv[0], hv[1], hv[2], tf, 0, s);
    k_hyperv(g, Pp->data, hv[0], hv[1], hv[2], tf, 0, s);
    k_hyperv(g, Z->data, hv[0], hv[1], hv[2], tf, 0, s);
    k_hyperv(g, B->data, hd[0], hd[1], hd[2], tf, 0, s);
}

// CALC_BOUSSI_ETD_SPONGE(UZ, B, DT), mod_march.f90:1436-1469: UZ and B to PFP
// (RTRAN, VERFFT), damped per z-plane with the m = 0 modes made real, back to
// FFF (TOFF) at the current chop.  The state field B's buffer is swapped an
// even number of times, so it ends in its own buffer.
void mlegs_ctx::sponge(Field* UZ, Field* B, double dt) {
    if (p.rmv_sw != 2 || p.adams) return;
    const double* damp = (dt == p.dt) ? sp_damp : (dt == p.dt * 0.5 ? sp_damp_h : nullptr);
    if (!damp) throw ApiError(MLEGS_ERR_ARG, "CALC_BOUSSI_ETD_SPONGE: DT other than TIM%DT or TIM%DT/2");
    for (Field* f : {UZ, B}) {
        require(f, MLEGS_FFF, "SPONGE: INPUT MUST BE IN FFF_SPACE");
        rtran(f, 1, 0);
        verfft(f, 1);
        k_sponge(g, f->data, damp, s);
        toff(f, 0);
    }
}

// RICH_BOUSSI_FE_BE (mod_march.f90:535-606).  hist: 0 N_PSI, 1 N_CHI, 2 N_B.
void mlegs_ctx::rich_fe_be() {
    const double dt = p.dt, hdt = dt * 0.5;
    t += dt;
    n += 1;
    Field *NP = hist[0], *NC = hist[1], *NB = hist[2];
    force(psi, chi, b, NP, NC, NB);
    Field *P2 = tmp(), *C2 = tmp(), *B2 = tmp();
    const size_t N = fff();
    k_axpby_ln(P2->data, 1.0, psi->data, hdt, NP->data, 0.0, N, P2->ln, 1.0, psi->ln, hdt, NP->ln, 0.0, s);
    k_axpby_ln(C2->data, 1.0, chi->data, hdt, NC->data, 0.0, N, C2->ln, 1.0, chi->ln, hdt, NC->ln, 0.0, s);
    k_axpby_ln(B2->data, 1.0, b->data, hdt, NB->data, 0.0, N, B2->ln, 0.0, nullptr, 0.0, nullptr, 0.0, s);
    P2->space = C2->space = B2->space = MLEGS_FFF;
    visc_be(P2, C2, B2, hdt);
    hyperv3(P2, C2, B2, hdt / p.dt);
    Field *PN = tmp(), *CN = tmp(), *BN = tmp();
    force(P2, C2, B2, PN, CN, BN);
    k_axpby_ln(P2->data, hdt, PN->data, 0.0, nullptr, 1.0, N, P2->ln, hdt, PN->ln, 0.0, nullptr, 1.0, s);
    k_axpby_ln(C2->data, hdt, CN->data, 0.0, nullptr, 1.0, N, C2->ln, hdt, CN->ln, 0.0, nullptr, 1.0, s);
    k_axpby(B2->data, hdt, BN->data, 0.0, nullptr, 1.0, N, s);
    rel(PN);
    rel(CN);
    rel(BN);
    visc_be(P2, C2, B2, hdt);
    hyperv3(P2, C2, B2, hdt / p.dt);
    k_axpby_ln(psi->data, dt, NP->data, 0.0, nullptr, 1.0, N, psi->ln, dt, NP->ln, 0.0, nullptr, 1.0, s);
    k_axpby_ln(chi->data, dt, NC->data, 0.0, nullptr, 1.0, N, chi->ln, dt, NC->ln, 0.0, nullptr, 1.0, s);
    k_axpby(b->data, dt, NB->data, 0.0, nullptr, 1.0, N, s);
    visc_be(psi, chi, b, dt);
    hyperv3(psi, chi, b, 1.0);
    k_axpby_ln(psi->data, 2.0, P2->data, 0.0, nullptr, -1.0, N, psi->ln, 2.0, P2->ln, 0.0, nullptr, -1.0, s);
    k_axpby_ln(chi->data, 2.0, C2->data, 0.0, nullptr, -1.0, N, chi->ln, 2.0, C2->ln, 0.0, nullptr, -1.0, s);
    k_axpby(b->data, 2.0, B2->data, 0.0, nullptr, -1.0, N, s);
    rel(P2);
    rel(C2);
    rel(B2);
}

// STEP_BOUSSI_AB_CN (mod_march.f90:609-661).
void mlegs_ctx::step_ab_cn() {
    const double dt = p.dt;
    t += dt;
    n += 1;
    Field *NP = hist[0], *NC = hist[1], *NB = hist[2];
    Field *PN = tmp(), *CN = tmp(), *BN = tmp();
    force(psi, chi, b, PN, CN, BN);
    Field *P0 = tmp(), *C0 = tmp(), *B0 = tmp();
    copy0(P0, psi, 0);
    copy0(C0, chi, 0);
    copy0(B0, b, 0);
    const size_t N = fff();
    k_axpby_ln(psi->data, 1.5 * dt, PN->data, -0.5 * dt, NP->data, 1.0, N,
               psi->ln, 1.5 * dt, PN->ln, -0.5 * dt, NP->ln, 1.0, s);
    k_axpby_ln(chi->data, 1.5 * dt, CN->data, -0.5 * dt, NC->data, 1.0, N,
               chi->ln, 1.5 * dt, CN->ln, -0.5 * dt, NC->ln, 1.0, s);
    k_axpby(b->data, 1.5 * dt, BN->data, -0.5 * dt, NB->data, 1.0, N, s);
    copy0(NP, PN, 0);
    copy0(NC, CN, 0);
    copy0(NB, BN, 0);
    rel(PN);
    rel(CN);
    rel(BN);
    visc_cn(psi, chi, b, P0, C0, B0);
    rel(P0);
    rel(C0);
    rel(B0);
    hyperv3(psi, chi, b, 1.0);
}

// STEP_BOUSSI_ETDFE_BE (mod_march.f90:664-753), in place on (P, C, B).
// hist (store = true): 0 N_B, 1 R_N_R, 2 R_N_P, 3 N_Z, 4 R_PI_R, 5 R_PI_P, 6 PI_Z.
void mlegs_ctx::etdfe_be(Field* P, Field* C, Field* B, const double* E, const double* NL, double dt, bool store) {
    Field *RURN = tmp(), *RUPN = tmp(), *UZN = tmp(), *RORN = tmp(), *ROPN = tmp(), *OZN = tmp(), *BN = tmp();
    pc2vel(P, C, RURN, RUPN, UZN, 3);
    pc2vor(P, C, RORN, ROPN, OZN, 3);
    nonlin(B, RURN, RUPN, UZN, RORN, ROPN, OZN, BN);
    etd_hyperv(RORN, ROPN, OZN, BN, dt / p.dt);
    pc2vel(P, C, RURN, RUPN, UZN, 3);
    k_etd(g, E, NL, dt, 0, RURN->data, RUPN->data, UZN->data, B->data, RORN->data, ROPN->data, OZN->data,
          BN->data, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, s);
    sponge(UZN, B, dt);
    etd_hyperv(RURN, RUPN, UZN, B, dt / p.dt);
    if (store) {
        const size_t N = fff();
        k_copy(hist[0]->data, BN->data, N, s);
        k_copy(hist[1]->data, RORN->data, N, s);
        k_copy(hist[2]->data, ROPN->data, N, s);
        k_copy(hist[3]->data, OZN->data, N, s);
        k_copy(hist[4]->data, RURN->data, N, s);
        k_copy(hist[5]->data, RUPN->data, N, s);
        k_copy(hist[6]->data, UZN->data, N, s);
    }
    rel(BN);
    rel(RORN);
    rel(ROPN);
    rel(OZN);
    Field* W = tmp();
    Field* Pn = tmp();
    project(RURN, RUPN, UZN, Pn, W, 2, 0.0);
    copy0(P, Pn, 0);
    idel2ln(W, C, 0);
    rel(W);
    rel(Pn);
    if (store) {
        pc2vel(P, C, RURN, RUPN, UZN, 3);
        const size_t N = fff();
        k_axpby(hist[4]->data, 0.5, hist[4]->data, -0.5, RURN->data, 0.0, N, s);
        k_axpby(hist[5]->data, 0.5, hist[5]->data, -0.5, RUPN->data, 0.0, N, s);
        k_axpby(hist[6]->data, 0.5, hist[6]->data, -0.5, UZN->data, 0.0, N, s);
    }
    rel(RURN);
    rel(RUPN);
    rel(UZN);
}

// RICH_BOUSSI_ETDFE_BE (mod_march.f90:756-808).
void mlegs_ctx::rich_etdfe_be() {
    const double dt = p.dt, hdt = dt * 0.5;
    t += dt;
    n += 1;
    Field *P2 = tmp(), *C2 = tmp(), *B2 = tmp();
    copy0(P2, psi, 0);
    copy0(C2, chi, 0);
    copy0(B2, b, 0);
    etdfe_be(P2, C2, B2, hetdE, hetdN, hdt, false);
    visc_be(P2, C2, B2, hdt);
    etdfe_be(P2, C2, B2, hetdE, hetdN, hdt, false);
    visc_be(P2, C2, B2, hdt);
    etdfe_be(psi, chi, b, etdE, etdN, dt, true);
    visc_be(psi, chi, b, dt);
    const size_t N = fff();
    k_axpby_ln(psi->data, 2.0, P2->data, 0.0, nullptr, -1.0, N, psi->ln, 2.0, P2->ln, 0.0, nullptr, -1.0, s);
    k_axpby_ln(chi->data, 2.0, C2->data, 0.0, nullptr, -1.0, N, chi->ln, 2.0, C2->ln, 0.0, nullptr, -1.0, s);
    k_axpby(b->data, 2.0, B2->data, 0.0, nullptr, -1.0, N, s);
    rel(P2);
    rel(C2);
    rel(B2);
}

// STEP_BOUSSI_ETDAB_CN (mod_march.f90:811-901).  The HYPERV filters, the
// second PC2VEL, CALC_BOUSSI_ETDAB_SUB and the history copies run as one
// kernel; PROJECT writes the new PSI in place (its inputs do not alias PSI),
// and the closing R_PI_* -= PC2VEL(PSI, CHI) is one kernel.
void mlegs_ctx::step_etdab_cn() {
    const double dt = p.dt;
    t += dt;
    n += 1;
    Field *P0 = nullptr, *C0 = nullptr, *B0 = nullptr;
    if (p.visc_sw == 1) {  // CALC_BOUSSI_VISC_CN uses the state at the start of the step
        P0 = tmp();
        C0 = tmp();
        B0 = tmp();
        copy0(P0, psi, 0);
        copy0(C0, chi, 0);
        copy0(B0, b, 0);
    }
    Field *RURN = tmp(), *RUPN = tmp(), *UZN = tmp(), *RORN = tmp(), *ROPN = tmp(), *OZN = tmp(), *BN = tmp();
    pc2vel(psi, chi, RURN, RUPN, UZN, 3);
    // PC2VOR on s2: the RTRAN(+1) of the velocity starts beside it
    cudaEvent_t ef = next_event();
    CK(cudaEventRecord(ef, s));
    CK(cudaStreamWaitEvent(s2, ef, 0));
    pc2vor(psi, chi, RORN, ROPN, OZN, 3, s2);
    cudaEvent_t ev = next_event();
    CK(cudaEventRecord(ev, s2));
    Field *PN = tmp(), *CN = tmp();  // projected nonlinear terms as (PSI_N, CHI_N)
    nonlin(b, RURN, RUPN, UZN, RORN, ROPN, OZN, BN, ev, PN, CN);
    EtdAbArgs a{};
    a.E = etdE;
    a.N = etdN;
    a.dt = dt;
    a.hyper = p.visc_sw == 3 ? 1 : 0;
    for (int q = 0; q < 3; ++q) {
        a.hv[q] = hv[q];
        a.hd[q] = hd[q];
    }
    a.psi = psi->data;
    a.chi = chi->data;
    a.psi_ln = psi->ln;
    a.chi_ln = chi->ln;
    a.rur = RURN->data;
    a.rup = RUPN->data;
    a.uz = UZN->data;
    a.b = b->data;
    a.npsi = PN->data;
    a.nchi = CN->data;
    a.npsi_ln = PN->ln;
    a.nchi_ln = CN->ln;
    a.bn = BN->data;
    for (int q = 0; q < 7; ++q) a.hist[q] = hist[q]->data;
    a.out_ln[0] = RURN->ln;
    a.out_ln[1] = RUPN->ln;
    a.out_ln[2] = UZN->ln;
    const bool sp = (p.rmv_sw == 2);
    a.raw_out = sp ? 1 : 0;
    k_etd_ab_fused(g, a, s);
    RURN->space = RUPN->space = UZN->space = MLEGS_FFF;
    if (sp) {  // CALC_BOUSSI_ETD_SPONGE, then the filters and R_PI_* (mod_march.f90:864-866)
        sponge(UZN, b, dt);
        etd_hyperv(RURN, RUPN, UZN, b, 1.0);
        const size_t N = fff();
        k_copy(hist[4]->data, RURN->data, N, s);
        k_copy(hist[5]->data, RUPN->data, N, s);
        k_copy(hist[6]->data, UZN->data, N, s);
    }
    rel(CN);
    rel(PN);
    rel(BN);
    rel(RORN);
    rel(ROPN);
    rel(OZN);
    Field* W = tmp();
    project_fff_ln2(RURN, RUPN, UZN, psi, W);
    idel2ln(W, chi, 0);
    rel(W);
    rel(RURN);
    rel(RUPN);
    rel(UZN);
    k_pc2vel_fused(g, psi->data, psi->ln, chi->data, chi->ln, hist[4]->data, hist[5]->data, hist[6]->data, 3, s, 1);
    if (p.visc_sw == 1) {
        visc_cn(psi, chi, b, P0, C0, B0);
        rel(P0);
        rel(C0);
        rel(B0);
    }
}

// ====================================================================== C ABI

extern "C" {

int mlegs_create(const mlegs_params* p, mlegs_ctx** out) {
    if (!p || !out) return MLEGS_ERR_ARG;
    *out = nullptr;
    mlegs_ctx* c = new (std::nothrow) mlegs_ctx();
    if (!c) return MLEGS_ERR_NOMEM;
    int64_t* prev = g_launch_counter;
    std::vector<void*>* prev_allocs = g_allocs;
    g_allocs = &c->allocs;
    try {
        c->init(*p);
    } catch (const ApiError& e) {
        fprintf(stderr, "mlegs_create: %s\n", e.what());
        g_launch_counter = prev;
        g_allocs = prev_allocs;
        c->destroy();
        delete c;
        return e.code;
    } catch (const std::exception& e) {
        fprintf(stderr, "mlegs_create: %s\n", e.what());
        g_launch_counter = prev;
        g_allocs = prev_allocs;
        c->destroy();
        delete c;
        return MLEGS_ERR_CUDA;
    }
    g_launch_counter = prev;
    g_allocs = prev_allocs;
    *out = c;
    return MLEGS_OK;
}

int mlegs_destroy(mlegs_ctx* ctx) {
    if (!ctx) return MLEGS_ERR_ARG;
    cudaSetDevice(ctx->dev);
    if (ctx->s) cudaStreamSynchronize(ctx->s);
    ctx->destroy();
    delete ctx;
    return MLEGS_OK;
}

const char* mlegs_last_error(const mlegs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int mlegs_set_wait_limit(mlegs_ctx* ctx, int64_t cycles) {
    if (!ctx || cycles < 0) return MLEGS_ERR_ARG;
    ctx->split_wait = (uint64_t)cycles;
    return MLEGS_OK;
}

int mlegs_sync(mlegs_ctx* ctx) {
    return guard(ctx, [&] {
        CK(cudaStreamSynchronize(ctx->s));
        int e = 0;
        CK(cudaMemcpy(&e, ctx->split_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {  // reported once; the context stays usable
            CK(cudaMemset(ctx->split_err, 0, sizeof(int)));
            throw ApiError(MLEGS_ERR_TIMEOUT, "tensor-core GEMM: a bounded wait timed out (results invalid)");
        }
        if (bulk_gemm_error(true) > 0)
            throw ApiError(MLEGS_ERR_TIMEOUT, "RTRAN(+1) GEMM: a bounded pipeline wait timed out (results invalid)");
    });
}

int mlegs_dims(const mlegs_ctx* c, int32_t out[9]) {
    if (!c || !out) return MLEGS_ERR_ARG;
    const Dims& d = c->d;
    int32_t v[9] = {d.NDIMR, d.NDIMTH, d.NX, d.NRCHOPDIM, d.NTCHOPDIM, d.NXCHOPDIM, d.NRH, d.NR, d.NTH};
    memcpy(out, v, sizeof(v));
    return MLEGS_OK;
}

int mlegs_field_alloc(mlegs_ctx* ctx, int space, mlegs_field** out) {
    if (!out) return MLEGS_ERR_ARG;
    if (space < 0 || space > 3) return MLEGS_ERR_TRANSFORM;  // SALLOC: INVALID SPACE TAG
    return guard(ctx, [&] { *out = ctx->new_field_h(space, true); });
}

int mlegs_field_free(mlegs_ctx* ctx, mlegs_field* f) {
    // Memory is released with the context; the handle just stops being used.
    if (!ctx || !f) return MLEGS_ERR_ARG;
    return MLEGS_OK;
}

int mlegs_field_space(const mlegs_field* f) { return f ? f->f.space : -1; }

int mlegs_grid(const mlegs_ctx* c, double* x, double* w, double* r) {
    if (!c) return MLEGS_ERR_ARG;
    for (int i = 0; i < c->d.NR; ++i) {
        if (x) x[i] = c->h_x[i];
        if (w) w[i] = c->h_w[i];
        if (r) r[i] = c->d.ELL * std::sqrt((1 + c->h_x[i]) / (1 - c->h_x[i]));
    }
    return MLEGS_OK;
}

int mlegs_field_axpby(mlegs_ctx* ctx, mlegs_field* y, double a, const mlegs_field* x1, double b,
                      const mlegs_field* x2, double c) {
    return guard(ctx, [&] {
        Field* fy = F(y);
        const Field* f1 = x1 ? F(x1) : nullptr;
        const Field* f2 = x2 ? F(x2) : nullptr;
        for (const Field* q : {(const Field*)fy, f1, f2})
            if (q && q->space != MLEGS_FFF) throw ApiError(MLEGS_ERR_TRANSFORM, "axpby: FFF fields only");
        k_axpby_ln(fy->data, a, f1 ? f1->data : nullptr, b, f2 ? f2->data : nullptr, c, ctx->fff(),
                   fy->ln, a, f1 ? f1->ln : nullptr, b, f2 ? f2->ln : nullptr, c, ctx->s);
    });
}

int mlegs_field_set_ln(mlegs_ctx* ctx, mlegs_field* f, double ln) {
    return guard(ctx, [&] { k_ln_set(F(f)->ln, ln, ctx->s); });
}

int mlegs_field_upload(mlegs_ctx* ctx, mlegs_field* f, int space, const double* host, double ln) {
    if (!host) return MLEGS_ERR_ARG;
    if (space < 0 || space > 3) return MLEGS_ERR_TRANSFORM;
    return guard(ctx, [&] {
        Field* fd = F(f);
        const Dims& d = ctx->d;
        size_t ref = (space == MLEGS_FFF) ? (size_t)d.NRCHOPDIM * d.NTCHOPDIM * d.NXCHOPDIM
                     : (space == MLEGS_PFF) ? (size_t)d.NDIMR * d.NTCHOPDIM * d.NXCHOPDIM
                                            : (size_t)d.NDIMR * d.NDIMTH * d.NX;
        CK(cudaMemcpyAsync(ctx->staging, host, ref * sizeof(double2), cudaMemcpyHostToDevice, ctx->s));
        k_from_ref(ctx->g, space, ctx->staging, fd->data, ctx->s);
        fd->space = space;
        CK(cudaMemcpyAsync(fd->ln, &ln, sizeof(double), cudaMemcpyHostToDevice, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
    });
}

int mlegs_field_download(mlegs_ctx* ctx, const mlegs_field* f, double* host, double* ln) {
    if (!host) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        const Field* fd = F(f);
        const Dims& d = ctx->d;
        int space = fd->space;
        size_t ref = (space == MLEGS_FFF) ? (size_t)d.NRCHOPDIM * d.NTCHOPDIM * d.NXCHOPDIM
                     : (space == MLEGS_PFF) ? (size_t)d.NDIMR * d.NTCHOPDIM * d.NXCHOPDIM
                                            : (size_t)d.NDIMR * d.NDIMTH * d.NX;
        k_to_ref(ctx->g, space, fd->data, ctx->staging, ctx->s);
        CK(cudaMemcpyAsync(host, ctx->staging, ref * sizeof(double2), cudaMemcpyDeviceToHost, ctx->s));
        double lv = 0.0;
        CK(cudaMemcpyAsync(&lv, fd->ln, sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        if (ln) *ln = lv;
    });
}

// ---------------------------------------------------------------- snapshots
// The reference's snapshot files (mod_fft.f90:2224-2642), little-endian, for
// one process:
//   global (MSAVEX / MLOADX): one Fortran unformatted sequential file whose
//     records are [NR NTH NX] [NRCHOP NTCHOP NXCHOP] [SPACE LN] [ZLEN ELL]
//     [MINC MKLINK] [SIZE1 SIZE2 SIZE3] [E(:,:,:)], each framed by 4-byte
//     length markers (INTEGER 4 bytes, REAL(P8) 8, COMPLEX(P8) 16);
//   MPI form (MPISAVEX / MPILOADX): FN.info with the records [NDIMR NDIMTH
//     NDIMX] [NRCHOPDIM NTCHOPDIM NXCHOPDIM] [SPACE LN] [ZLEN ELL]
//     [MINC MKLINK], and FN holding E(:,:,:) as raw COMPLEX(P8), which for
//     one process is the whole array in Fortran order.
// E is the field in the reference's layout of its space (SALLOC shapes).
extern "C++" {
namespace {
size_t ref_elems(const Dims& d, int space, int32_t sz[3]) {
    if (space == MLEGS_FFF) { sz[0] = d.NRCHOPDIM; sz[1] = d.NTCHOPDIM; sz[2] = d.NXCHOPDIM; }
    else if (space == MLEGS_PFF) { sz[0] = d.NDIMR; sz[1] = d.NTCHOPDIM; sz[2] = d.NXCHOPDIM; }
    else { sz[0] = d.NDIMR; sz[1] = d.NDIMTH; sz[2] = d.NX; }
    return (size_t)sz[0] * sz[1] * sz[2];
}
struct Bytes {
    std::vector<unsigned char> b;
    template <class T>
    void put(T v) {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
        b.insert(b.end(), p, p + sizeof(T));
    }
};
void write_record(FILE* fp, const void* data, size_t n) {
    if (n > 0x7fffffffu) throw ApiError(MLEGS_ERR_ARG, "snapshot: records over 2 GiB are not supported");
    const int32_t len = (int32_t)n;
    if (fwrite(&len, 4, 1, fp) != 1 || (n && fwrite(data, 1, n, fp) != n) || fwrite(&len, 4, 1, fp) != 1)
        throw ApiError(MLEGS_ERR_ARG, "snapshot: write failed");
}
std::vector<unsigned char> read_record(FILE* fp, size_t expect) {
    int32_t len = 0, tail = 0;
    if (fread(&len, 4, 1, fp) != 1 || len < 0) throw ApiError(MLEGS_ERR_ARG, "snapshot: bad record marker");
    std::vector<unsigned char> v((size_t)len);
    if ((len && fread(v.data(), 1, (size_t)len, fp) != (size_t)len) || fread(&tail, 4, 1, fp) != 1 || tail != len)
        throw ApiError(MLEGS_ERR_ARG, "snapshot: truncated record");
    if (expect && (size_t)len != expect) throw ApiError(MLEGS_ERR_ARG, "snapshot: unexpected record length");
    return v;
}
template <class T>
T get_at(const std::vector<unsigned char>& v, size_t off) {
    T x;
    std::memcpy(&x, v.data() + off, sizeof(T));
    return x;
}
struct FileCloser {
    FILE* f;
    ~FileCloser() {
        if (f) fclose(f);
    }
};
}  // namespace
}  // extern "C++"

int mlegs_msave(mlegs_ctx* ctx, const mlegs_field* f, const char* path, int global) {
    if (!f || !path) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        const Dims& d = ctx->d;
        int32_t sz[3];
        const int space = F(f)->space;
        std::vector<double> host(2 * ref_elems(d, space, sz));
        double ln = 0.0;
        const int rc = mlegs_field_download(ctx, f, host.data(), &ln);
        if (rc) throw ApiError(rc, ctx->err);
        const std::string fn(path);
        FileCloser hdr{fopen(global ? fn.c_str() : (fn + ".info").c_str(), "wb")};
        if (!hdr.f) throw ApiError(MLEGS_ERR_ARG, "snapshot: cannot open " + fn);
        auto rec3 = [&](int32_t a, int32_t b, int32_t c) {
            Bytes r;
            r.put(a);
            r.put(b);
            r.put(c);
            write_record(hdr.f, r.b.data(), r.b.size());
        };
        if (global) {
            rec3(d.NR, d.NTH, d.NX);
            rec3(d.NRCHOP, d.NTCHOP, d.NXCHOP);
        } else {
            rec3(d.NDIMR, d.NDIMTH, d.NX);
            rec3(d.NRCHOPDIM, d.NTCHOPDIM, d.NXCHOPDIM);
        }
        {
            Bytes r;
            r.put((int32_t)space);
            r.put(ln);
            write_record(hdr.f, r.b.data(), r.b.size());
        }
        {
            Bytes r;
            r.put(ctx->p.zlen);
            r.put(ctx->p.ell);
            write_record(hdr.f, r.b.data(), r.b.size());
        }
        {
            Bytes r;
            r.put((int32_t)1);  // MINC
            r.put((int32_t)0);  // MKLINK
            write_record(hdr.f, r.b.data(), r.b.size());
        }
        const size_t nbytes = host.size() * sizeof(double);
        if (global) {
            rec3(sz[0], sz[1], sz[2]);
            write_record(hdr.f, host.data(), nbytes);
        } else {
            FileCloser raw{fopen(fn.c_str(), "wb")};
            if (!raw.f) throw ApiError(MLEGS_ERR_ARG, "snapshot: cannot open " + fn);
            if (fwrite(host.data(), 1, nbytes, raw.f) != nbytes) throw ApiError(MLEGS_ERR_ARG, "snapshot: write failed");
        }
    });
}

int mlegs_mload(mlegs_ctx* ctx, const char* path, mlegs_field* f, int global) {
    if (!f || !path) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        const Dims& d = ctx->d;
        const std::string fn(path);
        FileCloser hdr{fopen(global ? fn.c_str() : (fn + ".info").c_str(), "rb")};
        if (!hdr.f) throw ApiError(MLEGS_ERR_ARG, "snapshot: cannot open " + fn);
        read_record(hdr.f, 12);  // NR NTH NX (global) or NDIMR NDIMTH NDIMX
        read_record(hdr.f, 12);  // chops or chop dims
        const auto sl = read_record(hdr.f, 12);
        const int space = get_at<int32_t>(sl, 0);
        const double ln = get_at<double>(sl, 4);
        read_record(hdr.f, 16);  // ZLEN ELL: the reference only warns on a mismatch
        read_record(hdr.f, 8);   // MINC MKLINK: likewise
        if (space < 0 || space > 3) throw ApiError(MLEGS_ERR_TRANSFORM, "snapshot: unknown SPACE");
        int32_t sz[3];
        const size_t n = ref_elems(d, space, sz);
        std::vector<double> host(2 * n);
        if (global) {
            const auto s3 = read_record(hdr.f, 12);
            if (get_at<int32_t>(s3, 0) != sz[0] || get_at<int32_t>(s3, 4) != sz[1] || get_at<int32_t>(s3, 8) != sz[2])
                throw ApiError(MLEGS_ERR_DIMMISMATCH, "snapshot: array sizes differ from this context's");
            const auto e = read_record(hdr.f, n * 16);
            std::memcpy(host.data(), e.data(), n * 16);
        } else {
            FileCloser raw{fopen(fn.c_str(), "rb")};
            if (!raw.f) throw ApiError(MLEGS_ERR_ARG, "snapshot: cannot open " + fn);
            if (fread(host.data(), 1, n * 16, raw.f) != n * 16)
                throw ApiError(MLEGS_ERR_DIMMISMATCH, "snapshot: raw file shorter than this context's array");
            unsigned char extra;
            if (fread(&extra, 1, 1, raw.f) == 1)
                throw ApiError(MLEGS_ERR_DIMMISMATCH,
                               "snapshot: raw file longer than this context's array (several writers?)");
        }
        const int rc = mlegs_field_upload(ctx, f, space, host.data(), ln);
        if (rc) throw ApiError(rc, ctx->err);
    });
}

int mlegs_field_copy(mlegs_ctx* ctx, mlegs_field* dst, const mlegs_field* src, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        ctx->copy0(F(dst), F(src), pad);
    });
}

int mlegs_chopdo(mlegs_ctx* ctx, mlegs_field* f, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        ctx->chopdo(F(f), pad);
    });
}

// In-place transforms on user fields swap with the context's scratch buffer
// and then copy back so that the handle keeps its own buffer.
static void user_inplace(mlegs_ctx* ctx, Field* f, const std::function<void(Field*)>& fn);

int mlegs_rtran(mlegs_ctx* ctx, mlegs_field* f, int is, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        if (is != 1 && is != -1) throw ApiError(MLEGS_ERR_ARG, "RTRAN: IS must be +1 or -1");
        user_inplace(ctx, F(f), [&](Field* x) { ctx->rtran(x, is, pad); });
    });
}
int mlegs_horfft(mlegs_ctx* ctx, mlegs_field* f, int is) {
    return guard(ctx, [&] { user_inplace(ctx, F(f), [&](Field* x) { ctx->horfft(x, is); }); });
}
int mlegs_verfft(mlegs_ctx* ctx, mlegs_field* f, int is) {
    return guard(ctx, [&] { user_inplace(ctx, F(f), [&](Field* x) { ctx->verfft(x, is); }); });
}
int mlegs_plnfft(mlegs_ctx* ctx, mlegs_field* f, int is) {
    return guard(ctx, [&] { user_inplace(ctx, F(f), [&](Field* x) { ctx->plnfft(x, is); }); });
}
int mlegs_toff(mlegs_ctx* ctx, mlegs_field* f, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        user_inplace(ctx, F(f), [&](Field* x) { ctx->toff(x, pad); });
    });
}
int mlegs_tofp(mlegs_ctx* ctx, mlegs_field* f, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        user_inplace(ctx, F(f), [&](Field* x) { ctx->tofp(x, pad); });
    });
}

int mlegs_delsqh(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->delsqh(F(a), F(b), pad); });
}
int mlegs_idelsqh(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->idelsqh(F(b), F(a), pad); });
}
int mlegs_mulxm(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->mulxm(F(a), F(b), pad); });
}
int mlegs_xxdx(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->xxdx(F(a), F(b), pad); });
}
int mlegs_del2(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->del2(F(a), F(b), pad); });
}
int mlegs_idel2(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int has_ln, double ln, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->idel2(F(b), F(a), has_ln, ln, pad); });
}
int mlegs_idel2ln(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->idel2ln(F(b), F(a), pad); });
}
// IDEL2LN with the elimination scratch in the library's fixed __device__
// array instead of the context's allocation: the same kernels in the same
// order as mlegs_idel2ln, and no device allocation of any kind.
int mlegs_idel2ln_static(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        const Field* fb = F(b);
        Field* fa = F(a);
        ctx->require(fb, MLEGS_FFF, "IDEL2LN");
        const size_t need = (size_t)ctx->d.NRCHOPDIM * 4 * ctx->d.NTCHOPDIM * ctx->d.NXCHOPDIM;
        double* scr = nullptr;
        char msg[256];
        int rc = static_solve_scratch(ctx->dev, need, &scr, msg, sizeof msg);
        if (rc == 1) throw ApiError(MLEGS_ERR_ARG, msg);
        if (rc != 0) throw CudaError(msg);
        ctx->copy0(fa, fb, pad);
        ctx->ln_zero(fa);
        k_solve_del2(ctx->g, fa->data, fa->ln, 0, 0.0, 0, 0.0, nullptr, scr, pad, ctx->s);
        ctx->chopdo(fa, pad);
        k_farfield_fix(ctx->g, fa->data, ctx->d.NRCHOP + pad, ctx->s);
    });
}
int mlegs_ihelmp(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int p, double alp, double nu, int pad) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        ctx->ihelmp(F(b), F(a), p, alp, nu, pad);
    });
}
int mlegs_hyperv(mlegs_ctx* ctx, mlegs_field* a, double nu, double nup, int p, double dt) {
    return guard(ctx, [&] {
        if (p < 4 || p > 14 || p % 2) throw ApiError(MLEGS_ERR_ARG, "HYPERV: P must be even, 4..14");
        if (dt == 0.0) throw ApiError(MLEGS_ERR_ARG, "HYPERV: DT must not be zero");
        ctx->mark();
        ctx->hyperv2(F(a), nu, nup, p, dt);
        ctx->restore();
    });
}
int mlegs_ihelm(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, double alp, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->ihelm(F(b), F(a), alp, pad); });
}
int mlegs_grad(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* rgr, mlegs_field* rgp, mlegs_field* gz,
               int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->grad(F(a), F(rgr), F(rgp), F(gz), pad); });
}
int mlegs_pc2vel(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, mlegs_field* rur,
                 mlegs_field* rup, mlegs_field* uz, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->pc2vel(F(psi), F(chi), F(rur), F(rup), F(uz), pad); });
}
int mlegs_pc2vor(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, mlegs_field* ror,
                 mlegs_field* rop, mlegs_field* oz, int pad) {
    return guard(ctx, [&] { check_pad(ctx, pad); ctx->pc2vor(F(psi), F(chi), F(ror), F(rop), F(oz), pad); });
}
int mlegs_project(mlegs_ctx* ctx, mlegs_field* rur, mlegs_field* rup, mlegs_field* uz, mlegs_field* psi,
                  mlegs_field* chi, int ln_mode, double ln) {
    return guard(ctx, [&] {
        if (ln_mode < 0 || ln_mode > 2) throw ApiError(MLEGS_ERR_ARG, "PROJECT: bad ln_mode");
        Field *a = F(rur), *b2 = F(rup), *c = F(uz);
        // work on temporaries so the user fields keep their buffers
        Field *ta = ctx->tmp(), *tb = ctx->tmp(), *tc = ctx->tmp();
        ctx->copy0(ta, a, 0);
        ctx->copy0(tb, b2, 0);
        ctx->copy0(tc, c, 0);
        // FFF velocity with PSI%LN by reference and zero input log terms: the
        // steppers' form, one composite FFF -> FFF product per m
        bool composite = false;
        if (ln_mode == 2 && a->space == MLEGS_FFF && b2->space == MLEGS_FFF && c->space == MLEGS_FFF) {
            double lns[3];
            CK(cudaMemcpyAsync(&lns[0], a->ln, sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaMemcpyAsync(&lns[1], b2->ln, sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaMemcpyAsync(&lns[2], c->ln, sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            composite = lns[0] == 0.0 && lns[1] == 0.0 && lns[2] == 0.0;
        }
        if (composite)
            ctx->project_fff_ln2(ta, tb, tc, F(psi), F(chi));
        else
            ctx->project(ta, tb, tc, F(psi), F(chi), ln_mode, ln);
        ctx->copy0(a, ta, 0);
        ctx->copy0(b2, tb, 0);
        ctx->copy0(c, tc, 0);
        ctx->rel(ta);
        ctx->rel(tb);
        ctx->rel(tc);
    });
}
int mlegs_boussi_force(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                       mlegs_field* psin, mlegs_field* chin, mlegs_field* bn) {
    return guard(ctx, [&] {
        ctx->mark();
        ctx->force(F(psi), F(chi), F(b), F(psin), F(chin), F(bn));
        ctx->restore();
    });
}
int mlegs_boussi_nonlin(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* rur, mlegs_field* rup, mlegs_field* uz,
                        mlegs_field* bn, mlegs_field* ror, mlegs_field* rop, mlegs_field* oz) {
    return guard(ctx, [&] {
        const Field* B = F(b);
        Field *a[7] = {F(rur), F(rup), F(uz), F(ror), F(rop), F(oz), F(bn)};
        if (B->space != MLEGS_FFF)
            throw ApiError(MLEGS_ERR_LEGOPERATOR, "CALC_BOUSSI_NONLIN: B SHOULD BE IN FFF SPACE!");
        for (int i = 0; i < 6; ++i) ctx->require(a[i], MLEGS_FFF, "CALC_BOUSSI_NONLIN");
        for (int i = 0; i < 7; ++i) {
            if (a[i]->data == B->data) throw ApiError(MLEGS_ERR_ARG, "CALC_BOUSSI_NONLIN: fields must be distinct");
            for (int j = 0; j < i; ++j)
                if (a[i]->data == a[j]->data)
                    throw ApiError(MLEGS_ERR_ARG, "CALC_BOUSSI_NONLIN: fields must be distinct");
        }
        ctx->mark();
        ctx->nonlin(B, a[0], a[1], a[2], a[3], a[4], a[5], a[6]);
        ctx->restore();
    });
}
int mlegs_legendre_table(mlegs_ctx* ctx, double* pf) {
    return guard(ctx, [&] {
        if (!pf) throw ApiError(MLEGS_ERR_ARG, "null table");
        const size_t n = (size_t)ctx->d.NTCHOPDIM * (ctx->d.NRCHOPDIM + 1) * ctx->d.NRH;
        CK(cudaStreamSynchronize(ctx->s));
        CK(cudaMemcpy(pf, ctx->pf, n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int mlegs_boussi_energy(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                        double* ke, double* pe, double* dke) {
    return guard(ctx, [&] {
        ctx->mark();
        try {
            ctx->energy(F(psi), F(chi), F(b), ke, pe, dke);
        } catch (...) {
            ctx->restore();
            throw;
        }
        ctx->restore();
    });
}

int mlegs_diagnost(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, double* out) {
    if (!out) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        ctx->mark();
        try {
            ctx->diagnost(F(psi), F(chi), out);
        } catch (...) {
            ctx->restore();
            throw;
        }
        ctx->restore();
    });
}

int mlegs_boussi_pe(mlegs_ctx* ctx, const mlegs_field* b, double* pe) {
    return guard(ctx, [&] {
        ctx->mark();
        try {
            ctx->boussi_pe(F(b), pe);
        } catch (...) {
            ctx->restore();
            throw;
        }
        ctx->restore();
    });
}

int mlegs_qvortex(mlegs_ctx* ctx, const mlegs_vortex* vortices, int n, const int32_t* noise_seeds, mlegs_field* psi,
                  mlegs_field* chi) {
    return guard(ctx, [&] {
        if (F(psi)->data == F(chi)->data) throw ApiError(MLEGS_ERR_ARG, "QVORTEX: PSI and CHI must be distinct");
        if (noise_seeds && (noise_seeds[0] < 0 || noise_seeds[1] < 0))
            throw ApiError(MLEGS_ERR_ARG, "QVORTEX: noise seeds must be non-negative");
        ctx->mark();
        try {
            ctx->qvortex(vortices, n, noise_seeds, F(psi), F(chi));
        } catch (...) {
            ctx->restore();
            throw;
        }
        ctx->restore();
    });
}

int mlegs_enemon(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, int pad, double* em, double* ek) {
    return guard(ctx, [&] {
        check_pad(ctx, pad);
        ctx->mark();
        try {
            ctx->enemon(F(psi), F(chi), pad, em, ek);
        } catch (...) {
            ctx->restore();
            throw;
        }
        ctx->restore();
    });
}

int mlegs_hyp3adj(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b) {
    return guard(ctx, [&] {
        ctx->mark();
        try {
            ctx->hyp3adj(F(psi), F(chi), b ? F(b) : nullptr);
        } catch (...) {
            ctx->restore();
            throw;
        }
        ctx->restore();
    });
}

int mlegs_hyp3_coeffs(mlegs_ctx* ctx, double* out) {
    if (!out) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        for (int q = 0; q < 3; ++q) {
            out[q] = ctx->nup3[q];
            out[3 + q] = ctx->kap3[q];
        }
    });
}

int mlegs_solver_init(mlegs_ctx* ctx, mlegs_field* psi, mlegs_field* chi, mlegs_field* b) {
    return guard(ctx, [&] {
        Field *P = F(psi), *C = F(chi), *B = F(b);
        if (P->space != MLEGS_FFF || C->space != MLEGS_FFF || B->space != MLEGS_FFF)
            throw ApiError(MLEGS_ERR_TRANSFORM, "solver state must be in FFF space");
        ctx->psi = P;
        ctx->chi = C;
        ctx->b = B;
        ctx->t = 0.0;
        ctx->n = 0;
        for (Field* h : ctx->hist) {
            ctx->zero_fff(h);
            ctx->ln_zero(h);
            h->space = MLEGS_FFF;
        }
        // factors of the steady step's solves, so that a captured step finds them
        ctx->factors(0, 0, 0.0);
        if (!ctx->p.adams) ctx->factors(1, 0, 0.0);
        if (ctx->p.visc_sw == 1) {  // VISC2's Helmholtz shifts (same expression as visc2)
            ctx->factors(2, 0, 2 / ctx->p.nu / ctx->p.dt);
            if (ctx->p.kappa != 0.0) ctx->factors(2, 0, 2 / ctx->p.kappa / ctx->p.dt);
        }
        ctx->mark();
        if (ctx->p.adams) ctx->rich_fe_be();
        else ctx->rich_etdfe_be();
        ctx->restore();
        ctx->solver_ready = true;
        if (ctx->gexec) {
            cudaGraphExecDestroy(ctx->gexec);
            ctx->gexec = nullptr;
        }
        if (ctx->graph) {
            cudaGraphDestroy(ctx->graph);
            ctx->graph = nullptr;
        }
    });
}

int mlegs_step(mlegs_ctx* ctx, int nsteps) {
    return guard(ctx, [&] {
        if (!ctx->solver_ready) throw ApiError(MLEGS_ERR_STATE, "mlegs_solver_init has not run");
        for (int q = 0; q < nsteps; ++q) {
            ctx->mark();
            ctx->step_once();
            ctx->restore();
        }
    });
}

// nsteps replays of the captured steady step on ctx->s (captured on first use)
static void graph_steps(mlegs_ctx* ctx, int nsteps) {
    if (!ctx->gexec) {
        ctx->mark();
        double t0 = ctx->t;
        int n0 = ctx->n;
        int64_t before = ctx->launches;
        CK(cudaStreamBeginCapture(ctx->s, cudaStreamCaptureModeThreadLocal));
        try {
            ctx->step_once();
        } catch (...) {
            cudaGraph_t gtmp = nullptr;
            cudaStreamEndCapture(ctx->s, &gtmp);
            if (gtmp) cudaGraphDestroy(gtmp);
            ctx->restore();
            throw;
        }
        CK(cudaStreamEndCapture(ctx->s, &ctx->graph));
        ctx->graph_launches = ctx->launches - before;
        ctx->launches = before;
        ctx->restore();
        ctx->t = t0;
        ctx->n = n0;
        CK(cudaGraphInstantiate(&ctx->gexec, ctx->graph, 0));
    }
    for (int q = 0; q < nsteps; ++q) {
        CK(cudaGraphLaunch(ctx->gexec, ctx->s));
        ctx->launches += ctx->graph_launches;
        ctx->t += ctx->p.dt;
        ctx->n += 1;
    }
}

int mlegs_step_graph(mlegs_ctx* ctx, int nsteps) {
    return guard(ctx, [&] {
        if (!ctx->solver_ready) throw ApiError(MLEGS_ERR_STATE, "mlegs_solver_init has not run");
        graph_steps(ctx, nsteps);
    });
}

// Per step: mlegs_field_upload of the three state fields (FFF) from host[i] /
// ln[i], one graph replay, mlegs_field_download into the same buffers.  The
// copies run on s_up / s_down and the layout conversions and the step on
// ctx->s.  Each field moves in IO_CHUNKS pieces and the next step's upload of
// a piece waits only for that piece's download, so the uploads run beside the
// downloads one piece behind them.
int mlegs_run_host(mlegs_ctx* ctx, int nsteps, double* const* host, double* ln) {
    if (nsteps < 0 || !host || !ln) return MLEGS_ERR_ARG;
    for (int i = 0; i < 3; ++i)
        if (!host[i]) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        if (!ctx->solver_ready) throw ApiError(MLEGS_ERR_STATE, "mlegs_solver_init has not run");
        const Dims& d = ctx->d;
        const size_t bytes = (size_t)d.NRCHOPDIM * d.NTCHOPDIM * d.NXCHOPDIM * sizeof(double2);
        Field* st[3] = {ctx->psi, ctx->chi, ctx->b};
        // set up on first use (each piece again if an earlier set-up stopped half way)
        if (!ctx->s_up) CK(cudaStreamCreateWithFlags(&ctx->s_up, cudaStreamNonBlocking));
        if (!ctx->s_down) CK(cudaStreamCreateWithFlags(&ctx->s_down, cudaStreamNonBlocking));
        for (cudaEvent_t& e : ctx->io_ev)
            if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (int i = 0; i < 3; ++i) {
            if (!ctx->io_in[i]) ctx->io_in[i] = dalloc<double2>(bytes / sizeof(double2));
            if (!ctx->io_out[i]) ctx->io_out[i] = dalloc<double2>(bytes / sizeof(double2));
        }
        if (!ctx->io_ln) CK(cudaHostAlloc((void**)&ctx->io_ln, 3 * sizeof(double), cudaHostAllocDefault));
        if (nsteps == 0) return;
        for (int i = 0; i < 3; ++i) ctx->io_ln[i] = ln[i];
        // the first uploads overwrite the state's LN slots: after the work already queued on ctx->s
        cudaEvent_t* ev = ctx->io_ev;
        constexpr int NC = mlegs_ctx::IO_CHUNKS;
        size_t cut[NC + 1];  // byte offsets of the pieces, on 16-byte entries
        const size_t elems = bytes / sizeof(double2);
        for (int j = 0; j <= NC; ++j) cut[j] = elems * j / NC * sizeof(double2);
        CK(cudaEventRecord(ev[0], ctx->s));
        CK(cudaStreamWaitEvent(ctx->s_up, ev[0], 0));
        try {
            for (int k = 0; k < nsteps; ++k) {
                for (int i = 0; i < 3; ++i) {
                    for (int j = 0; j < NC; ++j) {
                        if (k > 0) CK(cudaStreamWaitEvent(ctx->s_up, ev[6 + NC * i + j], 0));
                        CK(cudaMemcpyAsync((char*)ctx->io_in[i] + cut[j], (const char*)host[i] + cut[j],
                                           cut[j + 1] - cut[j], cudaMemcpyHostToDevice, ctx->s_up));
                    }
                    CK(cudaMemcpyAsync(st[i]->ln, ctx->io_ln + i, sizeof(double), cudaMemcpyHostToDevice, ctx->s_up));
                    CK(cudaEventRecord(ev[i], ctx->s_up));
                    CK(cudaStreamWaitEvent(ctx->s, ev[i], 0));
                    k_from_ref(ctx->g, MLEGS_FFF, ctx->io_in[i], st[i]->data, ctx->s);
                    st[i]->space = MLEGS_FFF;
                }
                graph_steps(ctx, 1);
                for (int i = 0; i < 3; ++i) {
                    k_to_ref(ctx->g, MLEGS_FFF, st[i]->data, ctx->io_out[i], ctx->s);
                    CK(cudaEventRecord(ev[3 + i], ctx->s));
                    CK(cudaStreamWaitEvent(ctx->s_down, ev[3 + i], 0));
                    for (int j = 0; j < NC; ++j) {
                        CK(cudaMemcpyAsync((char*)host[i] + cut[j], (const char*)ctx->io_out[i] + cut[j],
                                           cut[j + 1] - cut[j], cudaMemcpyDeviceToHost, ctx->s_down));
                        if (j == NC - 1)  // the last piece's event covers the LN too
                            CK(cudaMemcpyAsync(ctx->io_ln + i, st[i]->ln, sizeof(double), cudaMemcpyDeviceToHost,
                                               ctx->s_down));
                        CK(cudaEventRecord(ev[6 + NC * i + j], ctx->s_down));
                    }
                }
            }
        } catch (...) {  // no copy to or from the caller's buffers outlives the call
            cudaStreamSynchronize(ctx->s_up);
            cudaStreamSynchronize(ctx->s_down);
            throw;
        }
        CK(cudaStreamSynchronize(ctx->s_down));
        CK(cudaStreamSynchronize(ctx->s));
        for (int i = 0; i < 3; ++i) ln[i] = ctx->io_ln[i];
    });
}

int mlegs_time(const mlegs_ctx* ctx, double* t, int32_t* n) {
    if (!ctx) return MLEGS_ERR_ARG;
    if (t) *t = ctx->t;
    if (n) *n = ctx->n;
    return MLEGS_OK;
}

int mlegs_check_finite(mlegs_ctx* ctx) {
    int flag = 0;
    int rc = guard(ctx, [&] {
        if (!ctx->psi) throw ApiError(MLEGS_ERR_STATE, "no solver state");
        CK(cudaMemsetAsync(ctx->dflag, 0, sizeof(int), ctx->s));
        for (Field* f : {ctx->psi, ctx->chi, ctx->b}) k_finite(f->data, ctx->fff(), ctx->dflag, ctx->s);
        CK(cudaMemcpyAsync(&flag, ctx->dflag, sizeof(int), cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
    });
    if (rc) return rc;
    if (flag) {
        ctx->set_error("ANYNAN: non-finite value in the solver state");
        return MLEGS_ERR_NONFINITE;
    }
    return MLEGS_OK;
}

int mlegs_kernel_time(mlegs_ctx* ctx, int kernel, int reps, double* ms_per_launch, double* bytes_per_launch) {
    if (reps < 1 || kernel < 0 || kernel > 17) return MLEGS_ERR_ARG;
    return guard(ctx, [&] {
        const Dims& d = ctx->d;
        const DevGrid& g = ctx->g;
        cudaStream_t s = ctx->s;
        if ((kernel == 11 || kernel == 12) && !ctx->split_S)
            throw ApiError(MLEGS_ERR_STATE, "context was not created with MLEGS_PREC_SPLIT");
        if (kernel == 14 && !ctx->compV) throw ApiError(MLEGS_ERR_STATE, "needs an FP64 context on the tensor path");
        // k_dmma_peak writes one double per thread: SMs x 4 CTAs x 256 threads
        if (kernel == 17 && (double)d.cap() * 2.0 < dmma_peak_flops() / (8.0 * 4096 * 8 * 512.0 / 256.0))
            throw ApiError(MLEGS_ERR_ARG, "field buffers too small for the FP64 ceiling kernel's output");
        // the temporaries go back to the pool however the timing ends
        struct PoolReturn {
            mlegs_ctx* c;
            std::vector<Field*> taken;
            ~PoolReturn() {
                for (auto it = taken.rbegin(); it != taken.rend(); ++it) c->rel(*it);
            }
        } ret{ctx, {}};
        auto take = [&]() {
            Field* f = ctx->tmp();
            ret.taken.push_back(f);
            return f;
        };
        Field *a = take(), *b = take(), *c = take(), *e = take();
        Field* f9[9];
        for (auto& q : f9) q = take();
        // deterministic non-trivial contents: fill FFF/PPP-sized buffers via axpby of zeros
        // is pointless for timing, so keep whatever the scratch buffers hold (finite zeros
        // after allocation) -- arithmetic cost does not depend on the values.
        auto launch = [&]() {
            switch (kernel) {
                case 0: k_rtran_b2p(g, a->data, b->data, nullptr, 0, s); break;
                case 1: ctx->fold(0, ctx->pf, d.NRCHOPDIM + 1, a->data, b->data, 0 | 2, 0, 0, 0, s); break;
                case 2:
                    if (!k_verfft4(g, ctx->fft, a->data, b->data, +1, s)) k_verfft_b(g, ctx->fft, a->data, b->data, s);
                    break;
                case 3:
                    if (!k_verfft4(g, ctx->fft, a->data, b->data, -1, s)) k_verfft_f(g, ctx->fft, a->data, b->data, s);
                    break;
                case 4: k_horfft_b(g, ctx->fft, a->data, b->data, s); break;
                case 5: k_horfft_f(g, ctx->fft, a->data, b->data, s); break;
                case 6:
                    k_force_pointwise(g, f9[0]->data, f9[1]->data, f9[2]->data, f9[3]->data, f9[4]->data,
                                      f9[5]->data, f9[6]->data, f9[7]->data, f9[8]->data, a->data, b->data,
                                      1.0, 1.0, 1, s);
                    break;
                case 7: {
                    const auto* f = ctx->factors(0, 0, 0.0);
                    if (f) k_solve_factored(g, f->F5, f->F7, a->data, b->data, c->ln, 0, 0, 0.0, 0, 1, s);
                    else k_solve_del2(g, a->data, c->ln, 0, 0.0, 0, 0.0, nullptr, ctx->solve_scr, 0, s);
                } break;
                case 8: {
                    const double2* in[10] = {f9[0]->data, f9[1]->data, f9[2]->data, f9[3]->data, f9[4]->data,
                                             f9[5]->data, f9[6]->data, f9[7]->data, f9[8]->data, a->data};
                    double2* out[4] = {b->data, c->data, f9[0]->data, f9[1]->data};
                    k_theta_fused(g, ctx->fft, in, out, 1.0, 1.0, 1, s);
                } break;
                case 15: {  // the nonlinear-term form of the step: 9 inputs, no linear terms
                    const double2* in[10] = {f9[0]->data, f9[1]->data, f9[2]->data, f9[3]->data, f9[4]->data,
                                             f9[5]->data, f9[6]->data, f9[7]->data, f9[8]->data, nullptr};
                    double2* out[4] = {a->data, b->data, c->data, e->data};
                    k_theta_fused(g, ctx->fft, in, out, 0.0, 0.0, 0, s);
                } break;
                case 17:  // the FP64 tensor-path ceiling (FLOPs in place of bytes)
                    k_dmma_peak((double*)a->data, s);
                    break;
                case 16:  // TOFP then TOFF of one FFF field (RTRAN, VERFFT, HORFFT and back)
                    ctx->mark();
                    a->space = MLEGS_FFF;
                    ctx->tofp(a, 0);
                    ctx->toff(a, 0);
                    ctx->restore();
                    break;
                case 9: k_horfft_warp(g, ctx->fft, a->data, b->data, +1, s); break;
                case 11:
                    if (!ctx->split_S) throw ApiError(MLEGS_ERR_STATE, "context was not created with MLEGS_PREC_SPLIT");
                    k_split_b2p(g, ctx->split_S, ctx->split_img, ctx->split_eA, a->data, b->data, nullptr, 0,
                                ctx->split_err, ctx->split_wait, s);
                    break;
                case 10: k_horfft_warp(g, ctx->fft, a->data, b->data, -1, s); break;
                case 12:
                    if (!ctx->split_S) throw ApiError(MLEGS_ERR_STATE, "context was not created with MLEGS_PREC_SPLIT");
                    k_split_fold(g, ctx->split_S, ctx->fimg[0], ctx->feA[0], d.NRCHOPDIM + 1, a->data, b->data, 0,
                                 0, 0, 0, 1, ctx->split_err, ctx->split_wait, s);
                    break;
                case 14:  // PROJECT of FFF inputs f9[0..2] -> b, c through the composites
                    if (!ctx->compV) throw ApiError(MLEGS_ERR_STATE, "needs an FP64 context on the tensor path");
                    k_project_fff_dmma(g, ctx->compV, ctx->compD, ctx->compT, f9[0]->data, f9[1]->data, f9[2]->data,
                                       b->data, c->data, c->ln, ctx->v2p_fff, s);
                    break;
                case 13: {  // PROJECT's fold products: f9[0..2] (PFF) -> b, c (FFF)
                    const int wr = d.NRCHOPDIM;
                    if (!ctx->split_S && ctx->fc_V) {
                        ctx->project_bulk(f9[0]->data, f9[1]->data, f9[2]->data, b->data, c->data, s);
                    } else if (!ctx->split_S && dmma_supported(g)) {
                        k_project_dmma(g, ctx->V, ctx->D, ctx->T, f9[0]->data, f9[1]->data, f9[2]->data, b->data,
                                       c->data, s);
                    } else {
                        ctx->fold(1, ctx->V, wr, f9[0]->data, b->data, 0, 2, 0, 0);
                        ctx->fold(2, ctx->D, wr, f9[1]->data, b->data, 1, 1, 1, 0);
                        ctx->fold(2, ctx->D, wr, f9[0]->data, c->data, 1, 3, 0, 0);
                        ctx->fold(1, ctx->V, wr, f9[1]->data, c->data, 0, 4, 1, 0);
                        ctx->fold(3, ctx->T, wr, f9[2]->data, c->data, 0, 1, 1, 0);
                    }
                } break;
            }
        };
        const double B16 = 16.0;
        double bytes = 0.0;
        switch (kernel) {
            case 0: case 1: case 11: case 12: bytes = B16 * ((double)d.fff() + (double)d.pff()); break;
            case 2: case 3: bytes = B16 * ((double)d.pff() + (double)d.pfp()); break;
            case 4: case 5: bytes = B16 * ((double)d.pfp() + (double)d.ppp()); break;
            case 6: bytes = B16 * 14.0 * (double)d.ppp(); break;  // 10 fields read, 4 written
            case 7: bytes = (B16 * 2.0 + 40.0) * (double)d.fff(); break;  // rhs in, solution out, 5 factors
            case 8: bytes = B16 * 14.0 * (double)d.pfp(); break;  // 10 PFP lines read, 4 written
            case 15: bytes = B16 * 13.0 * (double)d.pfp(); break;  // 9 read, 4 written
            case 13: bytes = B16 * (3.0 * (double)d.pff() + 2.0 * (double)d.fff()); break;
            case 14: bytes = B16 * 5.0 * (double)d.fff(); break;
            // each stage reads its input and writes its output, both ways
            case 16: bytes = 2.0 * B16 * ((double)d.fff() + 2.0 * (double)d.pff() + 2.0 * (double)d.pfp() + (double)d.ppp()); break;
            case 17: bytes = dmma_peak_flops(); break;  // FLOPs, not bytes
            default: bytes = B16 * ((double)d.pfp() + (double)d.ppp()); break;
        }
        for (int q = 0; q < 3; ++q) launch();  // warm-up
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, s));
        for (int q = 0; q < reps; ++q) launch();
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms_per_launch) *ms_per_launch = ms / reps;
        if (bytes_per_launch) *bytes_per_launch = bytes;
    });
}

int64_t mlegs_launch_count(const mlegs_ctx* ctx) { return ctx ? ctx->launches : 0; }
void mlegs_reset_launch_count(mlegs_ctx* ctx) {
    if (ctx) ctx->launches = 0;
}
void* mlegs_stream(mlegs_ctx* ctx) { return ctx ? (void*)ctx->s : nullptr; }

}  // extern "C"

static void user_inplace(mlegs_ctx* ctx, Field* f, const std::function<void(Field*)>& fn) {
    Field* t = ctx->tmp(f->space);
    ctx->mark();
    k_copy(t->data, f->data, ctx->d.elems(f->space), ctx->s);
    cudaMemcpyAsync(t->ln, f->ln, sizeof(double), cudaMemcpyDeviceToDevice, ctx->s);
    t->space = f->space;
    fn(t);
    k_copy(f->data, t->data, ctx->d.elems(t->space), ctx->s);
    cudaMemcpyAsync(f->ln, t->ln, sizeof(double), cudaMemcpyDeviceToDevice, ctx->s);
    f->space = t->space;
    ctx->rel(t);
    ctx->restore();
}
