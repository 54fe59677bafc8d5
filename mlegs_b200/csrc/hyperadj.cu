// Adaptive hyperviscosity: host-side spectrum metrics and controllers.
//
// Restates mod_march.f90:
//   2619-2698  SPECURV(ESPEC, USE_RATIO)  Legendre P2 curvature of log10 E (trapezoidal)
//   2700-2774  SPESLOP(ESPEC, RATIO)      Legendre P1 slope of log10 E over log10 k
//   2776-2812  PDAJUST(COEFF, ...)        proportional-derivative update with a floor
//   3000-3182  HYP3ADJ                    curvature and slope controllers for the
//                                         (R, T, X) coefficients, maximum of the two
// without the printing.  The spectra are a few hundred values per call, so
// this is plain host code; ENEMON and CALC_BOUSSI_PE that feed it run on the
// device (ctx.cu).  Index arithmetic keeps the reference's 1-based IS / IE.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mlegs_internal.h"

namespace mlegs {

namespace {
const double kCurvParams[4] = {2.0, 1.0, 0.05, 0.8};   // [KP, KD, OFFSET, SCALE]
const double kSlopeParams[4] = {1.5, 0.5, 1.5, 1.0};
const double kBaselineNup = 0.8;
}  // namespace

double specurv(const double* e, int size, double use_ratio) {
    const double floor_ = 1.0e-22, target = -0.05;
    int ie = size;
    const int is = ie - std::max(1, (int)(ie * use_ratio));
    while (ie > is && e[ie - 1] < floor_) --ie;
    const double r_trunc = 1.0 - (double)(ie - is) / (double)(size - is);
    const int n = ie - is + 1;
    if (n < 10 || r_trunc > 0.2) return target;
    const double dx = 2.0 / (n - 1), c = std::sqrt(5.0 / 8.0);
    double curv = 0.0;
    for (int i = 1; i <= n; ++i) {
        const double x = -1.0 + 2.0 * (i - 1) / (n - 1);
        const double fac = (i == 1 || i == n) ? 0.5 : 1.0;
        curv += fac * std::log10(e[is - 1 + i - 1]) * dx * c * (3.0 * x * x - 1.0);
    }
    return std::min(10.0, std::max(-10.0, curv));
}

double speslop(const double* e, int size, double ratio) {
    const double floor_ = 1.0e-24, drop = 1.0e10;
    int ie = size;
    const int is = ie - std::max(1, (int)(ie * ratio));
    const int k_start = is;
    double peak = -INFINITY;
    for (int i = is; i <= ie; ++i) peak = std::max(peak, e[i - 1]);
    const double rel_floor = peak / drop;
    while (ie > is && (e[ie - 1] < floor_ || e[ie - 1] < rel_floor)) --ie;
    const int n = ie - is + 1;
    if (n < 3) return -3.0;
    const double xi_min = std::log10((double)k_start), xi_max = std::log10((double)(k_start + n - 1));
    const double dx = 2.0 / (n - 1), c = std::sqrt(3.0 / 2.0);
    double slope = 0.0;
    for (int i = 1; i <= n; ++i) {
        const double xi = std::log10((double)(k_start + i - 1));
        const double x = -1.0 + 2.0 * (xi - xi_min) / (xi_max - xi_min);
        const double fac = (i == 1 || i == n) ? 0.5 : 1.0;
        slope += fac * std::log10(e[is - 1 + i - 1]) * dx * c * x;
    }
    slope = slope * 2.0 / (xi_max - xi_min);
    return std::min(5.0, std::max(-15.0, slope));
}

double pdajust(double coeff, double current, double previous, double baseline, const double params[4],
               bool has_threshold, double threshold) {
    double control = params[0] * (current - previous) + params[1] * current + params[2];
    if (has_threshold && current < threshold && previous < threshold) {
        const double severity = std::min(5.0, std::fabs(current - threshold));
        control = -(0.1 + 0.05 * severity);
    }
    control = std::min(1.0, std::max(-0.4, params[3] * control));
    coeff = (1.0 + control) * coeff;
    return coeff < baseline ? baseline : coeff;
}

namespace {
// (R, T, X) <- the curvature and slope controllers of one field (3045-3095 / 3114-3162).
void control3(double coef[3], const double met[4], const double old[4], double base) {
    const double mc = met[0], kc = met[1], ms = met[2], ks = met[3];
    const double cmo = old[0], cko = old[1], smo = old[2], sko = old[3];
    const double t_c = pdajust(coef[1], mc, cmo, base, kCurvParams, true, -1.0);
    const double x_c = pdajust(coef[2], kc, cko, base, kCurvParams, true, -1.0);
    const double t_s = pdajust(coef[1], ms, smo, base, kSlopeParams, false, 0.0);
    const double x_s = pdajust(coef[2], ks, sko, base, kSlopeParams, false, 0.0);
    auto radial = [](double m, double k, double mo, double ko, double& cur, double& prev) {
        if (m > k) {
            prev = (3.0 * mo + ko) / 4.0;
            cur = (3.0 * m + k) / 4.0;
        } else {
            prev = (mo + 3.0 * ko) / 4.0;
            cur = (m + 3.0 * k) / 4.0;
        }
    };
    double cur, prev;
    radial(mc, kc, cmo, cko, cur, prev);
    const double r_c = pdajust(coef[0], cur, prev, base, kCurvParams, true, -1.0);
    radial(ms, ks, smo, sko, cur, prev);
    const double r_s = pdajust(coef[0], cur, prev, base, kSlopeParams, false, 0.0);
    coef[0] = std::min(std::max(r_c, r_s), 2.0);
    coef[1] = std::max(t_c, t_s);
    coef[2] = std::max(x_c, x_s);
}

void metrics(const double* em, int nm, const double* ek, int nk, double met[4]) {
    met[0] = specurv(em, nm, 0.25);
    met[1] = specurv(ek, nk, 0.25);
    met[2] = speslop(em, nm, 1.0 / 3.0);
    met[3] = speslop(ek, nk, 1.0 / 3.0);
}
}  // namespace

void hyp3adj_update(Hyp3State& st, const double* em, int nm, const double* ek, int nk, double nup[3],
                    const double* pm, int npm, const double* pk, int npk, double kap[3]) {
    double met[4];
    metrics(em, nm, ek, nk, met);
    if (st.nupb < 0.0) {
        std::copy(met, met + 4, st.hist);
        st.nupb = kBaselineNup;
    }
    control3(nup, met, st.hist, st.nupb);
    std::copy(met, met + 4, st.hist);
    if (pm && pk) {
        metrics(pm, npm, pk, npk, met);
        if (st.kappapb < 0.0) {
            std::copy(met, met + 4, st.phist);
            st.kappapb = st.nupb;
        }
        control3(kap, met, st.phist, st.kappapb);
        std::copy(met, met + 4, st.phist);
    }
}

}  // namespace mlegs

// ------------------------------------------------------------------ C ABI
extern "C" {

int mlegs_specurv(const double* espec, int n, double use_ratio, double* curv) {
    if (!espec || !curv || n < 1) return MLEGS_ERR_ARG;
    *curv = mlegs::specurv(espec, n, use_ratio);
    return MLEGS_OK;
}

int mlegs_speslop(const double* espec, int n, double ratio, double* slope) {
    if (!espec || !slope || n < 1) return MLEGS_ERR_ARG;
    *slope = mlegs::speslop(espec, n, ratio);
    return MLEGS_OK;
}

int mlegs_hyp3_controller(const double* em, int nm, const double* ek, int nk, double* state, double* coef) {
    if (!em || !ek || !state || !coef || nm < 1 || nk < 1) return MLEGS_ERR_ARG;
    mlegs::Hyp3State st;
    st.nupb = state[0];
    for (int q = 0; q < 4; ++q) st.hist[q] = state[1 + q];
    mlegs::hyp3adj_update(st, em, nm, ek, nk, coef, nullptr, 0, nullptr, 0, nullptr);
    state[0] = st.nupb;
    for (int q = 0; q < 4; ++q) state[1 + q] = st.hist[q];
    return MLEGS_OK;
}

int mlegs_pdajust(double* coeff, double current, double previous, double baseline, const double* params,
                  int has_threshold, double threshold) {
    if (!coeff || !params) return MLEGS_ERR_ARG;
    *coeff = mlegs::pdajust(*coeff, current, previous, baseline, params, has_threshold != 0, threshold);
    return MLEGS_OK;
}

}  // extern "C"
