// Grid tables generated in FP64 on the device.
//
//  k_tables_gauss  : GAUSS_LEGENDRE (mod_lin_legendre.f90:79-131): Newton
//                    iteration on P_n from z0 = cos(pi (i - 1/4)/(n + 1/2)),
//                    stop at |dz| <= 1e-15, one thread per root pair.
//  k_tables_pf     : the orthonormal associated Legendre table of LEG_TBL3
//                    (mod_lin_legendre.f90:526-644), PF[m][nn][i] =
//                    Pbar^m_{m+nn}(x_i), Condon-Shortley phase, int Pbar^2 = 1.
//                    The reference evaluates an unnormalised recurrence in
//                    50-digit FM arithmetic so that (1-x^2)^(m/2) cannot
//                    underflow; here the normalised three-term recurrence runs
//                    in FP64 on a value carried with a separate binary
//                    exponent (renormalised whenever it leaves [2^-400, 2^400]),
//                    so nothing underflows until the final rounding, where
//                    values below the FP64 normal range flush to zero as in
//                    the reference (617-633).
//  k_tables_project: the V, D, T weight matrices of PROJECT
//                    (mod_legops.f90:2485-2497).
#include "mlegs_internal.h"

namespace mlegs {

__global__ void gauss_kernel(double* x, double* w, int n) {
    // Roots i = 1..ceil(n/2) (1-based); for even n the reference's extra
    // iteration i = n/2+1 only rewrites the mirror pair of i = n/2.
    int nroot = (n + 1) / 2;
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > nroot) return;
    const double PI = 3.14159265358979323846;
    double z = cos(PI * (i - 0.25) / (n + 0.5));
    double z1 = 2.0, pp = 1.0;
    int it = 0;
    while (fabs(z - z1) > 1e-15 && it < 100) {
        double p1 = 1.0, p2 = 0.0, p3;
        for (int j = 1; j <= n; ++j) {
            p3 = p2;
            p2 = p1;
            p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
        }
        pp = n * (z * p1 - p2) / (z * z - 1);
        z1 = z;
        z = z1 - p1 / pp;
        ++it;
    }
    double wi = 2.0 / ((1 - z * z) * pp * pp);
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = wi;
    w[n - i] = wi;
}

void k_tables_gauss(double* x, double* w, int n, cudaStream_t s) {
    int nroot = (n + 1) / 2;
    gauss_kernel<<<(nroot + 127) / 128, 128, 0, s>>>(x, w, n);
    count_launch();
}

// One thread per (i, m): recurrence over nn = 0..ne-1.
__global__ void pf_kernel(const double* x, double* pf, int nrh, int ne, int ntchopdim) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int m = blockIdx.y;
    if (i >= nrh || m >= ntchopdim) return;
    double xi = x[i];
    double s = sqrt((1.0 - xi) * (1.0 + xi));
    // Pbar^m_m = (-1)^m sqrt(1/2 prod_{k<=m} (2k+1)/(2k)) s^m, as mantissa * 2^e
    double p = sqrt(0.5);
    int e = 0;
    for (int k = 1; k <= m; ++k) {
        p *= sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
        if (fabs(p) < 0x1p-400 && p != 0.0) {
            p = ldexp(p, 400);
            e -= 400;
        }
    }
    if (m & 1) p = -p;
    double* out = pf + (size_t)m * ne * nrh + i;
    double pm2 = 0.0, pm1 = p;
    out[0] = ldexp(pm1, e);
    if (ne > 1) {
        double v = xi * sqrt(2.0 * m + 3.0) * pm1;
        pm2 = pm1;
        pm1 = v;
        out[(size_t)nrh] = ldexp(pm1, e);
    }
    for (int nn = 2; nn < ne; ++nn) {
        int n = m + nn;
        double a = sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
        double b = sqrt(((double)(n - 1) * (n - 1) - (double)m * m) * (2.0 * n + 1.0) /
                        (((double)n * n - (double)m * m) * (2.0 * n - 3.0)));
        double v = a * xi * pm1 - b * pm2;
        pm2 = pm1;
        pm1 = v;
        if (fabs(pm1) > 0x1p400) {
            pm1 = ldexp(pm1, -400);
            pm2 = ldexp(pm2, -400);
            e += 400;
        }
        out[(size_t)nn * nrh] = ldexp(pm1, e);
    }
}

__global__ void flush_tiny(double* p, size_t n) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n && fabs(p[t]) < 2.2250738585072014e-308) p[t] = 0.0;
}

void k_tables_pf(const double* x, double* pf, int nrh, int ne, int ntchopdim, cudaStream_t s) {
    dim3 grid((nrh + 127) / 128, ntchopdim);
    pf_kernel<<<grid, 128, 0, s>>>(x, pf, nrh, ne, ntchopdim);
    count_launch();
    size_t n = (size_t)ntchopdim * ne * nrh;
    flush_tiny<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pf, n);
    count_launch();
}

// V[m][n][i] = PF/(N(N+1)F_i), D = PFD/(N(N+1)F_i), T = PF w_i,  F_i = (1-x_i^2)/w_i,
// N = max(1, m+n), PFD[:, n] = PF[:, n-1] XXDX(n-1, n) + PF[:, n+1] XXDX(n+1, n)
// (columns of PF . BAND_LOGLEG_XXDX(NN+1), mod_legops.f90:2487-2488).
__global__ void project_kernel(DevGrid g, double* V, double* D, double* T, int pad) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = blockIdx.y;
    int m = blockIdx.z;
    if (i >= g.NRH) return;
    size_t o = ((size_t)m * g.NRCHOPDIM + n) * g.NRH + i;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    if (n >= nn) {
        V[o] = 0.0;
        D[o] = 0.0;
        T[o] = 0.0;
        return;
    }
    int ne = g.NRCHOPDIM + 1;
    const double* pf = g.pf + (size_t)m * ne * g.NRH;
    double xi = g.x[i], wi = g.w[i];
    double F = (1.0 - xi * xi) / wi;
    int N = m + n;
    if (N < 1) N = 1;
    double den = (double)N * (N + 1) * F;
    double p = pf[(size_t)n * g.NRH + i];
    // XXDX band rows: row l sub entry multiplies column l-1, super entry column l+1
    const double* xb = g.xxdx + (size_t)m * g.NB * 2;
    double pfd = pf[(size_t)(n + 1) * g.NRH + i] * xb[(size_t)(n + 1) * 2 + 0];
    if (n >= 1) pfd += pf[(size_t)(n - 1) * g.NRH + i] * xb[(size_t)(n - 1) * 2 + 1];
    V[o] = p / den;
    D[o] = pfd / den;
    T[o] = p * wi;
}

void k_tables_project(const DevGrid& g, double* V, double* D, double* T, int pad, cudaStream_t s) {
    dim3 grid((g.NRH + 127) / 128, g.NRCHOPDIM, g.NTCHOPDIM);
    project_kernel<<<grid, 128, 0, s>>>(g, V, D, T, pad);
    count_launch();
}

}  // namespace mlegs
