// theta and z FFTs in FP64, shared-memory Stockham radix-4 (radix-2 for an
// odd log2 length), many lines per CTA.
//
//  VERFFT (mod_fft.f90:928-1113): complex FFT of length NX along z for each
//    (r, m); forward (FFTW_FORWARD) scaled by 1/NX and chopped to
//    k in [0, NXCHOP) U (NX-NXCHOP, NX) stored at 0..NXCHOPDIM-1 (1028-1029);
//    backward unscaled after zero-filling the chopped band (1062-1065).
//  HORFFT (mod_fft.f90:771-926): real FFT of length 2*NTH of the packed
//    samples E(j) = s_{2j} + i s_{2j+1} (844-848), computed as a complex FFT
//    of length NTH plus the standard even/odd split; forward scaled by
//    1/(2 NTH), chopped at NTCHOP with Im(m=0) = 0 (863-866, 883-886).
#include "mlegs_internal.h"

namespace mlegs {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// Stockham autosort FFT of nl lines of length N = 2^L held in a (scratch b).
// SIGN = -1: forward exp(-2 pi i jk/N); +1: backward.  tw[q] = exp(-2 pi i q/N).
// Returns the buffer holding the result.  All threads of the CTA must call it.
template <int SIGN>
__device__ double2* fft_lines(double2* a, double2* b, int nl, int N, int L, const double2* tw) {
    int Ns = 1;
    int bits = L;
    while (bits > 0) {
        if (bits >= 2) {
            const int nb = N >> 2;
            const int step = N / (Ns * 4);
            for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
                int line = t / nb, j = t - line * nb;
                const double2* in = a + (size_t)line * N;
                double2* out = b + (size_t)line * N;
                int k = j % Ns;
                double2 v0 = in[j], v1 = in[j + nb], v2 = in[j + 2 * nb], v3 = in[j + 3 * nb];
                if (k) {
                    double2 w1 = tw[k * step], w2 = tw[2 * k * step], w3 = tw[3 * k * step];
                    if (SIGN > 0) {
                        w1 = cconj(w1);
                        w2 = cconj(w2);
                        w3 = cconj(w3);
                    }
                    v1 = cmul(v1, w1);
                    v2 = cmul(v2, w2);
                    v3 = cmul(v3, w3);
                }
                double2 s02 = make_double2(v0.x + v2.x, v0.y + v2.y);
                double2 d02 = make_double2(v0.x - v2.x, v0.y - v2.y);
                double2 s13 = make_double2(v1.x + v3.x, v1.y + v3.y);
                double2 d13 = make_double2(v1.x - v3.x, v1.y - v3.y);
                // i*SIGN*d13
                double2 id13 = (SIGN > 0) ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);
                int base = (j / Ns) * Ns * 4 + k;
                out[base] = make_double2(s02.x + s13.x, s02.y + s13.y);
                out[base + Ns] = make_double2(d02.x + id13.x, d02.y + id13.y);
                out[base + 2 * Ns] = make_double2(s02.x - s13.x, s02.y - s13.y);
                out[base + 3 * Ns] = make_double2(d02.x - id13.x, d02.y - id13.y);
            }
            Ns *= 4;
            bits -= 2;
        } else {
            const int nb = N >> 1;
            const int step = N / (Ns * 2);
            for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
                int line = t / nb, j = t - line * nb;
                const double2* in = a + (size_t)line * N;
                double2* out = b + (size_t)line * N;
                int k = j % Ns;
                double2 v0 = in[j], v1 = in[j + nb];
                if (k) {
                    double2 w = tw[k * step];
                    if (SIGN > 0) w = cconj(w);
                    v1 = cmul(v1, w);
                }
                int base = (j / Ns) * Ns * 2 + k;
                out[base] = make_double2(v0.x + v1.x, v0.y + v1.y);
                out[base + Ns] = make_double2(v0.x - v1.x, v0.y - v1.y);
            }
            Ns *= 2;
            bits -= 1;
        }
        __syncthreads();
        double2* tmp = a;
        a = b;
        b = tmp;
    }
    return a;
}

static int lines_per_cta(int N) {
    int l = 2048 / N;  // <= 64 KB per ping-pong buffer pair
    if (l < 1) l = 1;
    if (l > 16) l = 16;
    return l;
}

// ---------------------------------------------------------------- VERFFT
// backward: PFF [m][r][k] -> PFP [r][z][m]; CTA = (r, block of ML m's).
__global__ void verfft_b_kernel(DevGrid g, const double2* tw, int L, const double2* pff, double2* pfp,
                                int ml) {
    extern __shared__ double2 sm[];
    const int N = g.NX;
    double2* a = sm;
    double2* b = sm + (size_t)ml * N;
    int r = blockIdx.x;
    int m0 = blockIdx.y * ml;
    int nl = min(ml, g.NTCHOPDIM - m0);
    for (int t = threadIdx.x; t < nl * N; t += blockDim.x) a[t] = make_double2(0.0, 0.0);
    __syncthreads();
    const int kd = g.NXCHOPDIM, kc = g.NXCHOP;
    for (int t = threadIdx.x; t < nl * kd; t += blockDim.x) {
        int line = t / kd, kk = t - line * kd;
        double2 v = pff[((size_t)(m0 + line) * g.NR + r) * kd + kk];
        int q = (kk < kc) ? kk : (N - kd + kk);  // NXCHOPH-1 + (kk - NXCHOP)
        a[(size_t)line * N + q] = v;
    }
    __syncthreads();
    double2* res = fft_lines<+1>(a, b, nl, N, L, tw);
    for (int t = threadIdx.x; t < nl * N; t += blockDim.x) {
        int z = t / nl, line = t - z * nl;
        pfp[((size_t)r * N + z) * g.NTCHOPDIM + m0 + line] = res[(size_t)line * N + z];
    }
}

// forward: PFP [r][z][m] -> PFF [m][r][k] (chopped, scaled 1/NX).
__global__ void verfft_f_kernel(DevGrid g, const double2* tw, int L, const double2* pfp, double2* pff,
                                int ml) {
    extern __shared__ double2 sm[];
    const int N = g.NX;
    double2* a = sm;
    double2* b = sm + (size_t)ml * N;
    int r = blockIdx.x;
    int m0 = blockIdx.y * ml;
    int nl = min(ml, g.NTCHOPDIM - m0);
    for (int t = threadIdx.x; t < nl * N; t += blockDim.x) {
        int z = t / nl, line = t - z * nl;
        a[(size_t)line * N + z] = pfp[((size_t)r * N + z) * g.NTCHOPDIM + m0 + line];
    }
    __syncthreads();
    double2* res = fft_lines<-1>(a, b, nl, N, L, tw);
    const int kd = g.NXCHOPDIM, kc = g.NXCHOP;
    const double sc = 1.0 / N;
    for (int t = threadIdx.x; t < nl * kd; t += blockDim.x) {
        int line = t / kd, kk = t - line * kd;
        int q = (kk < kc) ? kk : (N - kd + kk);
        double2 v = res[(size_t)line * N + q];
        pff[((size_t)(m0 + line) * g.NR + r) * kd + kk] = make_double2(v.x * sc, v.y * sc);
    }
}

// ---------------------------------------------------------------- HORFFT
// backward: PFP [r][z][m] -> PPP [r][z][j]; CTA = block of ZL (r,z) lines.
__global__ void horfft_b_kernel(DevGrid g, const double2* tw, const double2* twh, int L,
                                const double2* pfp, double2* ppp, int zl, int nlines) {
    extern __shared__ double2 sm[];
    const int N = g.NTH;
    double2* X = sm;                          // [zl][N+1]
    double2* a = X + (size_t)zl * (N + 1);    // [zl][N]
    double2* b = a + (size_t)zl * N;          // [zl][N]
    size_t l0 = (size_t)blockIdx.x * zl;
    int nl = (int)min((size_t)zl, nlines - l0);
    const int md = g.NTCHOPDIM;
    for (int t = threadIdx.x; t < nl * (N + 1); t += blockDim.x) {
        int line = t / (N + 1), m = t - line * (N + 1);
        double2 v = make_double2(0.0, 0.0);
        if (m < md && m < g.NTCHOP) v = pfp[(l0 + line) * md + m];
        if (m == 0) v.y = 0.0;
        X[t] = v;
    }
    __syncthreads();
    // Z_m = (X_m + X*_{N-m}) + i e^{i pi m/N} (X_m - X*_{N-m}),  m < N
    for (int t = threadIdx.x; t < nl * N; t += blockDim.x) {
        int line = t / N, m = t - line * N;
        double2 xm = X[(size_t)line * (N + 1) + m];
        double2 xc = cconj(X[(size_t)line * (N + 1) + N - m]);
        double2 s = make_double2(xm.x + xc.x, xm.y + xc.y);
        double2 d = make_double2(xm.x - xc.x, xm.y - xc.y);
        double2 e = cconj(twh[m]);  // e^{+i pi m/N}
        double2 ed = cmul(e, d);
        a[t] = make_double2(s.x - ed.y, s.y + ed.x);
    }
    __syncthreads();
    double2* res = fft_lines<+1>(a, b, nl, N, L, tw);
    for (int t = threadIdx.x; t < nl * N; t += blockDim.x) ppp[l0 * N + t] = res[t];
}

// forward: PPP [r][z][j] -> PFP [r][z][m] (m < NTCHOPDIM, scaled 1/(2 NTH)).
__global__ void horfft_f_kernel(DevGrid g, const double2* tw, const double2* twh, int L,
                                const double2* ppp, double2* pfp, int zl, int nlines) {
    extern __shared__ double2 sm[];
    const int N = g.NTH;
    double2* a = sm;
    double2* b = a + (size_t)zl * N;
    size_t l0 = (size_t)blockIdx.x * zl;
    int nl = (int)min((size_t)zl, nlines - l0);
    for (int t = threadIdx.x; t < nl * N; t += blockDim.x) a[t] = ppp[l0 * N + t];
    __syncthreads();
    double2* Z = fft_lines<-1>(a, b, nl, N, L, tw);
    const int md = g.NTCHOPDIM;
    const double sc = 1.0 / (2.0 * N);
    // X_m = 1/2 (Z_m + Z*_{N-m}) - i/2 e^{-i pi m/N} (Z_m - Z*_{N-m})
    for (int t = threadIdx.x; t < nl * md; t += blockDim.x) {
        int line = t / md, m = t - line * md;
        double2 zm = Z[(size_t)line * N + (m % N)];
        double2 zc = cconj(Z[(size_t)line * N + ((N - m) % N)]);
        double2 s = make_double2(zm.x + zc.x, zm.y + zc.y);
        double2 d = make_double2(zm.x - zc.x, zm.y - zc.y);
        double2 ed = cmul(twh[m], d);  // e^{-i pi m/N} d
        double2 x = make_double2(0.5 * (s.x + ed.y), 0.5 * (s.y - ed.x));
        x.x *= sc;
        x.y *= sc;
        if (m >= g.NTCHOP) x = make_double2(0.0, 0.0);
        if (m == 0) x.y = 0.0;
        pfp[(l0 + line) * md + m] = x;
    }
}

void fft_set_attributes() {
    const int lim = 160 * 1024;
    cudaFuncSetAttribute(verfft_b_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(verfft_f_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_b_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_f_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

void k_verfft_b(const DevGrid& g, const FFTPlan& p, const double2* pff, double2* pfp, cudaStream_t s) {
    int ml = lines_per_cta(g.NX);
    dim3 grid(g.NR, (g.NTCHOPDIM + ml - 1) / ml);
    size_t sm = 2 * (size_t)ml * g.NX * sizeof(double2);
    verfft_b_kernel<<<grid, 256, sm, s>>>(g, p.tw_x, p.lx, pff, pfp, ml);
    count_launch();
}
void k_verfft_f(const DevGrid& g, const FFTPlan& p, const double2* pfp, double2* pff, cudaStream_t s) {
    int ml = lines_per_cta(g.NX);
    dim3 grid(g.NR, (g.NTCHOPDIM + ml - 1) / ml);
    size_t sm = 2 * (size_t)ml * g.NX * sizeof(double2);
    verfft_f_kernel<<<grid, 256, sm, s>>>(g, p.tw_x, p.lx, pfp, pff, ml);
    count_launch();
}
void k_horfft_b(const DevGrid& g, const FFTPlan& p, const double2* pfp, double2* ppp, cudaStream_t s) {
    int zl = lines_per_cta(g.NTH);
    int nlines = g.NR * g.NX;
    size_t sm = ((size_t)zl * (g.NTH + 1) + 2 * (size_t)zl * g.NTH) * sizeof(double2);
    horfft_b_kernel<<<(nlines + zl - 1) / zl, 256, sm, s>>>(g, p.tw_t, p.tw_h, p.lt, pfp, ppp, zl, nlines);
    count_launch();
}
void k_horfft_f(const DevGrid& g, const FFTPlan& p, const double2* ppp, double2* pfp, cudaStream_t s) {
    int zl = lines_per_cta(g.NTH);
    int nlines = g.NR * g.NX;
    size_t sm = 2 * (size_t)zl * g.NTH * sizeof(double2);
    horfft_f_kernel<<<(nlines + zl - 1) / zl, 256, sm, s>>>(g, p.tw_t, p.tw_h, p.lt, ppp, pfp, zl, nlines);
    count_launch();
}

}  // namespace mlegs
