// Register-resident four-step FFT building blocks (FP64).
//
// N = N1 * N2 points per line, one group of N2 lanes per line (G = 32/N2
// groups per warp work on different lines/fields at once):
//   n = n2 + N2 n1, k = k1 + N1 k2
//   step 1  lane n2 holds x[n2 + N2 n1] (n1 < N1) and runs an N1-point DFT in
//           registers (radix-2 DIT, bit reversal resolved at compile time)
//   step 2  twiddle Y[k1] *= W_N^{n2 k1}
//   step 3  transpose through a padded shared-memory tile S[k1][n2]
//           (row pitch N2 + 1 to keep the 16-byte lanes on distinct banks)
//   step 4  lane t runs U = N1/N2 DFTs of N2 points for k1 = t U + u
// Output: lane t holds X[k1 + N1 k2] in o[u N2 + k2].
// Twiddles come from a shared-memory table tw[q] = exp(-2 pi i q / N), q <= N.
#pragma once

#include <cuda_runtime.h>

namespace mlegs {
namespace fft4 {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
template <int SIGN>
__device__ __forceinline__ double2 twid(const double2* tw, int q) {
    double2 w = tw[q];
    return SIGN > 0 ? conj(w) : w;
}

constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v / 2); }

// W_R^e v with W_R = exp(SIGN 2 pi i / R) for an exponent e that is a
// compile-time constant after unrolling: the multiples of pi/4 and pi/8 are
// applied with literal constants (a swap for +-i), the rest read tw[e S].
template <int R, int SIGN>
__device__ __forceinline__ double2 rot(double2 v, int e, const double2* tw, int S) {
    constexpr double C4 = 0.70710678118654752440084436210484903928;   // cos(pi/4)
    constexpr double C8 = 0.92387953251128675612818318939678828682;   // cos(pi/8)
    constexpr double S8 = 0.38268343236508977172845998403039886676;   // sin(pi/8)
    double c, sn;  // W = c + i SIGN sn (sn = sin of the angle 2 pi e / R)
    if (4 * e == R) return SIGN > 0 ? make_double2(-v.y, v.x) : make_double2(v.y, -v.x);
    if (8 * e == R) { c = C4; sn = C4; }
    else if (8 * e == 3 * R) { c = -C4; sn = C4; }
    else if (R == 16 && e == 1) { c = C8; sn = S8; }
    else if (R == 16 && e == 3) { c = S8; sn = C8; }
    else if (R == 16 && e == 5) { c = -S8; sn = C8; }
    else if (R == 16 && e == 7) { c = -C8; sn = S8; }
    else return cmul(twid<SIGN>(tw, e * S), v);
    const double si = SIGN > 0 ? sn : -sn;
    return make_double2(v.x * c - v.y * si, v.x * si + v.y * c);
}

// In-register DFT of size R (natural order in and out), self-sorting Stockham
// radix 2: every register index is a function of unrolled loop counters only,
// so the arrays stay in registers.  S = N / R maps W_R^q to tw[q * S].
template <int R, int SIGN>
__device__ __forceinline__ void dft(double2 (&v)[R], const double2* tw, int S) {
    constexpr int L = ilog2(R);
    double2 b[R];
#pragma unroll
    for (int st = 0; st < L; ++st) {
        const int Ns = 1 << st;
#pragma unroll
        for (int j = 0; j < R / 2; ++j) {
            const int k = j % Ns;
            double2 v0 = (st & 1) ? b[j] : v[j];
            double2 v1 = (st & 1) ? b[j + R / 2] : v[j + R / 2];
            if (k) v1 = rot<R, SIGN>(v1, k * (R / (2 * Ns)), tw, S);
            const int base = (j / Ns) * 2 * Ns + k;
            double2 s0 = make_double2(v0.x + v1.x, v0.y + v1.y);
            double2 s1 = make_double2(v0.x - v1.x, v0.y - v1.y);
            if (st & 1) {
                v[base] = s0;
                v[base + Ns] = s1;
            } else {
                b[base] = s0;
                b[base + Ns] = s1;
            }
        }
    }
    if (L & 1) {
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = b[i];
    }
}

// Four-step FFT of one line held by a group of N2 lanes (lane index t in the group).
// S: the group's transpose tile, N1 * (N2 + 1) complex.  All lanes of the warp
// must call this together (it synchronises the warp).
template <int N1, int N2, int SIGN>
__device__ __forceinline__ void line_fft(double2 (&v)[N1], double2* S, const double2* tw, int t,
                                         double2 (&o)[N1]) {
    constexpr int N = N1 * N2, U = N1 / N2;
    dft<N1, SIGN>(v, tw, N / N1);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        double2 y = v[k1];
        if (k1) y = cmul(twid<SIGN>(tw, t * k1), y);
        S[k1 * (N2 + 1) + t] = y;
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int k1 = t * U + u;
        double2 w[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) w[n2] = S[k1 * (N2 + 1) + n2];
        dft<N2, SIGN>(w, tw, N / N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) o[u * N2 + k2] = w[k2];
    }
    __syncwarp();
}

// Position of entry (k1, n2) of the N1 x N2 transpose tile inside a line slot
// of exactly N complex values: row-major with the column XOR-swizzled by the
// row's lane (k1 / U), so that both the column writes of step 3 (fixed k1,
// lanes t = n2) and the row reads of step 4 (lane t reads rows t U + u) hit
// distinct 16-byte bank groups.
template <int N1, int N2>
__device__ __forceinline__ int swz(int k1, int n2) {
    constexpr int U = N1 / N2;
    return k1 * N2 + (n2 ^ ((k1 / U) & (N2 - 1)));
}

// line_fft with the transpose done in place in the line's own slot L (N
// complex, element i at L[i * STRIDE]); L's previous contents must already be
// consumed by all lanes.
// tw2 (optional): the step-2 twiddles laid out tw2[k1 * N2 + t] = tw[t k1],
// so that the lanes of a group read consecutive entries (tw[t k1] puts them
// k1 entries apart, on the same shared-memory banks for even k1).
template <int N1, int N2, int SIGN>
__device__ __forceinline__ void line_fft_inplace(double2 (&v)[N1], double2* L, const double2* tw, int t,
                                                 double2 (&o)[N1], int stride = 1, const double2* tw2 = nullptr) {
    constexpr int N = N1 * N2, U = N1 / N2;
    dft<N1, SIGN>(v, tw, N / N1);
    // step 2 without tw2: W^{t k1} as running powers of W^t (one table read per
    // lane instead of N1 - 1 reads that share banks), at most N1 - 2 rounded
    // products away from the table value
    const double2 w1 = twid<SIGN>(tw, t);
    double2 wk = w1;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        double2 y = v[k1];
        if (k1) {
            if (tw2) {
                const double2 w = tw2[k1 * N2 + t];
                y = cmul(SIGN > 0 ? conj(w) : w, y);
            } else {
                if (k1 > 1) wk = cmul(wk, w1);
                y = cmul(wk, y);
            }
        }
        L[swz<N1, N2>(k1, t) * stride] = y;
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int k1 = t * U + u;
        double2 w[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) w[n2] = L[swz<N1, N2>(k1, n2) * stride];
        dft<N2, SIGN>(w, tw, N / N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) o[u * N2 + k2] = w[k2];
    }
    __syncwarp();
}

// Index of o[u * N2 + k2] in the line: k1 + N1 * k2 with k1 = t * U + u.
template <int N1, int N2>
__device__ __forceinline__ int out_index(int t, int idx) {
    constexpr int U = N1 / N2;
    return (t * U + idx / N2) + N1 * (idx % N2);
}

}  // namespace fft4
}  // namespace mlegs
