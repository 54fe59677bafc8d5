// Fused physical-space stage of CALC_BOUSSI_FORCE / CALC_BOUSSI_NONLIN:
//   HORFFT(+1) of the 9 (10) input fields  ->  VPRODSUB + VDOTPSUB (+ the
//   linear Coriolis/buoyancy terms)  ->  HORFFT(-1) of the 4 results,
// one (r, z) line per warp, so the NR x 2NTH x NX physical fields never reach
// HBM.  Inputs and outputs are PFP lines [r][z][m] (m < NTCHOPDIM).
//
// Restates mod_fft.f90:771-926 (HORFFT, packed real FFT of length 2*NTH),
// mod_legops.f90:2105-2130 (VPRODSUB cross product, z component / r^2),
// 2207-2225 (VDOTPSUB), mod_boussinesq.f90:385-391 (2 Omega z x u - b z,
// + N^2 u_z).  Each warp runs its line's FFT as a warp-synchronous Stockham
// (radix 4, radix 2 for an odd log2 NTH) in its own shared-memory slice;
// after the inverse transform every lane keeps its PP = NTH/32 packed
// samples of the running products in registers.
#include "mlegs_internal.h"
#include "fft4.cuh"

#include <algorithm>

namespace mlegs {

namespace {

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cj(double2 a) { return make_double2(a.x, -a.y); }

// Warp-synchronous Stockham FFT of length N on buffer a (scratch b); returns result buffer.
template <int SIGN>
__device__ __forceinline__ double2* warp_fft(double2* a, double2* b, int N, int L, const double2* tw, int lane) {
    int Ns = 1, bits = L;
    while (bits > 0) {
        if (bits >= 2) {
            const int nb = N >> 2, step = N / (Ns * 4);
            for (int j = lane; j < nb; j += 32) {
                int k = j % Ns;
                double2 v0 = a[j], v1 = a[j + nb], v2 = a[j + 2 * nb], v3 = a[j + 3 * nb];
                if (k) {
                    double2 w1 = tw[k * step], w2 = tw[2 * k * step], w3 = tw[3 * k * step];
                    if (SIGN > 0) { w1 = cj(w1); w2 = cj(w2); w3 = cj(w3); }
                    v1 = cm(v1, w1);
                    v2 = cm(v2, w2);
                    v3 = cm(v3, w3);
                }
                double2 s02 = make_double2(v0.x + v2.x, v0.y + v2.y), d02 = make_double2(v0.x - v2.x, v0.y - v2.y);
                double2 s13 = make_double2(v1.x + v3.x, v1.y + v3.y), d13 = make_double2(v1.x - v3.x, v1.y - v3.y);
                double2 id = (SIGN > 0) ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);
                int base = (j / Ns) * Ns * 4 + k;
                b[base] = make_double2(s02.x + s13.x, s02.y + s13.y);
                b[base + Ns] = make_double2(d02.x + id.x, d02.y + id.y);
                b[base + 2 * Ns] = make_double2(s02.x - s13.x, s02.y - s13.y);
                b[base + 3 * Ns] = make_double2(d02.x - id.x, d02.y - id.y);
            }
            Ns *= 4;
            bits -= 2;
        } else {
            const int nb = N >> 1, step = N / (Ns * 2);
            for (int j = lane; j < nb; j += 32) {
                int k = j % Ns;
                double2 v0 = a[j], v1 = a[j + nb];
                if (k) {
                    double2 w = tw[k * step];
                    if (SIGN > 0) w = cj(w);
                    v1 = cm(v1, w);
                }
                int base = (j / Ns) * Ns * 2 + k;
                b[base] = make_double2(v0.x + v1.x, v0.y + v1.y);
                b[base + Ns] = make_double2(v0.x - v1.x, v0.y - v1.y);
            }
            Ns *= 2;
            bits -= 1;
        }
        __syncwarp();
        double2* t = a;
        a = b;
        b = t;
    }
    return a;
}

// Inverse HORFFT of one PFP line into packed samples held in registers v[q] = z_{lane + 32 q}.
template <int PP>
__device__ __forceinline__ void line_inverse(const double2* __restrict__ src, int md, int ntchop, int N, int L,
                                             const double2* tw, const double2* twh, double2* X, double2* a,
                                             double2* b, int lane, double2 (&v)[PP]) {
    for (int m = lane; m <= N; m += 32) {
        double2 x = make_double2(0.0, 0.0);
        if (m < md && m < ntchop) x = src[m];
        if (m == 0) x.y = 0.0;
        X[m] = x;
    }
    __syncwarp();
    for (int m = lane; m < N; m += 32) {
        double2 xm = X[m], xc = cj(X[N - m]);
        double2 s = make_double2(xm.x + xc.x, xm.y + xc.y), d = make_double2(xm.x - xc.x, xm.y - xc.y);
        double2 ed = cm(cj(twh[m]), d);
        a[m] = make_double2(s.x - ed.y, s.y + ed.x);
    }
    __syncwarp();
    double2* r = warp_fft<+1>(a, b, N, L, tw, lane);
#pragma unroll
    for (int q = 0; q < PP; ++q) {
        int j = lane + 32 * q;
        v[q] = (j < N) ? r[j] : make_double2(0.0, 0.0);
    }
    __syncwarp();
}

// Forward HORFFT of packed samples in registers to a PFP line (m < md).
template <int PP>
__device__ __forceinline__ void line_forward(double2* __restrict__ dst, int md, int ntchop, int N, int L,
                                             const double2* tw, const double2* twh, double2* a, double2* b,
                                             int lane, const double2 (&v)[PP]) {
#pragma unroll
    for (int q = 0; q < PP; ++q) {
        int j = lane + 32 * q;
        if (j < N) a[j] = v[q];
    }
    __syncwarp();
    double2* Z = warp_fft<-1>(a, b, N, L, tw, lane);
    const double sc = 1.0 / (2.0 * N);
    for (int m = lane; m < md; m += 32) {
        double2 zm = Z[m % N], zc = cj(Z[(N - m) % N]);
        double2 s = make_double2(zm.x + zc.x, zm.y + zc.y), d = make_double2(zm.x - zc.x, zm.y - zc.y);
        double2 ed = cm(twh[m], d);
        double2 x = make_double2(0.5 * (s.x + ed.y) * sc, 0.5 * (s.y - ed.x) * sc);
        if (m >= ntchop) x = make_double2(0.0, 0.0);
        if (m == 0) x.y = 0.0;
        dst[m] = x;
    }
    __syncwarp();
}

}  // namespace

// in[0..8]: RUR RUP UZ ROR ROP OZ RBR RBP BZ (PFP); in[9]: B (PFP, linear only)
// out[0..3]: N_r N_theta N_z N_b (PFP)
struct PhysArgs {
    const double2* in[10];
    double2* out[4];
    double omega, bv0;
    int linear;
};

template <int PP>
__global__ void __launch_bounds__(256, 1) theta_fused_kernel(DevGrid g, PhysArgs A, const double2* tw,
                                                          const double2* twh, int L) {
    extern __shared__ double2 sm[];
    const int N = g.NTH, md = g.NTCHOPDIM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    double2* X = sm + (size_t)warp * (3 * N + 1);
    double2* a = X + (N + 1);
    double2* b = a + N;
    const int nlines = g.NR * g.NX;
    for (int line = blockIdx.x * nw + warp; line < nlines; line += gridDim.x * nw) {
        const int r = line / g.NX;
        const double rr = g.r[r];
        const double r2 = rr * rr;
        const size_t off = (size_t)line * md;
        double2 a1[PP], a2[PP], a3[PP], t[PP];
        double2 nr_[PP], np_[PP], nz_[PP], bn_[PP];
        line_inverse<PP>(A.in[0] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, a1);
        line_inverse<PP>(A.in[1] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, a2);
        line_inverse<PP>(A.in[2] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, a3);
        // b1 = r omega_r:  N_theta = a3 b1,  N_z = -a2 b1
        line_inverse<PP>(A.in[3] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            np_[q] = make_double2(a3[q].x * t[q].x, a3[q].y * t[q].y);
            nz_[q] = make_double2(-a2[q].x * t[q].x, -a2[q].y * t[q].y);
        }
        // b2 = r omega_theta: N_r = -a3 b2, N_z += a1 b2
        line_inverse<PP>(A.in[4] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            nr_[q] = make_double2(-a3[q].x * t[q].x, -a3[q].y * t[q].y);
            nz_[q].x += a1[q].x * t[q].x;
            nz_[q].y += a1[q].y * t[q].y;
        }
        // b3 = omega_z: N_r += a2 b3, N_theta -= a1 b3
        line_inverse<PP>(A.in[5] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            nr_[q].x += a2[q].x * t[q].x;
            nr_[q].y += a2[q].y * t[q].y;
            np_[q].x -= a1[q].x * t[q].x;
            np_[q].y -= a1[q].y * t[q].y;
            nz_[q].x /= r2;
            nz_[q].y /= r2;
        }
        // -(u . grad b): (a1 c1 + a2 c2)/r^2 + a3 c3
        line_inverse<PP>(A.in[6] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
#pragma unroll
        for (int q = 0; q < PP; ++q) bn_[q] = make_double2(a1[q].x * t[q].x, a1[q].y * t[q].y);
        line_inverse<PP>(A.in[7] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            bn_[q].x += a2[q].x * t[q].x;
            bn_[q].y += a2[q].y * t[q].y;
            bn_[q].x /= r2;
            bn_[q].y /= r2;
        }
        line_inverse<PP>(A.in[8] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
#pragma unroll
        for (int q = 0; q < PP; ++q) {
            bn_[q].x = -(bn_[q].x + a3[q].x * t[q].x);
            bn_[q].y = -(bn_[q].y + a3[q].y * t[q].y);
        }
        if (A.linear) {
            line_inverse<PP>(A.in[9] + off, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, t);
            const double o2 = 2 * A.omega, n2 = A.bv0 * A.bv0;
#pragma unroll
            for (int q = 0; q < PP; ++q) {
                nr_[q].x += o2 * a2[q].x;
                nr_[q].y += o2 * a2[q].y;
                np_[q].x -= o2 * a1[q].x;
                np_[q].y -= o2 * a1[q].y;
                nz_[q].x -= t[q].x;
                nz_[q].y -= t[q].y;
                bn_[q].x += n2 * a3[q].x;
                bn_[q].y += n2 * a3[q].y;
            }
        }
        line_forward<PP>(A.out[0] + off, md, g.NTCHOP, N, L, tw, twh, a, b, lane, nr_);
        line_forward<PP>(A.out[1] + off, md, g.NTCHOP, N, L, tw, twh, a, b, lane, np_);
        line_forward<PP>(A.out[2] + off, md, g.NTCHOP, N, L, tw, twh, a, b, lane, nz_);
        line_forward<PP>(A.out[3] + off, md, g.NTCHOP, N, L, tw, twh, a, b, lane, bn_);
    }
}

// Single-field warp-per-line HORFFT (same arithmetic as the fused kernel):
//  dir +1: PFP -> PPP,  dir -1: PPP -> PFP.
template <int PP>
__global__ void __launch_bounds__(256) horfft_warp_kernel(DevGrid g, const double2* src, double2* dst,
                                                          const double2* tw, const double2* twh, int L,
                                                          int dir) {
    extern __shared__ double2 sm[];
    const int N = g.NTH, md = g.NTCHOPDIM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    double2* X = sm + (size_t)warp * (3 * N + 1);
    double2* a = X + (N + 1);
    double2* b = a + N;
    const int nlines = g.NR * g.NX;
    for (int line = blockIdx.x * nw + warp; line < nlines; line += gridDim.x * nw) {
        double2 v[PP];
        if (dir > 0) {
            line_inverse<PP>(src + (size_t)line * md, md, g.NTCHOP, N, L, tw, twh, X, a, b, lane, v);
#pragma unroll
            for (int q = 0; q < PP; ++q) {
                int j = lane + 32 * q;
                if (j < N) dst[(size_t)line * N + j] = v[q];
            }
        } else {
#pragma unroll
            for (int q = 0; q < PP; ++q) {
                int j = lane + 32 * q;
                v[q] = (j < N) ? src[(size_t)line * N + j] : make_double2(0.0, 0.0);
            }
            line_forward<PP>(dst + (size_t)line * md, md, g.NTCHOP, N, L, tw, twh, a, b, lane, v);
        }
    }
}

// ------------------------------------------------------------------------
// Four-step versions (fft4.cuh): NTH = N1 * N2, G = 32 / N2 fields or lines
// per warp in parallel, packed samples staged in per-warp shared-memory lines.
namespace {

// Inverse HORFFT of one PFP line by one lane group; packed samples -> P[0..N).
template <int N1, int N2>
__device__ __forceinline__ void grp_inverse(const double2* __restrict__ src, bool valid, int md, int ntchop,
                                            const double2* tw, const double2* twh, double2* S, double2* P, int t) {
    constexpr int N = N1 * N2;
    double2 v[N1], o[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        const int m = t + N2 * n1, mc = N - m;
        double2 xm = make_double2(0.0, 0.0), xc = make_double2(0.0, 0.0);
        if (valid) {
            if (m < md && m < ntchop) xm = src[m];
            if (mc < md && mc < ntchop) xc = src[mc];
        }
        if (m == 0) xm.y = 0.0;
        if (mc == 0) xc.y = 0.0;
        xc = fft4::conj(xc);
        double2 sm = make_double2(xm.x + xc.x, xm.y + xc.y), d = make_double2(xm.x - xc.x, xm.y - xc.y);
        double2 ed = fft4::cmul(fft4::conj(twh[m]), d);  // e^{+i pi m/N} d
        v[n1] = make_double2(sm.x - ed.y, sm.y + ed.x);
    }
    fft4::line_fft<N1, N2, +1>(v, S, tw, t, o);
#pragma unroll
    for (int q = 0; q < N1; ++q) P[fft4::out_index<N1, N2>(t, q)] = o[q];
}

// Forward HORFFT of packed samples P[0..N) by one lane group -> PFP line dst (m < md).
template <int N1, int N2>
__device__ __forceinline__ void grp_forward(const double2* P, bool valid, double2* __restrict__ dst, int md,
                                            int ntchop, const double2* tw, const double2* twh, double2* S, int t) {
    constexpr int N = N1 * N2;
    double2 v[N1], o[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = P[t + N2 * n1];
    fft4::line_fft<N1, N2, -1>(v, S, tw, t, o);
#pragma unroll
    for (int q = 0; q < N1; ++q) S[fft4::out_index<N1, N2>(t, q)] = o[q];  // Z_k, natural order
    __syncwarp();
    const double sc = 1.0 / (2.0 * N);
    for (int m = t; m < md; m += N2) {
        double2 zm = S[m % N], zc = fft4::conj(S[(N - m) % N]);
        double2 sm = make_double2(zm.x + zc.x, zm.y + zc.y), d = make_double2(zm.x - zc.x, zm.y - zc.y);
        double2 ed = fft4::cmul(twh[m], d);  // e^{-i pi m/N} d
        double2 x = make_double2(0.5 * (sm.x + ed.y) * sc, 0.5 * (sm.y - ed.x) * sc);
        if (m >= ntchop) x = make_double2(0.0, 0.0);
        if (m == 0) x.y = 0.0;
        if (valid) dst[m] = x;
    }
    __syncwarp();
}

}  // namespace

template <int N1, int N2>
__global__ void __launch_bounds__(256) theta4_kernel(DevGrid g, PhysArgs A, const double2* tw_g,
                                                     const double2* twh_g) {
    constexpr int N = N1 * N2, G = 32 / N2;
    constexpr int TILE = N1 * (N2 + 1);
    extern __shared__ double2 sm[];
    double2* tw = sm;
    double2* twh = tw + (N + 1);
    for (int q = threadIdx.x; q <= N; q += blockDim.x) {
        tw[q] = tw_g[q];
        twh[q] = twh_g[q];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int gid = lane / N2, t = lane % N2;
    double2* P = twh + (N + 1) + (size_t)warp * (11 * N + G * TILE);  // 10 packed lines + 1 spare
    double2* S = P + 11 * N + gid * TILE;
    const int md = g.NTCHOPDIM, nin = A.linear ? 10 : 9;
    const int nlines = g.NR * g.NX;
    for (int line = blockIdx.x * nw + warp; line < nlines; line += gridDim.x * nw) {
        const size_t off = (size_t)line * md;
        for (int f0 = 0; f0 < nin; f0 += G) {
            const int f = f0 + gid;
            const bool ok = f < nin;
            grp_inverse<N1, N2>(ok ? A.in[f] + off : nullptr, ok, md, g.NTCHOP, tw, twh, S, P + (ok ? f : 10) * N, t);
        }
        __syncwarp();
        const double rr = g.r[line / g.NX];
        const double r2 = rr * rr;
        const double o2 = 2 * A.omega, n2 = A.bv0 * A.bv0;
        for (int j = lane; j < N; j += 32) {
            double2 a1 = P[j], a2 = P[N + j], a3 = P[2 * N + j];
            double2 b1 = P[3 * N + j], b2 = P[4 * N + j], b3 = P[5 * N + j];
            double2 c1 = P[6 * N + j], c2 = P[7 * N + j], c3 = P[8 * N + j];
            double2 nr_ = make_double2(a2.x * b3.x - a3.x * b2.x, a2.y * b3.y - a3.y * b2.y);
            double2 np_ = make_double2(a3.x * b1.x - a1.x * b3.x, a3.y * b1.y - a1.y * b3.y);
            double2 nz_ = make_double2((a1.x * b2.x - a2.x * b1.x) / r2, (a1.y * b2.y - a2.y * b1.y) / r2);
            double2 bn_ = make_double2(-((a1.x * c1.x + a2.x * c2.x) / r2 + a3.x * c3.x),
                                       -((a1.y * c1.y + a2.y * c2.y) / r2 + a3.y * c3.y));
            if (A.linear) {
                double2 bp = P[9 * N + j];
                nr_.x += o2 * a2.x;
                nr_.y += o2 * a2.y;
                np_.x -= o2 * a1.x;
                np_.y -= o2 * a1.y;
                nz_.x -= bp.x;
                nz_.y -= bp.y;
                bn_.x += n2 * a3.x;
                bn_.y += n2 * a3.y;
            }
            P[3 * N + j] = nr_;
            P[4 * N + j] = np_;
            P[5 * N + j] = nz_;
            P[6 * N + j] = bn_;
        }
        __syncwarp();
        for (int f0 = 0; f0 < 4; f0 += G) {
            const int f = f0 + gid;
            const bool ok = f < 4;
            grp_forward<N1, N2>(P + (3 + (ok ? f : 0)) * N, ok, ok ? A.out[f] + off : nullptr, md, g.NTCHOP, tw,
                                twh, S, t);
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------
// Fused physical stage with in-place line slots (9 slots of N per warp):
//   phase 1: RUR RUP UZ [B]  -> slots 0 1 2 3
//   phase 2: ROR ROP OZ RBR  -> slots 4 5 6 7, then per sample
//            slot 4 <- N_r, 5 <- N_theta, 6 <- N_z (all terms), 7 <- a1 c1
//   phase 3: RBP BZ          -> slots 3 8, then slot 7 <- N_b
//   forward: slots 4 5 6 7   -> OUT 0 1 2 3
// Each group's transposes run inside its own line slot (fft4::swz), so a warp
// needs 9 N complex of shared memory instead of 11 N plus padded tiles.
namespace {

// A group with no line in a round still takes part in the warp's barriers:
// grp_inverse5 and grp_forward5 each execute exactly four __syncwarp().
__device__ __forceinline__ void idle_group_syncs() {
    __syncwarp();
    __syncwarp();
    __syncwarp();
    __syncwarp();
}

// Position of physical sample k inside a line slot.  The inverse transform's
// lanes store samples U t + u + N1 k2 (stride U = N1/N2) and the forward
// transform's lanes load samples t + N2 n1; with N2 = 8, flipping the low
// log2(U) bits by the next ones puts both on distinct 16-byte bank groups.
// The pointwise products see the same permutation in every slot.
template <int N1, int N2>
__device__ __forceinline__ int phys_pos(int k) {
    constexpr int U = N1 / N2;
    if constexpr (N2 == 8 && U > 1) return k ^ ((k >> 3) & (U - 1));
    else return k;
}

// Inverse HORFFT of one PFP row into the packed samples L[phys_pos(0..N))
// loaded: the row is already in the slot (an earlier asynchronous copy that
// the warp has waited for); src is then not read.
template <int N1, int N2>
__device__ __forceinline__ void grp_inverse5(const double2* __restrict__ src, bool valid, int md, int ntchop,
                                             const double2* tw, const double2* twh, double2* L, int t,
                                             bool loaded = false) {
    constexpr int N = N1 * N2;
    const int mlim = md < ntchop ? md : ntchop;
    // coalesced row load into the slot (entries m >= mlim read as zero below)
    if (valid && !loaded)
        for (int m = t; m < mlim; m += N2) L[m] = src[m];
    __syncwarp();
    double2 v[N1], o[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
        const int m = t + N2 * n1, mc = N - m;
        double2 xm = make_double2(0.0, 0.0), xc = make_double2(0.0, 0.0);
        if (valid) {
            if (m < mlim) xm = L[m];
            if (mc < mlim) xc = L[mc];
        }
        if (m == 0) xm.y = 0.0;
        xc = fft4::conj(xc);
        double2 sm = make_double2(xm.x + xc.x, xm.y + xc.y), d = make_double2(xm.x - xc.x, xm.y - xc.y);
        double2 ed = fft4::cmul(fft4::conj(twh[m]), d);  // e^{+i pi m/N} d
        v[n1] = make_double2(sm.x - ed.y, sm.y + ed.x);
    }
    __syncwarp();
    fft4::line_fft_inplace<N1, N2, +1>(v, L, tw, t, o);
#pragma unroll
    for (int q = 0; q < N1; ++q) L[phys_pos<N1, N2>(fft4::out_index<N1, N2>(t, q))] = o[q];
}

// Asynchronous copy of one PFP row (m < mlim) into a line slot by the group's
// lanes; completion is waited for with cp.async.wait_group, then __syncwarp.
template <int N2>
__device__ __forceinline__ void row_async(const double2* __restrict__ src, int mlim, double2* L, int t) {
    for (int m = t; m < mlim; m += N2)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(L + m)),
                     "l"(src + m)
                     : "memory");
}
__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int K>
__device__ __forceinline__ void async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(K) : "memory"); }

// Forward HORFFT of the packed samples L[phys_pos(0..N))] to a PFP row (m < md).
template <int N1, int N2>
__device__ __forceinline__ void grp_forward5(double2* L, bool valid, double2* __restrict__ dst, int md, int ntchop,
                                             const double2* tw, const double2* twh, int t) {
    constexpr int N = N1 * N2;
    double2 v[N1], o[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = L[phys_pos<N1, N2>(t + N2 * n1)];
    __syncwarp();
    fft4::line_fft_inplace<N1, N2, -1>(v, L, tw, t, o);
#pragma unroll
    for (int q = 0; q < N1; ++q) L[fft4::out_index<N1, N2>(t, q)] = o[q];  // Z_k, natural order
    __syncwarp();
    const double sc = 1.0 / (2.0 * N);
    for (int m = t; m < md; m += N2) {
        double2 zm = L[m % N], zc = fft4::conj(L[(N - m) % N]);
        double2 sm = make_double2(zm.x + zc.x, zm.y + zc.y), d = make_double2(zm.x - zc.x, zm.y - zc.y);
        double2 ed = fft4::cmul(twh[m], d);  // e^{-i pi m/N} d
        double2 x = make_double2(0.5 * (sm.x + ed.y) * sc, 0.5 * (sm.y - ed.x) * sc);
        if (m >= ntchop) x = make_double2(0.0, 0.0);
        if (m == 0) x.y = 0.0;
        if (valid) dst[m] = x;
    }
}

// Kernel-argument arrays indexed by a run-time value without copying them to
// local memory.
__device__ __forceinline__ const double2* pick_in(const PhysArgs& A, int i) {
    const double2* p = A.in[0];
#pragma unroll
    for (int q = 1; q < 10; ++q)
        if (i == q) p = A.in[q];
    return p;
}
__device__ __forceinline__ double2* pick_out(const PhysArgs& A, int i) {
    double2* p = A.out[0];
#pragma unroll
    for (int q = 1; q < 4; ++q)
        if (i == q) p = A.out[q];
    return p;
}

// After phase 2 (slots: 0-2 velocity, 3 B, 4-6 vorticity, 7 RBR): slots 4-6 <-
// N_r, N_theta, N_z of VPRODSUB (+ the linear terms), slot 7 <- a1 c1.
template <int N>
__device__ __forceinline__ void theta_products_r2(double2* L, int lane, double ir2, double o2, int linear) {
    for (int j = lane; j < N; j += 32) {
        const double2 a1 = L[j], a2 = L[N + j], a3 = L[2 * N + j];
        const double2 b1 = L[4 * N + j], b2 = L[5 * N + j], b3 = L[6 * N + j], c1 = L[7 * N + j];
        double2 nr_ = make_double2(a2.x * b3.x - a3.x * b2.x, a2.y * b3.y - a3.y * b2.y);
        double2 np_ = make_double2(a3.x * b1.x - a1.x * b3.x, a3.y * b1.y - a1.y * b3.y);
        double2 nz_ = make_double2((a1.x * b2.x - a2.x * b1.x) * ir2, (a1.y * b2.y - a2.y * b1.y) * ir2);
        if (linear) {
            const double2 bp = L[3 * N + j];
            nr_.x += o2 * a2.x;
            nr_.y += o2 * a2.y;
            np_.x -= o2 * a1.x;
            np_.y -= o2 * a1.y;
            nz_.x -= bp.x;
            nz_.y -= bp.y;
        }
        L[4 * N + j] = nr_;
        L[5 * N + j] = np_;
        L[6 * N + j] = nz_;
        L[7 * N + j] = make_double2(a1.x * c1.x, a1.y * c1.y);
    }
}

// After phase 3 (slot 3 RBP, slot 8 BZ): slot 7 <- N_b of VDOTPSUB (+ N^2 u_z).
template <int N>
__device__ __forceinline__ void theta_products_r3(double2* L, int lane, double ir2, double n2, int linear) {
    for (int j = lane; j < N; j += 32) {
        const double2 a2 = L[N + j], a3 = L[2 * N + j], c2 = L[3 * N + j], c3 = L[8 * N + j];
        const double2 bp = L[7 * N + j];
        double2 bn_ = make_double2(-((bp.x + a2.x * c2.x) * ir2 + a3.x * c3.x),
                                   -((bp.y + a2.y * c2.y) * ir2 + a3.y * c3.y));
        if (linear) {
            bn_.x += n2 * a3.x;
            bn_.y += n2 * a3.y;
        }
        L[7 * N + j] = bn_;
    }
}

}  // namespace

template <int N1, int N2>
__global__ void __launch_bounds__(384, 1) theta5_kernel(DevGrid g, PhysArgs A, const double2* tw_g,
                                                     const double2* twh_g) {
    constexpr int N = N1 * N2, G = 32 / N2;
    static_assert(G == 4 || G == 2 || G == 8, "4 lines per round need G in {2, 4, 8}");
    extern __shared__ double2 sm[];
    double2* tw = sm;
    double2* twh = tw + (N + 1);
    for (int q = threadIdx.x; q <= N; q += blockDim.x) {
        tw[q] = tw_g[q];
        twh[q] = twh_g[q];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int gid = lane / N2, t = lane % N2;
    double2* L = twh + (N + 1) + (size_t)warp * 9 * N;
    const int md = g.NTCHOPDIM;
    const int nlines = g.NR * g.NX;
    const double o2 = 2 * A.omega, n2 = A.bv0 * A.bv0;
    if constexpr (G == 4) {
        // Rows arrive by cp.async one round ahead: the three (four) round-1
        // rows of the next line while this line's forward transforms run, the
        // round-2 rows (and, without the linear terms, the round-3 rows into
        // the then unused slots 3 and 8) while phase 1 computes.
        const int mlim = md < g.NTCHOP ? md : g.NTCHOP;
        auto issue_r1 = [&](int ln) {
            const size_t o = (size_t)ln * md;
            if (gid < 3) row_async<N2>(pick_in(A, gid) + o, mlim, L + (size_t)gid * N, t);
            else if (A.linear) row_async<N2>(A.in[9] + o, mlim, L + (size_t)3 * N, t);
            async_commit();
        };
        auto issue_r3 = [&](int ln) {
            const size_t o = (size_t)ln * md;
            if (gid < 2) row_async<N2>(pick_in(A, 7 + gid) + o, mlim, L + (size_t)(gid ? 8 : 3) * N, t);
            async_commit();
        };
        const int line0 = blockIdx.x * nw + warp;
        if (line0 < nlines) issue_r1(line0);
        for (int line = line0; line < nlines; line += gridDim.x * nw) {
            const size_t off = (size_t)line * md;
            const int nxt = line + gridDim.x * nw;
            if (lane < 10 && nxt < nlines && (lane < 9 || A.linear))
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(pick_in(A, lane) + (size_t)nxt * md),
                             "r"((unsigned)(md * sizeof(double2)))
                             : "memory");
            const double rr = g.r[line / g.NX];
            const double ir2 = 1.0 / (rr * rr);
            row_async<N2>(pick_in(A, 3 + gid) + off, mlim, L + (size_t)(4 + gid) * N, t);  // phase 2
            async_commit();
            if (!A.linear) issue_r3(line);
            // phase 1: fields 0-2 (and B with the linear terms) in slots 0-3
            if (A.linear) async_wait<1>();
            else async_wait<2>();
            __syncwarp();
            if (gid < 3 || A.linear)
                grp_inverse5<N1, N2>(nullptr, true, md, g.NTCHOP, tw, twh, L + (size_t)gid * N, t, true);
            else
                idle_group_syncs();
            __syncwarp();
            // phase 2: fields 3-6 in slots 4-7
            if (A.linear) async_wait<0>();
            else async_wait<1>();
            __syncwarp();
            grp_inverse5<N1, N2>(nullptr, true, md, g.NTCHOP, tw, twh, L + (size_t)(4 + gid) * N, t, true);
            __syncwarp();
            theta_products_r2<N>(L, lane, ir2, o2, A.linear);
            __syncwarp();
            // phase 3: RBP -> slot 3, BZ -> slot 8
            if (A.linear) issue_r3(line);
            async_wait<0>();
            __syncwarp();
            if (gid < 2)
                grp_inverse5<N1, N2>(nullptr, true, md, g.NTCHOP, tw, twh, L + (size_t)(gid ? 8 : 3) * N, t, true);
            else
                idle_group_syncs();
            __syncwarp();
            theta_products_r3<N>(L, lane, ir2, n2, A.linear);
            __syncwarp();
            if (nxt < nlines) issue_r1(nxt);  // slots 0-3 are free from here on
            grp_forward5<N1, N2>(L + (size_t)(4 + gid) * N, true, pick_out(A, gid) + off, md, g.NTCHOP, tw, twh, t);
            __syncwarp();
        }
    } else {
    for (int line = blockIdx.x * nw + warp; line < nlines; line += gridDim.x * nw) {
        const size_t off = (size_t)line * md;
        // the warp's next line: lanes 0..9 ask L2 for its ten input rows (md complex each)
        const int nxt = line + gridDim.x * nw;
        if (lane < 10 && nxt < nlines && (lane < 9 || A.linear)) {
            const double2* src = A.in[0];
#pragma unroll
            for (int q = 1; q < 10; ++q)
                if (lane == q) src = A.in[q];
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src + (size_t)nxt * md),
                         "r"((unsigned)(md * sizeof(double2)))
                         : "memory");
        }
        const double rr = g.r[line / g.NX];
        const double ir2 = 1.0 / (rr * rr);
        // phase 1 and 2 (G = 4: one field per group; G = 2: two passes; G = 8: half the groups idle)
        // phase 1: field q (q < 3) or B (q = 3, linear terms only) -> slot q;
        // phase 2: field 3 + q -> slot 4 + q
        for (int rd = 0; rd < 2; ++rd) {
            for (int f0 = 0; f0 < 4; f0 += G) {
                const int q = f0 + gid;
                if (q < 4) {
                    const int f = rd ? 3 + q : (q < 3 ? q : 9);
                    const bool ok = rd || q < 3 || A.linear;
                    grp_inverse5<N1, N2>(ok ? A.in[f] + off : nullptr, ok, md, g.NTCHOP, tw, twh,
                                         L + (size_t)(rd ? 4 + q : q) * N, t);
                } else {
                    idle_group_syncs();
                }
            }
            __syncwarp();
        }
        // round-2 products
        theta_products_r2<N>(L, lane, ir2, o2, A.linear);
        __syncwarp();
        // phase 3
        for (int f0 = 0; f0 < 4; f0 += G) {
            const int q = f0 + gid;
            if (q < 2)  // RBP -> slot 3, BZ -> slot 8
                grp_inverse5<N1, N2>(A.in[7 + q] + off, true, md, g.NTCHOP, tw, twh, L + (size_t)(q ? 8 : 3) * N, t);
            else
                idle_group_syncs();
        }
        __syncwarp();
        theta_products_r3<N>(L, lane, ir2, n2, A.linear);
        __syncwarp();
        // forward transforms of the four results
        for (int f0 = 0; f0 < 4; f0 += G) {
            const int q = f0 + gid;
            if (q < 4)
                grp_forward5<N1, N2>(L + (size_t)(4 + q) * N, true, A.out[q] + off, md, g.NTCHOP, tw, twh, t);
            else
                idle_group_syncs();
        }
        __syncwarp();
    }
    }
}

// Single-field HORFFT on the in-slot transforms of theta5_kernel: each lane
// group owns two line slots and, while it transforms the row in one, the next
// row of its line sequence arrives in the other by cp.async.
//   dir +1: PFP -> PPP (samples written from their slot positions),
//   dir -1: PPP -> PFP (the row copied straight to its slot positions).
template <int N1, int N2>
__global__ void __launch_bounds__(256) horfft5_kernel(DevGrid g, const double2* __restrict__ src,
                                                      double2* __restrict__ dst, const double2* tw_g,
                                                      const double2* twh_g, int dir) {
    constexpr int N = N1 * N2, G = 32 / N2;
    extern __shared__ double2 sm[];
    double2* tw = sm;
    double2* twh = tw + (N + 1);
    for (int q = threadIdx.x; q <= N; q += blockDim.x) {
        tw[q] = tw_g[q];
        twh[q] = twh_g[q];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int gid = lane / N2, t = lane % N2;
    double2* L0 = twh + (N + 1) + (size_t)(warp * G + gid) * 2 * N;
    const int md = g.NTCHOPDIM, mlim = md < g.NTCHOP ? md : g.NTCHOP;
    const int nlines = g.NR * g.NX;
    const int stride = gridDim.x * nw * G;
    // the warp's groups step through their lines together (the transforms
    // synchronise the warp); a group past the last line works on zeros
    auto fetch = [&](int line, double2* L) {
        if (line < nlines) {
            if (dir > 0) {
                row_async<N2>(src + (size_t)line * md, mlim, L, t);
            } else {
                const double2* row = src + (size_t)line * N;
                for (int j = t; j < N; j += N2)
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                     (uint32_t)__cvta_generic_to_shared(L + phys_pos<N1, N2>(j))),
                                 "l"(row + j)
                                 : "memory");
            }
        }
        async_commit();
    };
    const int first = (blockIdx.x * nw + warp) * G + gid;
    fetch(first, L0);
    int slot = 0;
    for (int base = (blockIdx.x * nw + warp) * G; base < nlines; base += stride, slot ^= 1) {
        const int line = base + gid;
        const bool ok = line < nlines;
        double2* L = L0 + slot * N;
        fetch(line + stride, L0 + (slot ^ 1) * N);
        async_wait<1>();
        __syncwarp();
        if (dir > 0) {
            grp_inverse5<N1, N2>(nullptr, ok, md, g.NTCHOP, tw, twh, L, t, true);
            __syncwarp();
            if (ok) {
                double2* out = dst + (size_t)line * N;
                for (int j = t; j < N; j += N2) out[j] = L[phys_pos<N1, N2>(j)];
            }
        } else {
            grp_forward5<N1, N2>(L, ok, ok ? dst + (size_t)line * md : nullptr, md, g.NTCHOP, tw, twh, t);
        }
        __syncwarp();  // the slot is refilled two lines on
    }
    async_wait<0>();
}

static int pp_of(int nth) {
    int pp = (nth + 31) / 32;
    if (pp <= 1) return 1;
    if (pp <= 2) return 2;
    if (pp <= 4) return 4;
    if (pp <= 8) return 8;
    return 16;
}

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

void phys_set_attributes() {
    const int lim = 200 * 1024;
    cudaFuncSetAttribute(theta_fused_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(theta_fused_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(theta_fused_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(theta_fused_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(theta_fused_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_warp_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_warp_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_warp_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_warp_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(horfft_warp_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

// ------------------------------------------------------------------------
// VERFFT with the four-step blocks.  CTA = (r, block of MB = W*G consecutive m);
// group (warp w, gid) owns line m0 + w*G + gid.  PFP rows [r][z][m0..m0+MB)
// move through a shared tile T[z][mloc] so global accesses stay contiguous.
template <int N1, int N2>
__global__ void __launch_bounds__(256) verfft4_kernel(DevGrid g, const double2* src, double2* dst,
                                                      const double2* tw_g, int dir) {
    constexpr int N = N1 * N2, G = 32 / N2;
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int gid = lane / N2, t = lane % N2;
    const int MB = nw * G;
    double2* tw = sm;
    double2* tw2 = tw + (N + 1);                // step-2 twiddles, [k1][t]
    double2* T = tw2 + N;                       // [N][MB + 1]; column mloc is line m0 + mloc
    for (int q = threadIdx.x; q <= N; q += blockDim.x) tw[q] = tw_g[q];
    for (int q = threadIdx.x; q < N; q += blockDim.x) tw2[q] = tw_g[(q % N2) * (q / N2)];
    const int r = blockIdx.y, m0 = blockIdx.x * MB;  // the m-blocks of one r run together
    const int mloc = warp * G + gid, m = m0 + mloc;
    const bool ok = m < g.NTCHOPDIM;
    const int kd = g.NXCHOPDIM, kc = g.NXCHOP, md = g.NTCHOPDIM;
    const int nmb = min(MB, md - m0);
    double2* col = T + mloc;                    // this group's line, stride MB + 1
    const int cs = MB + 1;
    double2 v[N1], o[N1];
    if (dir > 0) {  // PFF [m][r][k] -> PFP [r][z][m]
        __syncthreads();
        const double2* line = src + ((size_t)m * g.NR + r) * kd;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            const int q = t + N2 * n1;
            int kk = -1;
            if (q < kc) kk = q;
            else if (q >= N - kd + kc) kk = q - (N - kd);
            v[n1] = (ok && kk >= 0) ? line[kk] : make_double2(0.0, 0.0);
        }
        fft4::line_fft_inplace<N1, N2, +1>(v, col, tw, t, o, cs, tw2);
#pragma unroll
        for (int q = 0; q < N1; ++q) col[(size_t)fft4::out_index<N1, N2>(t, q) * cs] = o[q];
        __syncthreads();
        for (int e = threadIdx.x; e < N * nmb; e += blockDim.x) {
            const int z = e / nmb, ml = e - z * nmb;
            dst[((size_t)r * N + z) * md + m0 + ml] = T[(size_t)z * cs + ml];
        }
    } else {  // PFP [r][z][m] -> PFF [m][r][k], scaled 1/NX, chopped
        __syncthreads();
        // the tile [z][m0 .. m0 + nmb) by cp.async: every thread keeps its column
        // ml and issues all its rows before waiting (MB divides the block size)
        {
            const int ml = threadIdx.x % MB;
            if (ml < nmb)
                for (int z = threadIdx.x / MB; z < N; z += blockDim.x / MB)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(
                                     (uint32_t)__cvta_generic_to_shared(T + (size_t)z * cs + ml)),
                                 "l"(src + ((size_t)r * N + z) * md + m0 + ml)
                                 : "memory");
            asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[n1] = ok ? col[(size_t)(t + N2 * n1) * cs] : make_double2(0.0, 0.0);
        __syncwarp();
        fft4::line_fft_inplace<N1, N2, -1>(v, col, tw, t, o, cs, tw2);
#pragma unroll
        for (int q = 0; q < N1; ++q) col[(size_t)fft4::out_index<N1, N2>(t, q) * cs] = o[q];
        __syncwarp();
        const double sc = 1.0 / N;
        double2* line = dst + ((size_t)m * g.NR + r) * kd;
        for (int kk = t; kk < kd; kk += N2) {
            const int q = (kk < kc) ? kk : (N - kd + kk);
            double2 y = col[(size_t)q * cs];
            if (ok) line[kk] = make_double2(y.x * sc, y.y * sc);
        }
    }
}

template <int N1, int N2>
static void launch_verfft4(const DevGrid& g, const FFTPlan& p, const double2* src, double2* dst, int dir,
                           cudaStream_t s) {
    constexpr int N = N1 * N2, G = 32 / N2;
    // (+1): MB = 4 G lines per CTA, more and smaller CTAs per SM overlapping their
    // load, FFT and store phases; (-1): 8 warps, longer tile rows per cp.async pass
    int warps = dir > 0 ? 4 : 8;
    auto need = [&](int w) {
        int MB = w * G;
        return (size_t)((N + 1) + N + N * (MB + 1)) * sizeof(double2);
    };
    while (warps > 1 && need(warps) > 110 * 1024) --warps;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(verfft4_kernel<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    const int MB = warps * G;
    dim3 grid((g.NTCHOPDIM + MB - 1) / MB, g.NR);
    verfft4_kernel<N1, N2><<<grid, warps * 32, need(warps), s>>>(g, src, dst, p.tw_x, dir);
    count_launch();
}

bool k_verfft4(const DevGrid& g, const FFTPlan& p, const double2* src, double2* dst, int dir, cudaStream_t s) {
    switch (g.NX) {
        case 16: launch_verfft4<4, 4>(g, p, src, dst, dir, s); return true;
        case 32: launch_verfft4<8, 4>(g, p, src, dst, dir, s); return true;
        case 64: launch_verfft4<8, 8>(g, p, src, dst, dir, s); return true;
        case 128: launch_verfft4<16, 8>(g, p, src, dst, dir, s); return true;
        case 256: launch_verfft4<16, 16>(g, p, src, dst, dir, s); return true;
        case 512: launch_verfft4<32, 16>(g, p, src, dst, dir, s); return true;
        default: return false;
    }
}

template <int N1, int N2>
static void launch_theta4(const DevGrid& g, const FFTPlan& p, const PhysArgs& A, cudaStream_t s) {
    constexpr int N = N1 * N2, G = 32 / N2, TILE = N1 * (N2 + 1);
    const size_t per_warp = (size_t)(11 * N + G * TILE) * sizeof(double2);
    const size_t fixed = 2 * (size_t)(N + 1) * sizeof(double2);
    int warps = (int)((227 * 1024 - fixed) / per_warp);
    if (warps > 8) warps = 8;
    if (warps < 1) warps = 1;
    size_t sm = fixed + warps * per_warp;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(theta4_kernel<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    int nlines = g.NR * g.NX;
    int blocks = std::min((nlines + warps - 1) / warps, sm_count() * 2);
    theta4_kernel<N1, N2><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h);
    count_launch();
}

template <int N1, int N2>
static bool launch_theta5(const DevGrid& g, const FFTPlan& p, const PhysArgs& A, cudaStream_t s) {
    constexpr int N = N1 * N2;
    const size_t per_warp = (size_t)9 * N * sizeof(double2);
    const size_t fixed = 2 * (size_t)(N + 1) * sizeof(double2);
    int warps = (int)((227 * 1024 - fixed) / per_warp);
    if (warps > 12) warps = 12;
    if (warps < 1) return false;
    const size_t sm = fixed + warps * per_warp;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(theta5_kernel<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    const int nlines = g.NR * g.NX;
    const int blocks = std::min((nlines + warps - 1) / warps, sm_count());
    theta5_kernel<N1, N2><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h);
    count_launch();
    return true;
}

void k_theta_fused(const DevGrid& g, const FFTPlan& p, const double2* const in[10], double2* const out[4],
                   double omega, double bv0, int linear, cudaStream_t s) {
    PhysArgs A;
    for (int q = 0; q < 10; ++q) A.in[q] = in[q];
    for (int q = 0; q < 4; ++q) A.out[q] = out[q];
    A.omega = omega;
    A.bv0 = bv0;
    A.linear = linear;
    switch (g.NTH) {
        case 16: if (launch_theta5<4, 4>(g, p, A, s)) return; launch_theta4<4, 4>(g, p, A, s); return;
        case 32: if (launch_theta5<8, 4>(g, p, A, s)) return; launch_theta4<8, 4>(g, p, A, s); return;
        case 64: if (launch_theta5<8, 8>(g, p, A, s)) return; launch_theta4<8, 8>(g, p, A, s); return;
        case 128: if (launch_theta5<16, 8>(g, p, A, s)) return; launch_theta4<16, 8>(g, p, A, s); return;
        case 256: if (launch_theta5<16, 16>(g, p, A, s)) return; launch_theta4<16, 16>(g, p, A, s); return;
        case 512: if (launch_theta5<32, 16>(g, p, A, s)) return; launch_theta4<32, 16>(g, p, A, s); return;
        default: break;
    }
    const int warps = 8;
    size_t sm = (size_t)warps * (3 * g.NTH + 1) * sizeof(double2);
    int nlines = g.NR * g.NX;
    int blocks = std::min((nlines + warps - 1) / warps, sm_count() * 8);
    switch (pp_of(g.NTH)) {
        case 1: theta_fused_kernel<1><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h, p.lt); break;
        case 2: theta_fused_kernel<2><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h, p.lt); break;
        case 4: theta_fused_kernel<4><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h, p.lt); break;
        case 8: theta_fused_kernel<8><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h, p.lt); break;
        default: theta_fused_kernel<16><<<blocks, warps * 32, sm, s>>>(g, A, p.tw_t, p.tw_h, p.lt); break;
    }
    count_launch();
}

template <int N1, int N2>
static void launch_horfft5(const DevGrid& g, const FFTPlan& p, const double2* src, double2* dst, int dir,
                           cudaStream_t s) {
    constexpr int N = N1 * N2, G = 32 / N2;
    const size_t per_warp = (size_t)G * 2 * N * sizeof(double2);
    const size_t fixed = 2 * (size_t)(N + 1) * sizeof(double2);
    // two CTAs per SM
    int warps = (int)((227 * 1024 / 2 - 1024 - fixed) / per_warp);
    if (warps > 8) warps = 8;
    if (warps < 1) warps = 1;
    const size_t sm = fixed + warps * per_warp;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(horfft5_kernel<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    const int nlines = g.NR * g.NX;
    const int per_cta = warps * G;
    const int blocks = std::min((nlines + per_cta - 1) / per_cta, sm_count() * 2);
    horfft5_kernel<N1, N2><<<blocks, warps * 32, sm, s>>>(g, src, dst, p.tw_t, p.tw_h, dir);
    count_launch();
}

void k_horfft_warp(const DevGrid& g, const FFTPlan& p, const double2* src, double2* dst, int dir, cudaStream_t s) {
    switch (g.NTH) {
        case 16: launch_horfft5<4, 4>(g, p, src, dst, dir, s); return;
        case 32: launch_horfft5<8, 4>(g, p, src, dst, dir, s); return;
        case 64: launch_horfft5<8, 8>(g, p, src, dst, dir, s); return;
        case 128: launch_horfft5<16, 8>(g, p, src, dst, dir, s); return;
        case 256: launch_horfft5<16, 16>(g, p, src, dst, dir, s); return;
        case 512: launch_horfft5<32, 16>(g, p, src, dst, dir, s); return;
        default: break;
    }
    const int warps = 8;
    size_t sm = (size_t)warps * (3 * g.NTH + 1) * sizeof(double2);
    int nlines = g.NR * g.NX;
    int blocks = std::min((nlines + warps - 1) / warps, sm_count() * 8);
    switch (pp_of(g.NTH)) {
        case 1: horfft_warp_kernel<1><<<blocks, warps * 32, sm, s>>>(g, src, dst, p.tw_t, p.tw_h, p.lt, dir); break;
        case 2: horfft_warp_kernel<2><<<blocks, warps * 32, sm, s>>>(g, src, dst, p.tw_t, p.tw_h, p.lt, dir); break;
        case 4: horfft_warp_kernel<4><<<blocks, warps * 32, sm, s>>>(g, src, dst, p.tw_t, p.tw_h, p.lt, dir); break;
        case 8: horfft_warp_kernel<8><<<blocks, warps * 32, sm, s>>>(g, src, dst, p.tw_t, p.tw_h, p.lt, dir); break;
        default: horfft_warp_kernel<16><<<blocks, warps * 32, sm, s>>>(g, src, dst, p.tw_t, p.tw_h, p.lt, dir); break;
    }
    count_launch();
}

}  // namespace mlegs
