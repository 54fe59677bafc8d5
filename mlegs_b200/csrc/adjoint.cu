// Adjoint (vector-Jacobian products) of the AB2-CN step on the device.
//
// The reference has no adjoint.  These are the transposes of this library's
// forward operators for the real inner product <a, b> = sum(Re a Re b +
// Im a Im b) over the stored complex entries (plus LN_a LN_b for the log
// terms), composed into the VJPs of CALC_BOUSSI_FORCE (mod_boussinesq.f90:
// 317-410), one steady STEP_BOUSSI_AB_CN with VISC%SW = 1 (mod_march.f90:
// 609-661), the Richardson start-up RICH_BOUSSI_FE_BE (535-606), the seeded
// initial state and the energy objective of the gradient workload.  Most
// transposes are forward kernels of the library with other coefficients:
//   RTRAN(+1)^T   the fold GEMM with PF and no Gauss weights (EO fold), plus
//                 LN_bar = sum_i Re Y(i, 0, 0) (-log(1 - x_i));
//   RTRAN(-1)^T   the RTRAN(+1) GEMM without the log term, rows times w_i;
//   VERFFT(+1)^T  NX VERFFT(-1);  VERFFT(-1)^T  VERFFT(+1) / NX;
//   HORFFT(+1)^T  HORFFT(-1), modes times 2 NTH (m = 0, imaginary part
//                 dropped) and 4 NTH (m > 0);  HORFFT(-1)^T  HORFFT(+1) of the
//                 modes times 1/(2 NTH) (m = 0) and 1/(4 NTH) (m > 0);
//   XXDX^T, MULXM^T, DEL2^T  the band kernels on the transposed band tables
//                 (the truncated band matrix's transpose is the truncation of
//                 the transposed band), log-term rows folded into LN_bar;
//   PROJECT^T     the RTRAN(+1) GEMM with the V, D, T weights (rows padded to
//                 PF's stride), the mirror half negated for the OE segments,
//                 VEL2PLN^T and the far-field transpose;
//   IDEL2LN^T, IHELM^T  U^T then L^T substitutions with the stored factors.
// The pointwise products' adjoints (VPRODSUB, VDOTPSUB) are kernels here.
// FP64 contexts only.
#include "ctx_internal.h"

namespace mlegs {
namespace {

inline unsigned nb(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ int nrc(const DevGrid& g, int m, int pad) {
    const int v = g.NRCHOP + pad - m;
    return v < 0 ? 0 : v;
}

// out_ln (=|+=) sum_{r < 3} c_r Re y(r, m = 0, k = 0) of an FFF field.
__global__ void ln_rows_kernel(const DevGrid g, const double2* y, double c0, double c1, double c2, double* out,
                               int accumulate) {
    const size_t st = g.NXCHOPDIM;
    const double v = c0 * y[0].x + c1 * y[st].x + c2 * y[2 * st].x;
    *out = accumulate ? *out + v : v;
}

// y(0, 0, 0) = ln s (accumulate 0, imaginary part 0) or Re y(0, 0, 0) += ln s.
__global__ void ln_to_coef_kernel(double2* y, const double* ln, double s, int accumulate) {
    if (accumulate) y[0].x += (*ln) * s;
    else y[0] = make_double2((*ln) * s, 0.0);
}

// Block-wide sum of one value per thread (blockDim a multiple of 32, at most 256).
__device__ double block_sum(double v, double* part) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    __syncthreads();
    return t;
}

// LN_bar of RTRAN(+1): sum_{i < NR} Re Y(m = 0, i, k = 0) (-log(1 - x_i)) of a PFF field.
__global__ void ln_lnx_kernel(const DevGrid g, const double2* y, double* out) {
    __shared__ double part[8];
    double s = 0.0;
    for (int i = threadIdx.x; i < g.NR; i += blockDim.x) s += y[(size_t)i * g.NXCHOPDIM].x * g.lnx[i];
    s = block_sum(s, part);
    if (threadIdx.x == 0) *out = s;
}

// PFF rows times the Gauss weights: y(m, r, k) *= w_r.
__global__ void pff_rows_w_kernel(const DevGrid g, double2* y) {
    const size_t n = (size_t)g.NTCHOPDIM * g.NR * g.NXCHOPDIM;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double w = g.w[(t / g.NXCHOPDIM) % g.NR];
    y[t] = make_double2(y[t].x * w, y[t].y * w);
}

// PFP [r][z][m]: mode m = 0 times s0 (its imaginary part dropped when
// drop_im0), m > 0 times s1.
__global__ void pfp_mscale_kernel(const DevGrid g, double2* y, double s0, double s1, int drop_im0) {
    const size_t n = (size_t)g.NR * g.NX * g.NTCHOPDIM;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double2 v = y[t];
    if (t % g.NTCHOPDIM == 0) y[t] = make_double2(v.x * s0, drop_im0 ? 0.0 : v.y * s0);
    else y[t] = make_double2(v.x * s1, v.y * s1);
}

// out (PFF) (+)= t on rows r < NRH and -t on the mirror rows: the transpose of
// an OE fold from the RTRAN(+1) product of its cotangent.
__global__ void pff_mirror_kernel(const DevGrid g, double2* out, const double2* t, int accumulate) {
    const size_t n = (size_t)g.NTCHOPDIM * g.NR * g.NXCHOPDIM;
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const double s = ((q / g.NXCHOPDIM) % g.NR) < (size_t)g.NRH ? 1.0 : -1.0;
    const double2 o = accumulate ? out[q] : make_double2(0.0, 0.0);
    out[q] = make_double2(o.x + s * t[q].x, o.y + s * t[q].y);
}

// VEL2PLN (mod_legops.f90:2277-2339) changes the (m, k) = (0, 0) PFF line of
// RUP as line -> line - v (c . Re line), c the PSI%LN functional (Lpff) and
// v(i) = -(PF_0(i)/NORM(1) +- PF_1(i)/NORM(2)) (+ for i < NRH, - on the mirror
// rows).  Its transpose: line -> line - c (v . Re line).
__global__ void vel2pln_T_kernel(const DevGrid g, double2* y, const double* c) {
    __shared__ double part[8];
    const int nr = g.NR, nrh = g.NRH;
    double s = 0.0;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        const int ii = i < nrh ? i : nr - 1 - i;
        const double a = g.pf[ii] / g.norm0[0], b = g.pf[(size_t)g.NRH + ii] / g.norm0[1];
        const double v = i < nrh ? -(a + b) : -(a - b);
        s += v * y[(size_t)i * g.NXCHOPDIM].x;
    }
    const double dot = block_sum(s, part);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) y[(size_t)i * g.NXCHOPDIM].x -= c[i] * dot;
}

// Transpose of the far-field fix a(0, 0, k) -= sum_{n < nr} AT1(n) a(n, 0, k) / AT1(0)
// (CALCAT1, mod_scalar3.f90:286-310), in place on an FFF field: rows 1 .. nr-1
// of m = 0 -= AT1(n)/AT1(0) row 0, then row 0 = 0.
// CALCAT1's row-0 fix transposed: y(n, 0, k) -= AT1(n)/AT1(0) y(0, 0, k) for
// 1 <= n < nr, then y(0, 0, k) = 0.  A block is 32 k by 8 row groups; every
// thread reads y(0, 0, k) before the barrier, row 0 is zeroed after it.
__global__ void __launch_bounds__(256) farfield_T_kernel(const DevGrid g, double2* y, int nr) {
    const int kl = threadIdx.x & 31, ny = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + kl;
    const bool ok = k < g.NXCHOPDIM;
    const size_t st = g.NXCHOPDIM;
    const double2 y0 = ok ? y[k] : make_double2(0.0, 0.0);
    __syncthreads();
    if (!ok) return;
    for (int n = 1 + ny; n < nr && n < g.NRCHOPDIM; n += 8) {
        const double f = g.at1[n] / g.at1[0];
        const double2 v = y[(size_t)n * st + k];
        y[(size_t)n * st + k] = make_double2(v.x - f * y0.x, v.y - f * y0.y);
    }
    if (ny == 0) y[k] = make_double2(0.0, 0.0);
}

// Transposed banded solves with the stored unpivoted factors A = L U of the
// forward solves (solve.cu: F5 [row][5][system] = L(r, r-2), L(r, r-1),
// U(r, r), U(r, r+1), U(r, r+2); F7 [row][7][k] = L(r, r-3 .. r-1), U(r, r ..
// r+3)).  A^T x = y is U^T z = y, then L^T x = z.  One thread per (system, real
// or imaginary part), in place on the FFF field, rows from the system size on
// left as they are.
//   kind 0  IDEL2LN: 5-band factors for every (m, k);
//   kind 2  IHELM: m >= 1 5-band; m = 0 the forward solves (H XM) v = rhs on
//           NN - 1 rows and returns XM v (NN rows), so the transpose forms
//           w = XM^T y, solves (H XM)^T on NN - 1 rows and zeroes row NN - 1.
// The substitutions run in load blocks of TB (TW for the 7-band systems)
// rows: a block's right-hand sides and factors are loaded together, the
// diagonal's reciprocal and the scaled off-diagonals are formed off the
// recurrence, which then costs one dependent FMA per row.  wpad idle threads
// after the 7-band m = 0 systems of kind 2 keep them in warps of their own.
__global__ void __launch_bounds__(128) solve_T_kernel(const DevGrid g, const double* __restrict__ F5,
                                                      const double* __restrict__ F7, double2* yfield, int kind,
                                                      int pad, int wpad) {
    constexpr int TB = 16, TW = 8;
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int nw = 2 * g.NXCHOPDIM;
    if (wpad) {
        if (u >= nw && u < nw + wpad) return;
        if (u >= nw) u -= wpad;
    }
    const int t = u >> 1, comp = u & 1;
    if (t >= nsys) return;
    const int k = t % g.NXCHOPDIM, m = t / g.NXCHOPDIM;
    const int nn = nrc(g, m, pad);
    double* col = (double*)(yfield + (size_t)m * g.NRCHOPDIM * g.NXCHOPDIM + k) + comp;
    const size_t st = 2 * (size_t)g.NXCHOPDIM;
    if (!(m == 0 && kind == 2)) {
        const int size = nn;
        // U^T z = y: z(r) = (y(r) - U(r-1, r) z(r-1) - U(r-2, r) z(r-2)) / U(r, r)
        double z1 = 0.0, z2 = 0.0;
        for (int r0 = 0; r0 < size; r0 += TB) {
            double yv[TB], a1[TB], a2[TB];
#pragma unroll
            for (int q = 0; q < TB; ++q) {
                const int r = r0 + q;
                const bool ok = r < size;
                yv[q] = ok ? col[(size_t)r * st] : 0.0;
                const double d = ok ? F5[((size_t)r * 5 + 2) * nsys + t] : 1.0;
                a1[q] = (ok && r >= 1) ? F5[((size_t)(r - 1) * 5 + 3) * nsys + t] : 0.0;
                a2[q] = (ok && r >= 2) ? F5[((size_t)(r - 2) * 5 + 4) * nsys + t] : 0.0;
                const double ri = 1.0 / d;
                yv[q] = __dmul_rn(yv[q], ri);
                a1[q] = __dmul_rn(a1[q], ri);
                a2[q] = __dmul_rn(a2[q], ri);
            }
#pragma unroll
            for (int q = 0; q < TB; ++q) {
                if (r0 + q >= size) break;
                const double v = __fma_rn(-a1[q], z1, __fma_rn(-a2[q], z2, yv[q]));
                col[(size_t)(r0 + q) * st] = v;
                z2 = z1;
                z1 = v;
            }
        }
        // L^T x = z: x(r) = z(r) - L(r+1, r) x(r+1) - L(r+2, r) x(r+2)
        double x1 = 0.0, x2 = 0.0;
        for (int r1 = size - 1; r1 >= 0; r1 -= TB) {
            double zv[TB], e1[TB], e2[TB];
#pragma unroll
            for (int q = 0; q < TB; ++q) {
                const int r = r1 - q;
                const bool ok = r >= 0;
                zv[q] = ok ? col[(size_t)r * st] : 0.0;
                e1[q] = (ok && r + 1 < size) ? F5[((size_t)(r + 1) * 5 + 1) * nsys + t] : 0.0;
                e2[q] = (ok && r + 2 < size) ? F5[((size_t)(r + 2) * 5 + 0) * nsys + t] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < TB; ++q) {
                const int r = r1 - q;
                if (r < 0) break;
                const double v = __fma_rn(-e1[q], x1, __fma_rn(-e2[q], x2, zv[q]));
                col[(size_t)r * st] = v;
                x2 = x1;
                x1 = v;
            }
        }
        return;
    }
    if (nn <= 0) return;
    // w = XM^T y: w(r) = y(r) + XM(r+1, r) y(r+1) + XM(r-1, r) y(r-1), with
    // XM(l, l-1) = sub(l), XM(l, l+1) = super(l) (the m = 0 table [row][2])
    const double* xm = g.xm;
    {
        double prev = 0.0;
        for (int r0 = 0; r0 < nn; r0 += TW) {
            double yv[TW + 1];
#pragma unroll
            for (int q = 0; q <= TW; ++q) yv[q] = (r0 + q < nn) ? col[(size_t)(r0 + q) * st] : 0.0;
#pragma unroll
            for (int q = 0; q < TW; ++q) {
                const int r = r0 + q;
                if (r >= nn) break;
                double v = yv[q];
                if (r + 1 < nn) v = __fma_rn(xm[(size_t)(r + 1) * 2 + 0], yv[q + 1], v);
                if (r >= 1) v = __fma_rn(xm[(size_t)(r - 1) * 2 + 1], prev, v);
                col[(size_t)r * st] = v;
                prev = yv[q];
            }
        }
    }
    const int size = nn - 1;
    const size_t NK = g.NXCHOPDIM;
    auto f7 = [&](int r, int j) { return F7[((size_t)r * 7 + j) * NK + k]; };
    double z1 = 0.0, z2 = 0.0, z3 = 0.0;
    for (int r0 = 0; r0 < size; r0 += TW) {
        double yv[TW], a1[TW], a2[TW], a3[TW];
#pragma unroll
        for (int q = 0; q < TW; ++q) {
            const int r = r0 + q;
            const bool ok = r < size;
            yv[q] = ok ? col[(size_t)r * st] : 0.0;
            const double d = ok ? f7(r, 3) : 1.0;
            a1[q] = (ok && r >= 1) ? f7(r - 1, 4) : 0.0;
            a2[q] = (ok && r >= 2) ? f7(r - 2, 5) : 0.0;
            a3[q] = (ok && r >= 3) ? f7(r - 3, 6) : 0.0;
            const double ri = 1.0 / d;
            yv[q] = __dmul_rn(yv[q], ri);
            a1[q] = __dmul_rn(a1[q], ri);
            a2[q] = __dmul_rn(a2[q], ri);
            a3[q] = __dmul_rn(a3[q], ri);
        }
#pragma unroll
        for (int q = 0; q < TW; ++q) {
            if (r0 + q >= size) break;
            const double v = __fma_rn(-a1[q], z1, __fma_rn(-a2[q], z2, __fma_rn(-a3[q], z3, yv[q])));
            col[(size_t)(r0 + q) * st] = v;
            z3 = z2;
            z2 = z1;
            z1 = v;
        }
    }
    double x1 = 0.0, x2 = 0.0, x3 = 0.0;
    for (int r1 = size - 1; r1 >= 0; r1 -= TW) {
        double zv[TW], c1[TW], c2[TW], c3[TW];
#pragma unroll
        for (int q = 0; q < TW; ++q) {
            const int r = r1 - q;
            const bool ok = r >= 0;
            zv[q] = ok ? col[(size_t)r * st] : 0.0;
            c1[q] = (ok && r + 1 < size) ? f7(r + 1, 2) : 0.0;
            c2[q] = (ok && r + 2 < size) ? f7(r + 2, 1) : 0.0;
            c3[q] = (ok && r + 3 < size) ? f7(r + 3, 0) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < TW; ++q) {
            const int r = r1 - q;
            if (r < 0) break;
            const double v = __fma_rn(-c1[q], x1, __fma_rn(-c2[q], x2, __fma_rn(-c3[q], x3, zv[q])));
            col[(size_t)r * st] = v;
            x3 = x2;
            x2 = x1;
            x1 = v;
        }
    }
    col[(size_t)size * st] = 0.0;
}

// solve_T_kernel for small systems (NRCHOP + pad <= 72 rows): one warp takes 16
// systems, copies their factor rows and columns into shared memory in one
// burst of cp.async copies, and runs the same substitutions there; rows from
// the system size on are left as they are.  Blocks [0, nb0) hold the 7-band
// m = 0 systems of kind 2.  Shared memory per block: R x 144 doubles.
__global__ void __launch_bounds__(32) solve_T_small_kernel(const DevGrid g, const double* __restrict__ F5,
                                                           const double* __restrict__ F7, double2* yfield, int kind,
                                                           int pad, int t_begin, int nb0) {
    extern __shared__ __align__(16) double sms[];
    const int R = g.NRCHOP + pad;
    double* Fs = sms;                         // [R][7][16]
    double2* Xs = (double2*)(sms + R * 112);  // [R][16]
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int lane = threadIdx.x, sy = lane >> 1, comp = lane & 1;
    const bool wide = (int)blockIdx.x < nb0;
    const int tb = wide ? blockIdx.x * 16 : t_begin + (blockIdx.x - nb0) * 16;
    const int nsb = min(16, (wide ? t_begin : nsys) - tb);
    const size_t NK = g.NXCHOPDIM;
    if (wide) {
        for (int e = lane; e < R * 112; e += 32) {
            const int r = e / 112, j = (e / 16) % 7, q = e % 16;
            if (q < nsb)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                                 (uint32_t)__cvta_generic_to_shared(Fs + e)),
                             "l"(F7 + ((size_t)r * 7 + j) * NK + tb + q)
                             : "memory");
        }
    } else {
        for (int e = lane; e < R * 80; e += 32) {
            const int r = e / 80, j = (e / 16) % 5, q = e % 16;
            if (q < nsb)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                                 (uint32_t)__cvta_generic_to_shared(Fs + (r * 7 + j) * 16 + q)),
                             "l"(F5 + ((size_t)r * 5 + j) * nsys + tb + q)
                             : "memory");
        }
    }
    for (int e = lane; e < R * 16; e += 32) {
        const int r = e / 16, q = e % 16;
        if (q < nsb) {
            const int tq = tb + q, mq = tq / g.NXCHOPDIM, kq = tq - mq * g.NXCHOPDIM;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(Xs + e)),
                         "l"(yfield + (size_t)mq * g.NRCHOPDIM * NK + (size_t)r * NK + kq)
                         : "memory");
        }
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    if (sy >= nsb) return;
    const int t = tb + sy, k = t % g.NXCHOPDIM, m = t / g.NXCHOPDIM;
    const int nn = nrc(g, m, pad);
    double* X = (double*)Xs + sy * 2 + comp;  // row r at X[r * 32]
    auto F = [&](int r, int j) { return Fs[(r * 7 + j) * 16 + sy]; };
    int rows_out = 0;
    if (!wide) {
        const int size = nn;
        double z1 = 0.0, z2 = 0.0;
        for (int r = 0; r < size; ++r) {
            const double ri = 1.0 / F(r, 2);
            const double a1 = r >= 1 ? __dmul_rn(F(r - 1, 3), ri) : 0.0;
            const double a2 = r >= 2 ? __dmul_rn(F(r - 2, 4), ri) : 0.0;
            const double v = __fma_rn(-a1, z1, __fma_rn(-a2, z2, __dmul_rn(X[r * 32], ri)));
            X[r * 32] = v;
            z2 = z1;
            z1 = v;
        }
        double x1 = 0.0, x2 = 0.0;
        for (int r = size - 1; r >= 0; --r) {
            const double e1 = r + 1 < size ? F(r + 1, 1) : 0.0;
            const double e2 = r + 2 < size ? F(r + 2, 0) : 0.0;
            const double v = __fma_rn(-e1, x1, __fma_rn(-e2, x2, X[r * 32]));
            X[r * 32] = v;
            x2 = x1;
            x1 = v;
        }
        rows_out = size;
    } else if (nn > 0) {
        // w = XM^T y, then the transposed 7-band solve on NN - 1 rows, row NN - 1 zeroed
        const double* xm = g.xm;
        double prev = 0.0;
        for (int r = 0; r < nn; ++r) {
            const double yr = X[r * 32];
            double v = yr;
            if (r + 1 < nn) v = __fma_rn(xm[(size_t)(r + 1) * 2 + 0], X[(r + 1) * 32], v);
            if (r >= 1) v = __fma_rn(xm[(size_t)(r - 1) * 2 + 1], prev, v);
            X[r * 32] = v;
            prev = yr;
        }
        const int size = nn - 1;
        double z1 = 0.0, z2 = 0.0, z3 = 0.0;
        for (int r = 0; r < size; ++r) {
            const double ri = 1.0 / F(r, 3);
            const double a1 = r >= 1 ? __dmul_rn(F(r - 1, 4), ri) : 0.0;
            const double a2 = r >= 2 ? __dmul_rn(F(r - 2, 5), ri) : 0.0;
            const double a3 = r >= 3 ? __dmul_rn(F(r - 3, 6), ri) : 0.0;
            const double v = __fma_rn(-a1, z1, __fma_rn(-a2, z2, __fma_rn(-a3, z3, __dmul_rn(X[r * 32], ri))));
            X[r * 32] = v;
            z3 = z2;
            z2 = z1;
            z1 = v;
        }
        double x1 = 0.0, x2 = 0.0, x3 = 0.0;
        for (int r = size - 1; r >= 0; --r) {
            const double c1 = r + 1 < size ? F(r + 1, 2) : 0.0;
            const double c2 = r + 2 < size ? F(r + 2, 1) : 0.0;
            const double c3 = r + 3 < size ? F(r + 3, 0) : 0.0;
            const double v = __fma_rn(-c1, x1, __fma_rn(-c2, x2, __fma_rn(-c3, x3, X[r * 32])));
            X[r * 32] = v;
            x3 = x2;
            x2 = x1;
            x1 = v;
        }
        X[size * 32] = 0.0;
        rows_out = nn;
    }
    double* col = (double*)(yfield + (size_t)m * g.NRCHOPDIM * NK + k) + comp;
    const size_t st = 2 * NK;
    for (int r = 0; r < rows_out; ++r) col[(size_t)r * st] = X[r * 32];
}

// Adjoints of VPRODSUB's cross product and VDOTPSUB's dot product
// (mod_legops.f90:2105-2130, 2207-2225), pointwise on the packed physical
// samples [r][z][j] (real and imaginary parts are separate samples):
//   N_r = u2 w3 - u3 w2, N_t = u3 w1 - u1 w3, N_z = (u1 w2 - u2 w1) / r^2;
//   D = (a1 b1 + a2 b2) / r^2 + a3 b3.
struct P3 {
    const double2* a[3];
};
struct Q3 {
    double2* a[3];
};
__global__ void vprod_T_kernel(const DevGrid g, P3 U, P3 W, P3 B, Q3 Uo, Q3 Wo) {
    const size_t n = (size_t)g.NR * g.NX * g.NTH;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int r = (int)(t / ((size_t)g.NX * g.NTH));
    const double ir2 = 1.0 / (g.r[r] * g.r[r]);
    double u[2][3], w[2][3], b[2][3];
    for (int q = 0; q < 3; ++q) {
        const double2 uv = U.a[q][t], wv = W.a[q][t], bv = B.a[q][t];
        u[0][q] = uv.x;
        u[1][q] = uv.y;
        w[0][q] = wv.x;
        w[1][q] = wv.y;
        b[0][q] = bv.x;
        b[1][q] = bv.y;
    }
    double du[2][3], dw[2][3];
    for (int p = 0; p < 2; ++p) {
        const double b1 = b[p][0], b2 = b[p][1], b3r = b[p][2] * ir2;
        const double u1 = u[p][0], u2 = u[p][1], u3 = u[p][2];
        const double w1 = w[p][0], w2 = w[p][1], w3 = w[p][2];
        du[p][0] = -b2 * w3 + b3r * w2;
        du[p][1] = b1 * w3 - b3r * w1;
        du[p][2] = -b1 * w2 + b2 * w1;
        dw[p][0] = b2 * u3 - b3r * u2;
        dw[p][1] = -b1 * u3 + b3r * u1;
        dw[p][2] = b1 * u2 - b2 * u1;
    }
    for (int q = 0; q < 3; ++q) {
        Uo.a[q][t] = make_double2(du[0][q], du[1][q]);
        Wo.a[q][t] = make_double2(dw[0][q], dw[1][q]);
    }
}

// a_bar(q) += w_q b_q y and b_bar(q) = w_q a_q y, w = (1/r^2, 1/r^2, 1).
__global__ void vdotp_T_kernel(const DevGrid g, P3 A, P3 B, const double2* y, Q3 Ao, Q3 Bo) {
    const size_t n = (size_t)g.NR * g.NX * g.NTH;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int r = (int)(t / ((size_t)g.NX * g.NTH));
    const double ir2 = 1.0 / (g.r[r] * g.r[r]);
    const double2 yv = y[t];
    for (int q = 0; q < 3; ++q) {
        const double wq = q < 2 ? ir2 : 1.0;
        const double2 av = A.a[q][t], bv = B.a[q][t];
        const double2 o = Ao.a[q][t];
        Ao.a[q][t] = make_double2(o.x + wq * bv.x * yv.x, o.y + wq * bv.y * yv.y);
        Bo.a[q][t] = make_double2(wq * av.x * yv.x, wq * av.y * yv.y);
    }
}

// y = s W_r R(m, r, k) on PFF with W_r = w_r [/ (1 - x_r)^2] and m = 0 halved:
// the per-entry weights of the PRODCT_MK / L2NORM_MK quadratures of
// CALC_BOUSSI_ENERGY and CALC_BOUSSI_PE (mod_boussinesq.f90:112-206).
__global__ void pff_quadw_kernel(const DevGrid g, const double2* R, double2* y, double s, int inv_om2) {
    const size_t n = (size_t)g.NTCHOPDIM * g.NR * g.NXCHOPDIM;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int r = (int)((t / g.NXCHOPDIM) % g.NR);
    const int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NR));
    double w = g.w[r] * s * (m == 0 ? 0.5 : 1.0);
    if (inv_om2) {
        const double om = 1.0 - g.x[r];
        w /= om * om;
    }
    y[t] = make_double2(R[t].x * w, R[t].y * w);
}

// *out += sum over the FFF entries of Re a Re b + Im a Im b.
__global__ void fff_dot_kernel(const DevGrid g, const double2* a, const double2* b, double* out) {
    __shared__ double part[8];
    const size_t n = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    double s = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        s += a[t].x * b[t].x + a[t].y * b[t].y;
    s = block_sum(s, part);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// Zero the (m, k) = (0, 0) column of an FFF field (the fluctuation part).
__global__ void zero_col00_kernel(const DevGrid g, double2* y) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < g.NRCHOPDIM) y[(size_t)n * g.NXCHOPDIM] = make_double2(0.0, 0.0);
}

// V, D or T [m][NRCHOPDIM][NRH] copied into PF's row stride [m][NRCHOPDIM + 1][NRH]
// (last row zero), so that the RTRAN(+1) GEMM applies their transposes.
__global__ void pad_rows_kernel(const DevGrid g, const double* W, double* Wp) {
    const size_t n = (size_t)g.NTCHOPDIM * (g.NRCHOPDIM + 1) * g.NRH;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % g.NRH);
    const int row = (int)((t / g.NRH) % (g.NRCHOPDIM + 1));
    const int m = (int)(t / ((size_t)g.NRH * (g.NRCHOPDIM + 1)));
    Wp[t] = row < g.NRCHOPDIM ? W[((size_t)m * g.NRCHOPDIM + row) * g.NRH + i] : 0.0;
}

}  // namespace
}  // namespace mlegs

// ---------------------------------------------------------------------------
// Host side: the transposes and the VJPs over a context's fields and kernels.
namespace {

struct Adj {
    mlegs_ctx* c;
    explicit Adj(mlegs_ctx* ctx) : c(ctx) {}
    const DevGrid& g() const { return c->g; }
    cudaStream_t s() const { return c->s; }

    // Tables formed once per context, outside graph capture.
    void prepare() {
        if (c->split_S) throw ApiError(MLEGS_ERR_STATE, "adjoint: FP64 contexts only");
        if (c->adj_ready) return;
        c->no_capture("adjoint");
        const Dims& d = c->d;
        const int NB = d.NRCHOPDIM + 2;
        CK(cudaStreamSynchronize(c->s));
        // 5-band table with centre 2: T^T(n, n + j - 2) = T(n + j - 2, n), entry 4 - j of that row
        auto tr5 = [&](const double* dev) {
            const int w = 5, cc = 2;
            std::vector<double> h((size_t)d.NTCHOPDIM * NB * w), out(h.size(), 0.0);
            CK(cudaMemcpy(h.data(), dev, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int m = 0; m < d.NTCHOPDIM; ++m)
                for (int n = 0; n < NB; ++n)
                    for (int j = 0; j < w; ++j) {
                        const int src = n + (j - cc), sj = 2 * cc - j;
                        if (src < 0 || src >= NB) continue;
                        out[((size_t)m * NB + n) * w + j] = h[((size_t)m * NB + src) * w + sj];
                    }
            double* dp = dalloc<double>(out.size());
            CK(cudaMemcpy(dp, out.data(), out.size() * sizeof(double), cudaMemcpyHostToDevice));
            return (const double*)dp;
        };
        // (sub, super) tables: T^T(n, n-1) = super(n-1), T^T(n, n+1) = sub(n+1)
        auto tr3 = [&](const double* dev) {
            std::vector<double> h((size_t)d.NTCHOPDIM * NB * 2), out(h.size(), 0.0);
            CK(cudaMemcpy(h.data(), dev, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int m = 0; m < d.NTCHOPDIM; ++m)
                for (int n = 0; n < NB; ++n) {
                    if (n >= 1) out[((size_t)m * NB + n) * 2 + 0] = h[((size_t)m * NB + n - 1) * 2 + 1];
                    if (n + 1 < NB) out[((size_t)m * NB + n) * 2 + 1] = h[((size_t)m * NB + n + 1) * 2 + 0];
                }
            double* dp = dalloc<double>(out.size());
            CK(cudaMemcpy(dp, out.data(), out.size() * sizeof(double), cudaMemcpyHostToDevice));
            return (const double*)dp;
        };
        c->gT = c->g;
        c->gT.xxdx = tr3(c->g.xxdx);
        c->gT.xm = tr3(c->g.xm);
        c->gT.del2h = tr5(c->g.del2h);
        CK(cudaMemcpy(c->adj_n0, c->g.norm0, 3 * sizeof(double), cudaMemcpyDeviceToHost));
        const size_t np = (size_t)d.NTCHOPDIM * (d.NRCHOPDIM + 1) * d.NRH;
        const double* W[3] = {c->V, c->D, c->T};
        for (int q = 0; q < 3; ++q) {
            c->adj_w[q] = dalloc<double>(np);
            pad_rows_kernel<<<nb(np, 256), 256, 0, c->s>>>(c->g, W[q], c->adj_w[q]);
            count_launch();
        }
        c->adj_dot = dalloc<double>(1);
        CK(cudaStreamSynchronize(c->s));
        c->adj_ready = true;
    }

    // Temporaries; the pool grows on demand (outside capture), recorded in the
    // snapshot that restore() puts back at the end of the call.
    void grow() {
        c->no_capture("adjoint temporaries");
        Field* f = c->new_field(MLEGS_FFF, false);
        c->temps.push_back(f);
        c->snap.push_back(f->data);
        c->pool.push_back(f);
    }
    void reserve(size_t n) {
        while (c->pool.size() < n) grow();
    }
    Field* tmp() {
        if (c->pool.empty()) grow();
        return c->tmp(MLEGS_FFF);
    }
    void rel(Field* f) { c->rel(f); }
    void rel(std::initializer_list<Field*> fs) {
        for (Field* f : fs) c->rel(f);
    }
    void zero(Field* f) {
        k_fill(f->data, c->fff(), s());
        f->space = MLEGS_FFF;
        c->ln_zero(f);
    }
    void copy(Field* dst, const Field* src) {
        if (dst == src) return;
        k_copy_ln(dst->data, src->data, c->d.elems(src->space), dst->ln, src->ln, s());
        dst->space = src->space;
    }
    void add(Field* y, const Field* x, double a = 1.0) {  // y += a x, E and LN
        k_axpby_ln(y->data, a, x->data, 0.0, nullptr, 1.0, c->d.elems(y->space),
                   y->ln, a, x->ln, 0.0, nullptr, 1.0, s());
    }
    void scale(Field* y, double a) {
        k_axpby_ln(y->data, a, y->data, 0.0, nullptr, 0.0, c->d.elems(y->space),
                   y->ln, a, y->ln, 0.0, nullptr, 0.0, s());
    }
    void chop(Field* f, int pad) { c->chopdo(f, pad); }
    void ln_rows(const Field* y, Field* out, double c0, double c1, double c2, bool acc) {
        ln_rows_kernel<<<1, 1, 0, s()>>>(g(), y->data, c0, c1, c2, out->ln, acc ? 1 : 0);
        count_launch();
    }
    void ln_to_coef(Field* y, const double* ln, double sc, bool acc) {
        ln_to_coef_kernel<<<1, 1, 0, s()>>>(y->data, ln, sc, acc ? 1 : 0);
        count_launch();
    }
    const double* n0() const { return c->adj_n0; }

    // ------------------------------------------------------------- transforms
    // RTRAN(+1)^T at CHOPSET(pad): y (PFF) -> out (FFF with LN_bar)
    void rtran_p_T(const Field* y, Field* out, int pad) {
        k_fold_gemm(g(), g().pf, c->d.NRCHOPDIM + 1, y->data, out->data, 0, 0, 0, pad, s());
        out->space = MLEGS_FFF;
        chop(out, pad);
        ln_lnx_kernel<<<1, 256, 0, s()>>>(g(), y->data, out->ln);
        count_launch();
    }
    // RTRAN(-1)^T at CHOPSET(pad): y (FFF) -> out (PFF)
    void rtran_m_T(const Field* y, Field* out, int pad) {
        k_rtran_b2p(g(), y->data, out->data, nullptr, pad, s());
        pff_rows_w_kernel<<<nb(c->d.pff(), 256), 256, 0, s()>>>(g(), out->data);
        count_launch();
        out->space = MLEGS_PFF;
        c->ln_zero(out);
    }
    void verfft(const double2* src, double2* dst, int dir) {
        if (!k_verfft4(g(), c->fft, src, dst, dir, s())) {
            if (dir > 0) k_verfft_b(g(), c->fft, src, dst, s());
            else k_verfft_f(g(), c->fft, src, dst, s());
        }
    }
    void verfft_p_T(const Field* y, Field* out) {  // PFP -> PFF: NX VERFFT(-1)
        verfft(y->data, out->data, -1);
        k_axpby(out->data, (double)c->d.NX, out->data, 0.0, nullptr, 0.0, c->d.pff(), s());
        out->space = MLEGS_PFF;
        c->ln_zero(out);
    }
    void verfft_m_T(const Field* y, Field* out) {  // PFF -> PFP: VERFFT(+1) / NX
        verfft(y->data, out->data, +1);
        k_axpby(out->data, 1.0 / c->d.NX, out->data, 0.0, nullptr, 0.0, c->d.pfp(), s());
        out->space = MLEGS_PFP;
        c->ln_zero(out);
    }
    void horfft_p_T(const Field* y, Field* out) {  // PPP -> PFP
        k_horfft_warp(g(), c->fft, y->data, out->data, -1, s());
        const double n2 = 2.0 * c->d.NTH;
        pfp_mscale_kernel<<<nb(c->d.pfp(), 256), 256, 0, s()>>>(g(), out->data, n2, 2.0 * n2, 1);
        count_launch();
        out->space = MLEGS_PFP;
        c->ln_zero(out);
    }
    void horfft_m_T(const Field* y, Field* out, Field* work) {  // PFP -> PPP
        copy(work, y);
        const double n2 = 2.0 * c->d.NTH;
        pfp_mscale_kernel<<<nb(c->d.pfp(), 256), 256, 0, s()>>>(g(), work->data, 1.0 / n2, 0.5 / n2, 0);
        count_launch();
        k_horfft_warp(g(), c->fft, work->data, out->data, +1, s());
        out->space = MLEGS_PPP;
        c->ln_zero(out);
    }
    void tofp_T(const Field* y, Field* out, int pad) {  // PPP -> FFF
        Field *a = tmp(), *b = tmp();
        horfft_p_T(y, a);
        verfft_p_T(a, b);
        rtran_p_T(b, out, pad);
        rel({b, a});
    }
    void toff_T(const Field* y, Field* out, int pad) {  // FFF -> PPP
        Field *a = tmp(), *b = tmp();
        rtran_m_T(y, a, pad);
        verfft_m_T(a, b);
        horfft_m_T(b, out, a);
        rel({b, a});
    }

    // ------------------------------------------------------------- band operators
    void xxdx_T(const Field* y, Field* out, int pad) {
        k_band3(c->gT, y->data, out->data, 0, pad, s());
        ln_rows(y, out, 1.0 / n0()[0], 1.0 / n0()[1], 0.0, false);
        out->space = MLEGS_FFF;
    }
    void mulxm_T(const Field* y, Field* out, int pad) {
        k_band3(c->gT, y->data, out->data, 1, pad, s());
        c->ln_zero(out);
        out->space = MLEGS_FFF;
    }
    void delsqh_T(const Field* y, Field* out, int pad) {
        k_delsqh(g(), y->data, nullptr, out->data, pad, s());  // the diagonal; entry (0, 0, 0) = 0
        ln_rows(y, out, 1.0 / c->d.ELL2 / n0()[0], 0.0, 0.0, false);
        out->space = MLEGS_FFF;
    }
    void del2_T(const Field* y, Field* out, int pad) {
        k_del2(c->gT, y->data, out->data, pad, s());
        const double e2 = c->d.ELL2;
        ln_rows(y, out, 4.0 / 3 / n0()[0] / e2, -2.0 / n0()[1] / e2, 2.0 / 3 / n0()[2] / e2, false);
        out->space = MLEGS_FFF;
    }
    // out = op(x) on rows n < NRCHOPS(m) at pad (mk_kernel ops), LN 0
    void mk(int op, const Field* x, Field* out, int pad) {
        k_mk_combine(g(), op, x->data, nullptr, out->data, pad, s());
        c->ln_zero(out);
        out->space = MLEGS_FFF;
    }
    // GRAD (mod_legops.f90:1727-1786): RR = XXDX(A), RP = i m A, GZ = i k A
    void grad_T(const Field* rr, const Field* rp, const Field* gz, Field* out, int pad) {
        Field* t = tmp();
        xxdx_T(rr, out, pad);
        mk(7, rp, t, pad);
        add(out, t);
        mk(8, gz, t, pad);
        add(out, t);
        rel(t);
    }
    // PC2VEL (1789-1853): RUR = i m PSI + i k XXDX(CHI); RUP = -XXDX(PSI) - m k CHI;
    // UZ = -MULXM(MULXM(DELSQH(CHI)))
    void pc2vel_T(const Field* rur, const Field* rup, const Field* uz, Field* psi, Field* chi, int pad) {
        Field *t = tmp(), *u = tmp();
        mk(7, rur, psi, pad);
        xxdx_T(rup, t, pad);
        add(psi, t, -1.0);
        mk(8, rur, t, pad);
        xxdx_T(t, chi, pad);
        mk(10, rup, t, pad);
        add(chi, t);
        mk(6, uz, t, pad);
        mulxm_T(t, u, pad);
        mulxm_T(u, t, pad);
        delsqh_T(t, u, pad);
        add(chi, u);
        rel({u, t});
    }
    // PC2VOR (1856-1919): W = DEL2(CHI); ROR = -i m W + i k XXDX(PSI);
    // ROP = XXDX(W) - k m PSI; OZ = -MULXM(MULXM(DELSQH(PSI)))
    void pc2vor_T(const Field* ror, const Field* rop, const Field* oz, Field* psi, Field* chi, int pad) {
        Field *t = tmp(), *u = tmp(), *w = tmp();
        mk(4, ror, w, pad);
        xxdx_T(rop, t, pad);
        add(w, t);
        del2_T(w, chi, pad);
        mk(8, ror, t, pad);
        xxdx_T(t, psi, pad);
        mk(10, rop, t, pad);
        add(psi, t);
        mk(6, oz, t, pad);
        mulxm_T(t, u, pad);
        mulxm_T(u, t, pad);
        delsqh_T(t, u, pad);
        add(psi, u);
        rel({w, u, t});
    }

    // ------------------------------------------------------------- solves
    void farfield_T(Field* y, int nr) {
        farfield_T_kernel<<<nb(c->d.NXCHOPDIM, 32), 256, 0, s()>>>(g(), y->data, nr);
        count_launch();
    }
    const mlegs_ctx::SolveFactors* factors(int kind, double alp) {
        const auto* f = c->factors(kind, 0, alp);
        if (!f) throw ApiError(MLEGS_ERR_STATE, "adjoint: banded-solve factors unavailable");
        return f;
    }
    void solve_T(const mlegs_ctx::SolveFactors* f, Field* y, int kind) {
        if (c->d.NRCHOP <= 72) {  // the whole system fits in shared memory
            const int nsys = c->d.NTCHOPDIM * c->d.NXCHOPDIM, t_begin = kind == 2 ? c->d.NXCHOPDIM : 0;
            const int nb0 = (t_begin + 15) / 16, nb1 = (nsys - t_begin + 15) / 16;
            const size_t smem = (size_t)c->d.NRCHOP * 144 * sizeof(double);
            static size_t attr = 0;
            if (smem > attr && smem > 48 * 1024) {
                cudaFuncSetAttribute(solve_T_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                attr = smem;
            }
            solve_T_small_kernel<<<nb0 + nb1, 32, smem, s()>>>(g(), f->F5, f->F7, y->data, kind, 0, t_begin, nb0);
            count_launch();
            return;
        }
        const int nw = 2 * c->d.NXCHOPDIM, wpad = kind == 2 ? (32 - nw % 32) % 32 : 0;
        const int n = 2 * c->d.NTCHOPDIM * c->d.NXCHOPDIM + wpad;
        solve_T_kernel<<<nb(n, 128), 128, 0, s()>>>(g(), f->F5, f->F7, y->data, kind, 0, wpad);
        count_launch();
    }
    // IDEL2LN(B, A) (mod_legops.f90:1013-1176) as B -> (A, A%LN): A_bar -> B_bar (LN 0)
    void idel2ln_T(const Field* ab, Field* out) {
        const auto* f = factors(0, 0.0);
        copy(out, ab);
        farfield_T(out, c->d.NRCHOP);
        chop(out, 0);
        ln_to_coef(out, ab->ln, n0()[0], false);  // A(1,1,1) was replaced by A%LN / NORM(1,1)
        solve_T(f, out, 0);
        chop(out, 0);
        c->ln_zero(out);
        out->space = MLEGS_FFF;
    }
    // IHELM(B, A, ALP) (1204-1354) as (B, B%LN) -> (A, A%LN)
    void ihelm_T(const Field* ab, Field* out, double alp) {
        const auto* f = factors(2, alp);
        copy(out, ab);
        chop(out, 0);
        solve_T(f, out, 2);
        chop(out, 0);
        // A%LN = -B%LN/ALP, and the right-hand side's log-term rows are B + (B%LN/ALP) c
        const double e2 = c->d.ELL2;
        k_ln_copy(out->ln, ab->ln, -1.0 / alp, s());
        ln_rows(out, out, 4.0 / 3 / e2 / n0()[0] / alp, -2.0 / n0()[1] / e2 / alp, 2.0 / 3 / n0()[2] / e2 / alp,
                true);
        out->space = MLEGS_FFF;
    }
    // VISC2(A, AO, NU, DT) (mod_march.f90:1579-1636) -> (A_bar, AO_bar)
    void visc2_T(const Field* yb, Field* a_bar, Field* ao_bar, double nu, double dt) {
        const double alp = 2 / nu / dt;
        Field *wk = tmp(), *t = tmp();
        ihelm_T(yb, wk, alp);
        copy(a_bar, wk);
        scale(a_bar, -alp);
        copy(t, wk);
        scale(t, -1.0);
        c->ln_zero(t);
        chop(t, 0);
        del2_T(t, ao_bar, 2);
        rel({t, wk});
    }
    // VISC1(A, NU, DT) (1529-1576) = IHELM(-ALP A, ALP), ALP = 1/(NU DT)
    void visc1_T(const Field* yb, Field* a_bar, double nu, double dt) {
        const double alp = 1 / (nu * dt);
        ihelm_T(yb, a_bar, alp);
        scale(a_bar, -alp);
    }
    // IDELSQH(B, A) (136-241) at CHOPSET(pad): far-field transpose, the diagonal
    // -ELL2/(n(n+1)) for n >= 1 and B_bar(1,1,1) += A%LN_bar NORM(1,1) ELL2
    void idelsqh_T(const Field* ab, Field* out, int pad) {
        Field* y = tmp();
        copy(y, ab);
        farfield_T(y, c->d.NRCHOP + pad);
        k_idelsqh(g(), y->data, out->data, pad, s());
        ln_to_coef(out, ab->ln, n0()[0] * c->d.ELL2, true);
        c->ln_zero(out);
        out->space = MLEGS_FFF;
        rel(y);
    }

    // ------------------------------------------------------------- PROJECT
    // x_bar (PFF) (+)= fold^T(W_w, z): mode 0 an EO segment, 1 an OE segment
    void fold_T(int w, const Field* z, Field* out, int mode, bool first, Field* work) {
        DevGrid gw = g();
        gw.pf = c->adj_w[w];
        const size_t n = c->d.pff();
        if (mode == 0 && first) {
            k_rtran_b2p(gw, z->data, out->data, nullptr, 0, s());
            return;
        }
        k_rtran_b2p(gw, z->data, work->data, nullptr, 0, s());
        if (mode == 0) {
            k_axpby(out->data, 1.0, work->data, 0.0, nullptr, 1.0, n, s());
        } else {
            pff_mirror_kernel<<<nb(n, 256), 256, 0, s()>>>(g(), out->data, work->data, first ? 0 : 1);
            count_launch();
        }
    }
    // PROJECT(ROR, ROP, OZ, PSI, W, 0.0) of PPP inputs (CALC_BOUSSI_FORCE's and
    // CALC_BOUSSI_NONLIN's form, PSI%LN set to 0): (PSI_bar, W_bar) -> 3 PPP cotangents
    void project_ppp_ln0_T(const Field* psib, const Field* wb, Field* const out[3]) {
        Field *ps = tmp(), *ch = tmp(), *z = tmp(), *work = tmp();
        Field* x[3] = {tmp(), tmp(), tmp()};
        copy(ps, psib);
        farfield_T(ps, c->d.NRCHOP);
        chop(ps, 0);
        copy(ch, wb);
        chop(ch, 0);
        // PSI = -(i m) EO(V, rur) - OE(D, rup);  CHI = (i k) OE(D, rur) + m k EO(V, rup) - EO(T, uz)
        mk(8, ch, z, 0);
        fold_T(1, z, x[0], 1, true, work);
        mk(4, ps, z, 0);
        fold_T(0, z, x[0], 0, false, work);
        mk(6, ps, z, 0);
        fold_T(1, z, x[1], 1, true, work);
        mk(9, ch, z, 0);
        fold_T(0, z, x[1], 0, false, work);
        mk(6, ch, z, 0);
        fold_T(2, z, x[2], 0, true, work);
        for (Field* f : x) {
            f->space = MLEGS_PFF;
            c->ln_zero(f);
        }
        vel2pln_T_kernel<<<1, 256, 0, s()>>>(g(), x[1]->data, c->v2p_pff);
        count_launch();
        for (int q = 0; q < 3; ++q) {
            verfft_m_T(x[q], z);
            horfft_m_T(z, out[q], work);
        }
        rel({x[0], x[1], x[2], work, z, ch, ps});
    }

    // ------------------------------------------------------------- FORCE, the step, the start-up
    // CALC_BOUSSI_FORCE at (PSI, CHI, B): (PSIN_bar, CHIN_bar, BN_bar) -> (PSI_bar, CHI_bar, B_bar)
    void force_vjp(const Field* PSI, const Field* CHI, const Field* B, const Field* pnb, const Field* cnb,
                   const Field* bnb, Field* pb, Field* cb, Field* bb) {
        const int P3v = 3;  // CHOPSET(3)
        const size_t np = c->d.ppp();
        // the products' operands in PPP (TOFP of PC2VEL, PC2VOR and GRAD(B) at CHOPSET(3))
        Field* U[3] = {tmp(), tmp(), tmp()};
        Field* Wv[3] = {tmp(), tmp(), tmp()};
        Field* Gp[3] = {tmp(), tmp(), tmp()};
        c->pc2vel(PSI, CHI, U[0], U[1], U[2], P3v);
        c->pc2vor(PSI, CHI, Wv[0], Wv[1], Wv[2], P3v);
        c->grad(B, Gp[0], Gp[1], Gp[2], P3v);
        for (int q = 0; q < 3; ++q) {
            c->tofp(U[q], P3v);
            c->tofp(Wv[q], P3v);
            c->tofp(Gp[q], P3v);
        }
        // cotangents of (ROR, ROP, OZ) and BN in PPP
        Field *wbar = tmp(), *bnp = tmp();
        Field* nbf[3] = {tmp(), tmp(), tmp()};
        idel2ln_T(cnb, wbar);
        project_ppp_ln0_T(pnb, wbar, nbf);
        toff_T(bnb, bnp, 0);
        rel(wbar);
        // ROR = N_r + 2 OMEGA RUP, ROP = N_t - 2 OMEGA RUR, OZ = N_z - W, BN = -VDOTP(U, G) + N^2 UZ
        Field* ub[3] = {tmp(), tmp(), tmp()};
        Field* wb[3] = {tmp(), tmp(), tmp()};
        Field* gb[3] = {tmp(), tmp(), tmp()};
        Field* nbn = tmp();
        k_axpby(nbn->data, -1.0, bnp->data, 0.0, nullptr, 0.0, np, s());
        P3 Up{{U[0]->data, U[1]->data, U[2]->data}}, Wp{{Wv[0]->data, Wv[1]->data, Wv[2]->data}},
            Bp{{nbf[0]->data, nbf[1]->data, nbf[2]->data}}, Gpp{{Gp[0]->data, Gp[1]->data, Gp[2]->data}};
        Q3 Uo{{ub[0]->data, ub[1]->data, ub[2]->data}}, Wo{{wb[0]->data, wb[1]->data, wb[2]->data}},
            Go{{gb[0]->data, gb[1]->data, gb[2]->data}};
        vprod_T_kernel<<<nb(np, 256), 256, 0, s()>>>(g(), Up, Wp, Bp, Uo, Wo);
        count_launch();
        vdotp_T_kernel<<<nb(np, 256), 256, 0, s()>>>(g(), Up, Gpp, nbn->data, Uo, Go);
        count_launch();
        const double o2 = 2 * c->p.omega, n2 = c->p.bv0 * c->p.bv0;
        k_axpby(ub[0]->data, -o2, nbf[1]->data, 0.0, nullptr, 1.0, np, s());
        k_axpby(ub[1]->data, o2, nbf[0]->data, 0.0, nullptr, 1.0, np, s());
        k_axpby(ub[2]->data, n2, bnp->data, 0.0, nullptr, 1.0, np, s());
        for (int q = 0; q < 3; ++q) ub[q]->space = wb[q]->space = gb[q]->space = MLEGS_PPP;
        rel({nbn, bnp});
        for (int q = 0; q < 3; ++q) rel({U[q], Wv[q], Gp[q]});
        // back to FFF at CHOPSET(3): fu = TOFP^T(ub), then ub, wb reused for TOFP^T(wb), TOFP^T(gb)
        Field* fu[3] = {tmp(), tmp(), tmp()};
        for (int q = 0; q < 3; ++q) {
            tofp_T(ub[q], fu[q], P3v);
            tofp_T(wb[q], ub[q], P3v);
            tofp_T(gb[q], wb[q], P3v);
        }
        Field *p2 = tmp(), *c2 = tmp();
        pc2vel_T(fu[0], fu[1], fu[2], pb, cb, P3v);
        pc2vor_T(ub[0], ub[1], ub[2], p2, c2, P3v);
        grad_T(wb[0], wb[1], wb[2], bb, P3v);
        add(pb, p2);
        add(cb, c2);
        // B enters OZ through W = TOFP(B) at CHOPSET(0)
        k_axpby(gb[0]->data, -1.0, nbf[2]->data, 0.0, nullptr, 0.0, np, s());
        gb[0]->space = MLEGS_PPP;
        c->ln_zero(gb[0]);
        tofp_T(gb[0], p2, 0);
        chop(p2, 0);
        add(bb, p2);
        rel({p2, c2});
        for (int q = 0; q < 3; ++q) rel({nbf[q], ub[q], wb[q], gb[q], fu[q]});
        for (Field* f : {pb, cb, bb}) f->space = MLEGS_FFF;
    }

    // One steady STEP_BOUSSI_AB_CN (VISC%SW = 1) as the map of (psi, chi, b,
    // n_psi, n_chi, n_b) at st (psi, chi, b): cotangents bar[6] -> out[6]
    void ab2_step_vjp(Field* const st[3], Field* const bar[6], Field* const out[6]) {
        const double dt = c->p.dt;
        const double nu[3] = {c->p.nu, c->p.nu, c->p.kappa};
        Field* abar[3] = {tmp(), tmp(), tmp()};
        Field* aobar[3] = {tmp(), tmp(), tmp()};
        Field* yb = tmp();
        for (int q = 0; q < 3; ++q) {
            copy(yb, bar[q]);
            if (q == 2) c->ln_zero(yb);
            if (nu[q] != 0.0) {
                visc2_T(yb, abar[q], aobar[q], nu[q], dt);
            } else {
                copy(abar[q], yb);
                zero(aobar[q]);
            }
            if (q == 2) {
                c->ln_zero(abar[q]);
                c->ln_zero(aobar[q]);
            }
        }
        rel(yb);
        Field* fbar[3] = {tmp(), tmp(), tmp()};
        for (int q = 0; q < 3; ++q) {
            copy(fbar[q], bar[3 + q]);
            if (q == 2) c->ln_zero(fbar[q]);
            chop(fbar[q], 0);
            add(fbar[q], abar[q], 1.5 * dt);
            copy(out[3 + q], abar[q]);
            scale(out[3 + q], -0.5 * dt);
        }
        Field* fo[3] = {tmp(), tmp(), tmp()};
        force_vjp(st[0], st[1], st[2], fbar[0], fbar[1], fbar[2], fo[0], fo[1], fo[2]);
        for (int q = 0; q < 3; ++q) {
            copy(out[q], abar[q]);
            chop(aobar[q], 0);
            add(out[q], aobar[q]);
            add(out[q], fo[q]);
        }
        c->ln_zero(out[2]);
        c->ln_zero(out[5]);
        for (int q = 0; q < 3; ++q) rel({abar[q], aobar[q], fbar[q], fo[q]});
        for (int q = 0; q < 6; ++q) out[q]->space = MLEGS_FFF;
    }

    // BE viscous steps of CALC_BOUSSI_VISC_BE transposed, per field
    void visc_be_T(Field* const in[3], Field* const o[3], double h) {
        const double nu[3] = {c->p.nu, c->p.nu, c->p.kappa};
        for (int q = 0; q < 3; ++q) {
            if (nu[q] != 0.0) visc1_T(in[q], o[q], nu[q], h);
            else copy(o[q], in[q]);
        }
        c->ln_zero(o[2]);
    }

    // RICH_BOUSSI_FE_BE (mod_march.f90:535-606) as the map (psi, chi, b) ->
    // (psi, chi, b, n_psi, n_chi, n_b) at st: bar[6] -> out[3].  Forward:
    // F0 = FORCE(x0); x2 = BE(x0 + dt/2 F0, dt/2); x2' = BE(x2 + dt/2 FORCE(x2),
    // dt/2); x3 = BE(x0 + dt F0, dt); out = 2 x2' - x3, history F0.
    void startup_vjp(Field* const st[3], Field* const bar[6], Field* const out[3]) {
        const double dt = c->p.dt, hdt = 0.5 * dt;
        const size_t N = c->fff();
        Field* x2[3] = {tmp(), tmp(), tmp()};
        {
            Field* F0[3] = {tmp(), tmp(), tmp()};
            reserve(16);
            c->force(st[0], st[1], st[2], F0[0], F0[1], F0[2]);
            for (int q = 0; q < 3; ++q) {
                k_axpby_ln(x2[q]->data, 1.0, st[q]->data, hdt, F0[q]->data, 0.0, N,
                           x2[q]->ln, 1.0, st[q]->ln, hdt, F0[q]->ln, 0.0, s());
                x2[q]->space = MLEGS_FFF;
            }
            c->ln_zero(x2[2]);
            rel({F0[0], F0[1], F0[2]});
            reserve(4);
            c->visc_be(x2[0], x2[1], x2[2], hdt);
        }
        Field* y1[3] = {tmp(), tmp(), tmp()};
        Field* x2p[3] = {tmp(), tmp(), tmp()};
        {
            Field* w[3] = {tmp(), tmp(), tmp()};
            for (int q = 0; q < 3; ++q) {
                copy(w[q], bar[q]);
                if (q == 2) c->ln_zero(w[q]);
                scale(w[q], -1.0);
            }
            visc_be_T(w, y1, dt);
            for (int q = 0; q < 3; ++q) scale(w[q], -2.0);
            visc_be_T(w, x2p, hdt);
            for (int q = 0; q < 3; ++q) {
                copy(w[q], x2p[q]);
                scale(w[q], hdt);
            }
            Field* fx2[3] = {tmp(), tmp(), tmp()};
            force_vjp(x2[0], x2[1], x2[2], w[0], w[1], w[2], fx2[0], fx2[1], fx2[2]);
            for (int q = 0; q < 3; ++q) add(x2p[q], fx2[q]);
            rel({fx2[0], fx2[1], fx2[2], w[0], w[1], w[2]});
        }
        Field* z[3] = {x2[0], x2[1], x2[2]};  // x2 is no longer needed
        visc_be_T(x2p, z, hdt);
        Field* f0[3] = {x2p[0], x2p[1], x2p[2]};
        for (int q = 0; q < 3; ++q) {
            copy(f0[q], bar[3 + q]);
            if (q == 2) c->ln_zero(f0[q]);
            add(f0[q], y1[q], dt);
            add(f0[q], z[q], hdt);
        }
        Field* fx0[3] = {tmp(), tmp(), tmp()};
        force_vjp(st[0], st[1], st[2], f0[0], f0[1], f0[2], fx0[0], fx0[1], fx0[2]);
        for (int q = 0; q < 3; ++q) {
            copy(out[q], y1[q]);
            add(out[q], z[q]);
            add(out[q], fx0[q]);
            out[q]->space = MLEGS_FFF;
        }
        c->ln_zero(out[2]);
        for (int q = 0; q < 3; ++q) rel({x2[q], y1[q], x2p[q], fx0[q]});
    }

    // The seeded initial state psi = vortex + IDELSQH(-c_psi), chi likewise,
    // b = c_b with the far-field fix (each chopped): (psi, chi, b)_bar -> c_bar
    void initial_state_T(Field* const xb[3], Field* const cb[3]) {
        Field* q = tmp();
        for (int i = 0; i < 2; ++i) {
            copy(q, xb[i]);
            chop(q, 0);
            idelsqh_T(q, cb[i], 0);
            chop(cb[i], 0);
            scale(cb[i], -1.0);
            c->ln_zero(cb[i]);
        }
        copy(cb[2], xb[2]);
        chop(cb[2], 0);
        farfield_T(cb[2], c->d.NRCHOP);
        chop(cb[2], 0);
        c->ln_zero(cb[2]);
        cb[2]->space = MLEGS_FFF;
        rel(q);
    }

    // J = KE(psi - psi_bar, chi - chi_bar) + 1/2 int b^2 dV, psi_bar and
    // chi_bar the (m, k) = (0, 0) parts, in the quadrature forms of
    // CALC_BOUSSI_ENERGY (mod_boussinesq.f90:176-206: RTRAN(+1) of DELSQH /
    // DEL2 at CHOPSET(3)) and CALC_BOUSSI_PE (112-136), with the gradient.  J is
    // a homogeneous quadratic form, so J = (1/2) <x, grad J>.
    double objective(const Field* psi, const Field* chi, const Field* b, Field* gp, Field* gc, Field* gb) {
        const int P3v = 3;
        const double sc = 4.0 * 3.141592653589793238462643383279502884 * c->d.ZLEN * c->d.ELL2;
        Field *p = tmp(), *ch = tmp(), *bb = tmp(), *t = tmp(), *u = tmp(), *v = tmp();
        auto fluct = [&](const Field* src, Field* dst) {
            copy(dst, src);
            zero_col00_kernel<<<nb(c->d.NRCHOPDIM, 128), 128, 0, s()>>>(g(), dst->data);
            count_launch();
            c->ln_zero(dst);
        };
        fluct(psi, p);
        fluct(chi, ch);
        copy(bb, b);
        c->ln_zero(bb);
        auto WR = [&](const Field* src, Field* dst, double f, int inv) {  // f W RTRAN(+1)(src)
            k_rtran_b2p(g(), src->data, t->data, nullptr, P3v, s());
            pff_quadw_kernel<<<nb(c->d.pff(), 256), 256, 0, s()>>>(g(), t->data, dst->data, f * sc, inv);
            count_launch();
            dst->space = MLEGS_PFF;
        };
        // KE = 1/2 [ -<R p, R DELSQH p>_W + <R DEL2 c, R DELSQH c>_W ]
        c->delsqh(p, v, P3v);
        WR(v, u, -0.5, 0);
        rtran_p_T(u, gp, P3v);
        WR(p, u, -0.5, 0);
        rtran_p_T(u, v, P3v);
        delsqh_T(v, u, P3v);
        add(gp, u);
        c->delsqh(ch, v, P3v);
        WR(v, u, 0.5, 0);
        rtran_p_T(u, v, P3v);
        del2_T(v, gc, P3v);
        c->del2(ch, v, P3v);
        WR(v, u, 0.5, 0);
        rtran_p_T(u, v, P3v);
        delsqh_T(v, u, P3v);
        add(gc, u);
        // 1/2 int b^2 = 1/2 <R b, R b>_{W/(1-x)^2}
        WR(bb, u, 1.0, 1);
        rtran_p_T(u, gb, P3v);
        for (Field* f : {gp, gc}) {
            zero_col00_kernel<<<nb(c->d.NRCHOPDIM, 128), 128, 0, s()>>>(g(), f->data);
            count_launch();
        }
        for (Field* f : {gp, gc, gb}) {
            c->ln_zero(f);
            f->space = MLEGS_FFF;
        }
        CK(cudaMemsetAsync(c->adj_dot, 0, sizeof(double), s()));
        const Field* xs[3] = {psi, chi, b};
        const Field* gs[3] = {gp, gc, gb};
        for (int q = 0; q < 3; ++q) {
            fff_dot_kernel<<<148, 256, 0, s()>>>(g(), xs[q]->data, gs[q]->data, c->adj_dot);
            count_launch();
        }
        double J = 0.0;
        CK(cudaMemcpyAsync(&J, c->adj_dot, sizeof(double), cudaMemcpyDeviceToHost, s()));
        CK(cudaStreamSynchronize(s()));
        rel({p, ch, bb, t, u, v});
        return 0.5 * J;
    }
};

void require_fff(std::initializer_list<const Field*> fs, const char* who) {
    for (const Field* f : fs)
        if (f->space != MLEGS_FFF) throw ApiError(MLEGS_ERR_TRANSFORM, std::string(who) + ": fields must be in FFF");
}

void require_ab2_sw1(const mlegs_ctx* ctx) {
    if (!ctx->p.adams || ctx->p.visc_sw != 1)
        throw ApiError(MLEGS_ERR_ARG, "adjoint: AB2-CN contexts with VISC%SW = 1 only");
}

// Runs fn with the solver's state pointed at the context's scratch state
// (adj_state[0..2]); the AB history hist[0..2] is saved in adj_state[3..5] and
// put back, and so are the solver's time and step count.
template <class Fn>
void on_scratch_state(mlegs_ctx* ctx, Fn&& fn) {
    if (!ctx->adj_state[0]) {
        ctx->no_capture("step map");
        for (Field*& f : ctx->adj_state) f = ctx->new_field(MLEGS_FFF, true);
    }
    Field *P = ctx->psi, *C = ctx->chi, *B = ctx->b;
    Field* H[3] = {ctx->hist[0], ctx->hist[1], ctx->hist[2]};
    const double t0 = ctx->t;
    const int n0 = ctx->n;
    for (int q = 0; q < 3; ++q) ctx->copy0(ctx->adj_state[3 + q], H[q], 0);
    ctx->psi = ctx->adj_state[0];
    ctx->chi = ctx->adj_state[1];
    ctx->b = ctx->adj_state[2];
    auto put_back = [&] {
        ctx->psi = P;
        ctx->chi = C;
        ctx->b = B;
        ctx->t = t0;
        ctx->n = n0;
        for (int q = 0; q < 3; ++q) ctx->copy0(H[q], ctx->adj_state[3 + q], 0);
    };
    try {
        fn();
    } catch (...) {
        put_back();
        throw;
    }
    put_back();
}

// Runs fn through the context's graph cache G for the field set `key`: the
// first call with a key runs eagerly (tables, factors and temporaries are set up
// there), the second is captured into a CUDA graph and launched, later calls
// with the same key replay it.  fn must issue the same work for the same key.
template <class Fn>
void run_cached(mlegs_ctx* ctx, mlegs_ctx::AdjGraph& G, const std::vector<const void*>& key, Fn&& fn) {
    if (G.exec && G.key == key) {
        CK(cudaGraphLaunch(G.exec, ctx->s));
        ctx->launches += G.launches;
        return;
    }
    if (!G.warm || G.key != key) {
        if (G.exec) {
            cudaGraphExecDestroy(G.exec);
            G.exec = nullptr;
        }
        G.key = key;
        G.warm = true;
        ctx->mark();
        fn();
        ctx->restore();
        return;
    }
    ctx->mark();
    const int64_t before = ctx->launches;
    CK(cudaStreamBeginCapture(ctx->s, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
        fn();
    } catch (...) {
        cudaStreamEndCapture(ctx->s, &graph);
        if (graph) cudaGraphDestroy(graph);
        ctx->restore();
        G.warm = false;
        throw;
    }
    CK(cudaStreamEndCapture(ctx->s, &graph));
    G.launches = ctx->launches - before;
    ctx->launches = before;
    ctx->restore();
    const cudaError_t e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        G.exec = nullptr;
        throw CudaError(std::string("adjoint graph: ") + cudaGetErrorString(e));
    }
    CK(cudaGraphLaunch(G.exec, ctx->s));
    ctx->launches += G.launches;
}

std::vector<const void*> field_key(std::initializer_list<const Field*> fs) {
    std::vector<const void*> k;
    for (const Field* f : fs) {
        k.push_back(f);
        k.push_back(f->data);
    }
    return k;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int mlegs_transpose(mlegs_ctx* ctx, int op, const mlegs_field* const* y, mlegs_field* const* x, int pad, double p1) {
    return guard(ctx, [&] {
        if (!y || !x) throw ApiError(MLEGS_ERR_ARG, "mlegs_transpose: null field array");
        check_pad(ctx, pad);
        Adj A(ctx);
        A.prepare();
        ctx->mark();
        auto Y = [&](int i) { return F(y[i]); };
        auto X = [&](int i) { return F(x[i]); };
        switch (op) {
            case MLEGS_T_RTRAN_P: A.rtran_p_T(Y(0), X(0), pad); break;
            case MLEGS_T_RTRAN_M: A.rtran_m_T(Y(0), X(0), pad); break;
            case MLEGS_T_VERFFT_P: A.verfft_p_T(Y(0), X(0)); break;
            case MLEGS_T_VERFFT_M: A.verfft_m_T(Y(0), X(0)); break;
            case MLEGS_T_HORFFT_P: A.horfft_p_T(Y(0), X(0)); break;
            case MLEGS_T_HORFFT_M: {
                Field* w = A.tmp();
                A.horfft_m_T(Y(0), X(0), w);
                A.rel(w);
            } break;
            case MLEGS_T_TOFP: A.tofp_T(Y(0), X(0), pad); break;
            case MLEGS_T_TOFF: A.toff_T(Y(0), X(0), pad); break;
            case MLEGS_T_XXDX: A.xxdx_T(Y(0), X(0), pad); break;
            case MLEGS_T_MULXM: A.mulxm_T(Y(0), X(0), pad); break;
            case MLEGS_T_DELSQH: A.delsqh_T(Y(0), X(0), pad); break;
            case MLEGS_T_DEL2: A.del2_T(Y(0), X(0), pad); break;
            case MLEGS_T_GRAD: A.grad_T(Y(0), Y(1), Y(2), X(0), pad); break;
            case MLEGS_T_PC2VEL: A.pc2vel_T(Y(0), Y(1), Y(2), X(0), X(1), pad); break;
            case MLEGS_T_PC2VOR: A.pc2vor_T(Y(0), Y(1), Y(2), X(0), X(1), pad); break;
            case MLEGS_T_IDEL2LN: A.idel2ln_T(Y(0), X(0)); break;
            case MLEGS_T_IHELM:
                if (p1 == 0.0) throw ApiError(MLEGS_ERR_LEGOPERATOR, "IHELM: ALP CAN'T BE ZERO");
                A.ihelm_T(Y(0), X(0), p1);
                break;
            case MLEGS_T_PROJECT_PPP: {
                Field* o[3] = {X(0), X(1), X(2)};
                A.project_ppp_ln0_T(Y(0), Y(1), o);
            } break;
            case MLEGS_T_VISC2:
                if (p1 == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "VISC2: NU CAN'T BE ZERO");
                A.visc2_T(Y(0), X(0), X(1), p1, ctx->p.dt);
                break;
            case MLEGS_T_IDELSQH: A.idelsqh_T(Y(0), X(0), pad); break;
            case MLEGS_T_FARFIELD:
                A.copy(X(0), Y(0));
                A.farfield_T(X(0), ctx->d.NRCHOP + pad);
                break;
            default: throw ApiError(MLEGS_ERR_ARG, "mlegs_transpose: unknown op");
        }
        ctx->restore();
    });
}

int mlegs_boussi_force_vjp(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                           const mlegs_field* psin_bar, const mlegs_field* chin_bar, const mlegs_field* bn_bar,
                           mlegs_field* psi_bar, mlegs_field* chi_bar, mlegs_field* b_bar) {
    return guard(ctx, [&] {
        require_fff({F(psi), F(chi), F(b), F(psin_bar), F(chin_bar), F(bn_bar)}, "CALC_BOUSSI_FORCE VJP");
        Adj A(ctx);
        A.prepare();
        ctx->mark();
        A.force_vjp(F(psi), F(chi), F(b), F(psin_bar), F(chin_bar), F(bn_bar), F(psi_bar), F(chi_bar), F(b_bar));
        ctx->restore();
    });
}

int mlegs_ab2_step_map(mlegs_ctx* ctx, const mlegs_field* const* in, mlegs_field* const* out) {
    return guard(ctx, [&] {
        if (!in || !out) throw ApiError(MLEGS_ERR_ARG, "mlegs_ab2_step_map: null field array");
        require_ab2_sw1(ctx);
        for (int q = 0; q < 6; ++q) require_fff({F(in[q])}, "mlegs_ab2_step_map");
        const std::vector<const void*> key = field_key({F(in[0]), F(in[1]), F(in[2]), F(in[3]), F(in[4]), F(in[5]),
                                                         F(out[0]), F(out[1]), F(out[2]), F(out[3]), F(out[4]),
                                                         F(out[5])});
        on_scratch_state(ctx, [&] {
            run_cached(ctx, ctx->adj_g[0], key, [&] {
                for (int q = 0; q < 3; ++q) ctx->copy0(ctx->adj_state[q], F(in[q]), 0);
                for (int q = 0; q < 3; ++q) ctx->copy0(ctx->hist[q], F(in[3 + q]), 0);
                ctx->step_ab_cn();
                for (int q = 0; q < 3; ++q) ctx->copy0(F(out[q]), ctx->adj_state[q], 0);
                for (int q = 0; q < 3; ++q) ctx->copy0(F(out[3 + q]), ctx->hist[q], 0);
            });
            for (int q = 0; q < 6; ++q) F(out[q])->space = MLEGS_FFF;
        });
    });
}

int mlegs_ab2_startup_map(mlegs_ctx* ctx, const mlegs_field* const* in, mlegs_field* const* out) {
    return guard(ctx, [&] {
        if (!in || !out) throw ApiError(MLEGS_ERR_ARG, "mlegs_ab2_startup_map: null field array");
        require_ab2_sw1(ctx);
        for (int q = 0; q < 3; ++q) require_fff({F(in[q])}, "mlegs_ab2_startup_map");
        on_scratch_state(ctx, [&] {
            for (int q = 0; q < 3; ++q) ctx->copy0(ctx->adj_state[q], F(in[q]), 0);
            ctx->mark();
            ctx->rich_fe_be();
            ctx->restore();
            for (int q = 0; q < 3; ++q) ctx->copy0(F(out[q]), ctx->adj_state[q], 0);
            for (int q = 0; q < 3; ++q) ctx->copy0(F(out[3 + q]), ctx->hist[q], 0);
        });
    });
}

int mlegs_ab2_step_vjp(mlegs_ctx* ctx, const mlegs_field* const* state, const mlegs_field* const* bar,
                       mlegs_field* const* out) {
    return guard(ctx, [&] {
        if (!state || !bar || !out) throw ApiError(MLEGS_ERR_ARG, "mlegs_ab2_step_vjp: null field array");
        require_ab2_sw1(ctx);
        Field* st[3];
        Field* b6[6];
        Field* o6[6];
        for (int q = 0; q < 3; ++q) st[q] = const_cast<Field*>(F(state[q]));
        for (int q = 0; q < 6; ++q) {
            b6[q] = const_cast<Field*>(F(bar[q]));
            o6[q] = F(out[q]);
        }
        require_fff({st[0], st[1], st[2], b6[0], b6[1], b6[2], b6[3], b6[4], b6[5]}, "mlegs_ab2_step_vjp");
        Adj A(ctx);
        A.prepare();
        const std::vector<const void*> key = field_key({st[0], st[1], st[2], b6[0], b6[1], b6[2], b6[3], b6[4],
                                                         b6[5], o6[0], o6[1], o6[2], o6[3], o6[4], o6[5]});
        run_cached(ctx, ctx->adj_g[1], key, [&] { A.ab2_step_vjp(st, b6, o6); });
        for (int q = 0; q < 6; ++q) o6[q]->space = MLEGS_FFF;
    });
}

int mlegs_ab2_startup_vjp(mlegs_ctx* ctx, const mlegs_field* const* state, const mlegs_field* const* bar,
                          mlegs_field* const* out) {
    return guard(ctx, [&] {
        if (!state || !bar || !out) throw ApiError(MLEGS_ERR_ARG, "mlegs_ab2_startup_vjp: null field array");
        require_ab2_sw1(ctx);
        Field* st[3];
        Field* b6[6];
        Field* o3[3];
        for (int q = 0; q < 3; ++q) {
            st[q] = const_cast<Field*>(F(state[q]));
            o3[q] = F(out[q]);
        }
        for (int q = 0; q < 6; ++q) b6[q] = const_cast<Field*>(F(bar[q]));
        require_fff({st[0], st[1], st[2], b6[0], b6[1], b6[2], b6[3], b6[4], b6[5]}, "mlegs_ab2_startup_vjp");
        Adj A(ctx);
        A.prepare();
        ctx->mark();
        A.startup_vjp(st, b6, o3);
        ctx->restore();
    });
}

int mlegs_initial_state_T(mlegs_ctx* ctx, const mlegs_field* const* state_bar, mlegs_field* const* coef_bar) {
    return guard(ctx, [&] {
        if (!state_bar || !coef_bar) throw ApiError(MLEGS_ERR_ARG, "mlegs_initial_state_T: null field array");
        Field* xb[3];
        Field* cb[3];
        for (int q = 0; q < 3; ++q) {
            xb[q] = const_cast<Field*>(F(state_bar[q]));
            cb[q] = F(coef_bar[q]);
        }
        require_fff({xb[0], xb[1], xb[2]}, "mlegs_initial_state_T");
        Adj A(ctx);
        A.prepare();
        ctx->mark();
        A.initial_state_T(xb, cb);
        ctx->restore();
    });
}

int mlegs_energy_objective(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                           double* J, mlegs_field* gpsi, mlegs_field* gchi, mlegs_field* gb) {
    return guard(ctx, [&] {
        if (!J) throw ApiError(MLEGS_ERR_ARG, "mlegs_energy_objective: null J");
        require_fff({F(psi), F(chi), F(b)}, "mlegs_energy_objective");
        Adj A(ctx);
        A.prepare();
        ctx->mark();
        *J = A.objective(F(psi), F(chi), F(b), F(gpsi), F(gchi), F(gb));
        ctx->restore();
    });
}

int mlegs_field_device_copy(mlegs_ctx* ctx, mlegs_field* f, int to_field, int space, void* dev, double* ln_dev) {
    return guard(ctx, [&] {
        if (!dev) throw ApiError(MLEGS_ERR_ARG, "mlegs_field_device_copy: null device buffer");
        Field* fd = F(f);
        if (to_field) {
            if (space < 0 || space > 3) throw ApiError(MLEGS_ERR_TRANSFORM, "mlegs_field_device_copy: bad space");
            CK(cudaMemcpyAsync(fd->data, dev, ctx->d.elems(space) * sizeof(double2), cudaMemcpyDeviceToDevice,
                               ctx->s));
            fd->space = space;
            if (ln_dev) CK(cudaMemcpyAsync(fd->ln, ln_dev, sizeof(double), cudaMemcpyDeviceToDevice, ctx->s));
            else ctx->ln_zero(fd);
        } else {
            CK(cudaMemcpyAsync(dev, fd->data, ctx->d.elems(fd->space) * sizeof(double2), cudaMemcpyDeviceToDevice,
                               ctx->s));
            if (ln_dev) CK(cudaMemcpyAsync(ln_dev, fd->ln, sizeof(double), cudaMemcpyDeviceToDevice, ctx->s));
        }
    });
}

}  // extern "C"
