// Mapped-Legendre transforms as per-m parity GEMMs in FP64.
//
//  k_rtran_b2p  RTRAN(A, +1), mod_fft.f90:1264-1336:
//      BE(i,c) = sum_j PF(i, 2j)   A(2j,   c)   j < ceil(NN/2)
//      BO(i,c) = sum_j PF(i, 2j+1) A(2j+1, c)   j < floor(NN/2)
//      B(i) = BE + BO, B(NR-1-i) = BE - BO; (m,k) = (0,0) adds LN*(-log(1-x)).
//  k_fold_gemm  RTRAN(A, -1) (1189-1261) and the EOMUL/OEMUL products of
//      PROJECT (mod_legops.f90:2497-2535, 2548-2648):
//      out(n,c) (+)= s(m,k) sum_i Wt(n,i) F_par(n)(i,c),
//      F_e = in(i) + in(NR-1-i), F_o = in(i) - in(NR-1-i) (optionally x w_i).
// Complex fields are read as real matrices with 2*NXCHOPDIM interleaved
// columns, which is the reference's complex x real .MUL. as two real DGEMMs
// (mod_eig.f90:583-655) done in one pass.
#include "mlegs_internal.h"

namespace mlegs {

namespace {
constexpr int TM = 32, TN = 64, TK = 8;
}

__global__ void __launch_bounds__(128) rtran_b2p_kernel(DevGrid g, const double* __restrict__ A,
                                                        double* __restrict__ out, const double* ln,
                                                        int pad) {
    __shared__ double Ae[TK][TM], Ao[TK][TM];
    __shared__ double Be[TK][TN], Bo[TK][TN];
    const int m = blockIdx.z;
    const int ncol = 2 * g.NXCHOPDIM;
    const int i0 = blockIdx.y * TM, c0 = blockIdx.x * TN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    const int ke = (nn + 1) / 2, ko = nn / 2;
    const int ne = g.NRCHOPDIM + 1;
    const double* pf = g.pf + (size_t)m * ne * g.NRH;
    const double* a = A + (size_t)m * g.NRCHOPDIM * ncol;
    double ce[4][4] = {}, co[4][4] = {};
    for (int j0 = 0; j0 < ke; j0 += TK) {
        for (int t = threadIdx.x; t < TK * TM; t += 128) {
            int jj = t / TM, ii = t % TM;
            int j = j0 + jj, i = i0 + ii;
            double ve = 0.0, vo = 0.0;
            if (i < g.NRH) {
                if (j < ke) ve = pf[(size_t)(2 * j) * g.NRH + i];
                if (j < ko) vo = pf[(size_t)(2 * j + 1) * g.NRH + i];
            }
            Ae[jj][ii] = ve;
            Ao[jj][ii] = vo;
        }
        for (int t = threadIdx.x; t < TK * TN; t += 128) {
            int jj = t / TN, cc = t % TN;
            int j = j0 + jj, c = c0 + cc;
            double ve = 0.0, vo = 0.0;
            if (c < ncol) {
                if (j < ke) ve = a[(size_t)(2 * j) * ncol + c];
                if (j < ko) vo = a[(size_t)(2 * j + 1) * ncol + c];
            }
            Be[jj][cc] = ve;
            Bo[jj][cc] = vo;
        }
        __syncthreads();
#pragma unroll
        for (int jj = 0; jj < TK; ++jj) {
            double ae[4], ao[4], be[4], bo[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ae[q] = Ae[jj][ty * 4 + q];
                ao[q] = Ao[jj][ty * 4 + q];
                be[q] = Be[jj][tx * 4 + q];
                bo[q] = Bo[jj][tx * 4 + q];
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ce[p][q] = fma(ae[p], be[q], ce[p][q]);
                    co[p][q] = fma(ao[p], bo[q], co[p][q]);
                }
        }
        __syncthreads();
    }
    const double lnv = (m == 0 && ln) ? *ln : 0.0;
    double* o = out + (size_t)m * g.NR * ncol;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        int i = i0 + ty * 4 + p;
        if (i >= g.NRH) continue;
        int ih = g.NR - 1 - i;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int c = c0 + tx * 4 + q;
            if (c >= ncol) continue;
            double lo = ce[p][q] + co[p][q], hi = ce[p][q] - co[p][q];
            if (c == 0 && lnv != 0.0) {
                lo += lnv * g.lnx[i];
                hi += lnv * g.lnx[ih];
            }
            o[(size_t)i * ncol + c] = lo;
            o[(size_t)ih * ncol + c] = hi;
        }
    }
}

void k_rtran_b2p(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    if (b2p_bulk_supported(g)) {
        k_rtran_b2p_bulk(g, a, b, ln, pad, s);
        return;
    }
    if (dmma_supported(g)) {
        k_rtran_b2p_dmma(g, a, b, ln, pad, s);
        return;
    }
    int ncol = 2 * g.NXCHOPDIM;
    dim3 grid((ncol + TN - 1) / TN, (g.NRH + TM - 1) / TM, g.NTCHOPDIM);
    rtran_b2p_kernel<<<grid, 128, 0, s>>>(g, (const double*)a, (double*)b, ln, pad);
    count_launch();
}

namespace {
constexpr int FM = 32, FN = 64, FK = 16;
}

__global__ void __launch_bounds__(128) fold_gemm_kernel(DevGrid g, const double* __restrict__ Wt, int wt_rows,
                                                        const double* __restrict__ in, double* __restrict__ out,
                                                        int mode, int scale, int accumulate, int pad,
                                                        int use_w) {
    __shared__ double As[FK][FM];
    __shared__ double Fe[FK][FN], Fo[FK][FN];
    const int m = blockIdx.z;
    const int ncol = 2 * g.NXCHOPDIM;
    const int n0 = blockIdx.y * FM, c0 = blockIdx.x * FN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    double* o = out + (size_t)m * g.NRCHOPDIM * ncol;
    if (n0 >= nn) {
        if (!accumulate) {
            for (int t = threadIdx.x; t < FM * FN; t += 128) {
                int r = n0 + t / FN, c = c0 + t % FN;
                if (r < g.NRCHOPDIM && c < ncol) o[(size_t)r * ncol + c] = 0.0;
            }
        }
        return;
    }
    const double* w = Wt + (size_t)m * wt_rows * g.NRH;
    const double* x = in + (size_t)m * g.NR * ncol;
    double acc[4][4] = {};
    // rows of this thread: n0 + ty + 8q, all with the parity of (n0 + ty)
    const int par = ((n0 + ty) & 1) ^ (mode & 1);  // 0 -> even fold, 1 -> odd fold
    for (int i0 = 0; i0 < g.NRH; i0 += FK) {
        for (int t = threadIdx.x; t < FK * FM; t += 128) {
            int nr = t / FK, ii = t % FK;
            int n = n0 + nr, i = i0 + ii;
            As[ii][nr] = (n < nn && i < g.NRH) ? w[(size_t)n * g.NRH + i] : 0.0;
        }
        for (int t = threadIdx.x; t < FK * FN; t += 128) {
            int ii = t / FN, cc = t % FN;
            int i = i0 + ii, c = c0 + cc;
            double lo = 0.0, hi = 0.0;
            if (i < g.NRH && c < ncol) {
                lo = x[(size_t)i * ncol + c];
                hi = x[(size_t)(g.NR - 1 - i) * ncol + c];
            }
            double e = lo + hi, d = lo - hi;
            if (use_w && i < g.NRH) {
                e *= g.w[i];
                d *= g.w[i];
            }
            Fe[ii][cc] = e;
            Fo[ii][cc] = d;
        }
        __syncthreads();
        const double(*F)[FN] = par ? Fo : Fe;
#pragma unroll
        for (int ii = 0; ii < FK; ++ii) {
            double av[4], bv[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                av[q] = As[ii][ty + 8 * q];
                bv[q] = F[ii][tx * 4 + q];
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = fma(av[p], bv[q], acc[p][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        int n = n0 + ty + 8 * p;
        if (n >= g.NRCHOPDIM) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int c = c0 + tx * 4 + 2 * h;
            if (c >= ncol) continue;
            int k = c >> 1;
            double re = acc[p][2 * h], im = acc[p][2 * h + 1];
            double sr = re, si = im;
            switch (scale) {
                case 1: sr = -re; si = -im; break;
                case 2: { double f = -(double)m; sr = -im * f; si = re * f; } break;  // -i m v
                case 3: { double f = g.ak[k]; sr = -im * f; si = re * f; } break;     //  i k v
                case 4: { double f = (double)m * g.ak[k]; sr = re * f; si = im * f; } break;
                default: break;
            }
            double* dst = o + (size_t)n * ncol + c;
            if (n >= nn) {
                if (!accumulate) { dst[0] = 0.0; dst[1] = 0.0; }
            } else if (accumulate) {
                dst[0] += sr;
                dst[1] += si;
            } else {
                dst[0] = sr;
                dst[1] = si;
            }
        }
    }
}

void k_fold_gemm(const DevGrid& g, const double* Wt, int wt_rows, const double2* in, double2* out, int mode,
                 int scale, int accumulate, int pad, cudaStream_t s) {
    if (dmma_supported(g)) {
        k_fold_gemm_dmma(g, Wt, wt_rows, in, out, mode, scale, accumulate, pad, s);
        return;
    }
    int ncol = 2 * g.NXCHOPDIM;
    int use_w = (mode & 2) ? 1 : 0;
    dim3 grid((ncol + FN - 1) / FN, (g.NRCHOPDIM + FM - 1) / FM, g.NTCHOPDIM);
    fold_gemm_kernel<<<grid, 128, 0, s>>>(g, Wt, wt_rows, (const double*)in, (double*)out, mode & 1, scale,
                                          accumulate, pad, use_w);
    count_launch();
}

}  // namespace mlegs
