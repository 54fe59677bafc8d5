// FP64 Legendre GEMMs on the FP64 tensor path (mma.sync m8n8k4, FP64 in and
// out), used by MLEGS_PREC_FP64 contexts.  Same contracts as the FFMA
// kernels in gemm.cu:
//   RTRAN(A, +1)  (mod_fft.f90:1264-1336): per m and parity p of n,
//       C_p(i, c) = sum_t PF(i, 2t+p) A(2t+p, c),  B(i) = C_0 + C_1,
//       B(NR-1-i) = C_0 - C_1, plus the (m, k) = (0, 0) log term;
//   fold GEMMs    RTRAN(A, -1) (1189-1261) and the EOMUL/OEMUL products of
//       PROJECT (mod_legops.f90:2497-2535, 2548-2648):
//       out(n, c) (+)= s(m, k) sum_{i < NRH} Wt(n, i) F(i, c), F the even or
//       odd fold of the input rows (times w_i for RTRAN(-1)).
// One CTA (4 warps) computes a 32-column tile of one m for all output rows of
// the GEMM: the whole K extent of both operands is staged in shared memory by
// cp.async, then each warp runs m8n8k4 FP64 MMAs over its m-tiles x the
// tile's four n-tiles.
// Fragment layout of m8n8k4.f64 (g = lane / 4, q = lane % 4):
//   a = A[g][q] (8 x 4, row), b = B[q][g] (4 x 8, col), d = D[g][2q], D[g][2q+1].
// Shared-memory row strides are chosen so that a warp's fragment loads need
// only the minimum two wavefronts.
#include "mlegs_internal.h"

#include <algorithm>

namespace mlegs {

namespace {

constexpr int CT = 32;       // output columns per CTA
constexpr int SBS = CT + 8;  // B row stride (doubles), = 8 mod 16

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp16(void* dst, const void* src, bool ok) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(ok ? 16u : 0u)
                 : "memory");
}

__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

}  // namespace

// RTRAN(+1).  smem per parity pass: A [KP][SA] (PF rows t, i contiguous) and
// B [KP][SBS]; the even-parity products stay in registers during the odd pass.
template <int MTW>
__global__ void __launch_bounds__(128) b2p_dmma_kernel(DevGrid g, const double* __restrict__ A,
                                                       double* __restrict__ out, const double* ln, int pad,
                                                       int SA, int KPmax) {
    extern __shared__ double smd[];
    double* As = smd;                       // [KPmax][SA]
    double* Bs = smd + (size_t)KPmax * SA;  // [KPmax][SBS]
    const int m = blockIdx.y, c0 = blockIdx.x * CT;
    const int ncol = 2 * g.NXCHOPDIM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, q = lane & 3;
    const int RT = (g.NRH + 7) / 8;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    const int ne = g.NRCHOPDIM + 1;
    const double* pf = g.pf + (size_t)m * ne * g.NRH;
    const double* a = A + (size_t)m * g.NRCHOPDIM * ncol;
    double acc[2][MTW][4][2];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int i = 0; i < MTW; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[p][i][j][0] = acc[p][i][j][1] = 0.0;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const int kp = p ? nn / 2 : (nn + 1) / 2;
        const int KP = (kp + 3) & ~3;
        if (p) __syncthreads();  // the even pass is done with the buffers
        // stage A: rows t < KP of PF(:, 2t+p) over i (NRH), zero past kp
        const int ach = g.NRH / 2;  // 16-byte chunks per row (NRH is even)
        for (int e = tid; e < KP * ach; e += 128) {
            const int t = e / ach, ch = e - t * ach;
            const bool ok = t < kp;
            cp16(As + (size_t)t * SA + 2 * ch, ok ? pf + (size_t)(2 * t + p) * g.NRH + 2 * ch : pf, ok);
        }
        // stage B: rows t < KP of A(2t+p, c0 .. c0+31), zero past kp / ncol
        for (int e = tid; e < KP * (CT / 2); e += 128) {
            const int t = e / (CT / 2), ch = e - t * (CT / 2);
            const int c = c0 + 2 * ch;
            const bool ok = t < kp && c < ncol;
            cp16(Bs + (size_t)t * SBS + 2 * ch, ok ? a + (size_t)(2 * t + p) * ncol + c : a, ok);
        }
        cp_wait_all();
        __syncthreads();
        for (int k = 0; k < KP; k += 4) {
            double af[MTW], bf[4];
#pragma unroll
            for (int i = 0; i < MTW; ++i) {
                const int mt = warp * MTW + i;
                af[i] = (mt < RT) ? As[(size_t)(k + q) * SA + mt * 8 + gq] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = Bs[(size_t)(k + q) * SBS + j * 8 + gq];
#pragma unroll
            for (int i = 0; i < MTW; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[p][i][j], af[i], bf[j]);
        }
    }
    // butterfly + log term
    const double lnv = (m == 0 && ln) ? *ln : 0.0;
    double* o = out + (size_t)m * g.NR * ncol;
#pragma unroll
    for (int i = 0; i < MTW; ++i) {
        const int row = (warp * MTW + i) * 8 + gq;
        if (row >= g.NRH) continue;
        const int rh = g.NR - 1 - row;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * 8 + 2 * q;
            if (c >= ncol) continue;
            double2 lo = make_double2(acc[0][i][j][0] + acc[1][i][j][0], acc[0][i][j][1] + acc[1][i][j][1]);
            double2 hi = make_double2(acc[0][i][j][0] - acc[1][i][j][0], acc[0][i][j][1] - acc[1][i][j][1]);
            if (c == 0 && lnv != 0.0) {
                lo.x += lnv * g.lnx[row];
                hi.x += lnv * g.lnx[rh];
            }
            *(double2*)(o + (size_t)row * ncol + c) = lo;
            *(double2*)(o + (size_t)rh * ncol + c) = hi;
        }
    }
}

// Fold GEMM for the rows n = 2r + pr of one parity, K-pipelined.  The K rows
// i < NRH go in chunks of KC = 32; per chunk the CTA stages the weight rows
// A [RT*8][SAF] (Wt(n, i0..i0+31)) and the input rows x_i and x_{NR-1-i} of its
// 32 columns in a two-stage cp.async ring; the fold F(i) = (x_i +/- x_{NR-1-i}) w_i
// of a landed chunk is formed once into a shared B buffer for all warps.
constexpr int KCF = 32;          // K rows per chunk
constexpr int SAF = KCF + 4;     // weight row stride (doubles), = 4 mod 16
constexpr int SXF = CT + 8;      // input row stride (doubles), = 8 mod 16

template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32) fold_dmma_kernel(DevGrid g, const double* __restrict__ Wt, int wt_rows,
                                                        const double* __restrict__ in, double* __restrict__ out,
                                                        int mode, int scale, int accumulate, int pad, int use_w,
                                                        int RTmax) {
    extern __shared__ double smd[];
    const int m = blockIdx.z, pr = blockIdx.y, c0 = blockIdx.x * CT;
    const int ncol = 2 * g.NXCHOPDIM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, q = lane & 3;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    const int rows = (g.NRCHOPDIM - pr + 1) / 2;  // output rows n = 2r + pr < NRCHOPDIM
    const int RT = (rows + 7) / 8;
    const int nch = (g.NRH + KCF - 1) / KCF;
    const size_t stA = (size_t)RTmax * 8 * SAF, stX = (size_t)2 * KCF * SXF;
    double* ws = smd + 2 * (stA + stX);           // [nch*KCF] weights (1 without use_w, 0 past NRH)
    double* Bs = ws + nch * KCF;                  // [KCF][SXF] folded chunk, shared by the warps
    const double sgn = (pr ^ mode) ? -1.0 : 1.0;
    const double* w = Wt + (size_t)m * wt_rows * g.NRH;
    const double* x = in + (size_t)m * g.NR * ncol;
    for (int i = tid; i < nch * KCF; i += NW * 32) ws[i] = (i < g.NRH) ? (use_w ? g.w[i] : 1.0) : 0.0;

    // chunk ch -> stage ch & 1: A rows r (weights at i0..i0+31), X rows j < 32 (x_{i0+j}),
    // X rows 32 + j (x_{NR-1-i0-j}); i >= NRH reads as zero
    auto stage = [&](int ch) {
        double* As = smd + (ch & 1) * (stA + stX);
        double* Xs = As + stA;
        const int i0 = ch * KCF;
        for (int e = tid; e < RT * 8 * (KCF / 2); e += NW * 32) {
            const int r = e / (KCF / 2), c2 = e - r * (KCF / 2);
            const int n = 2 * r + pr, i = i0 + 2 * c2;
            const bool ok = n < nn && n < wt_rows && i < g.NRH;
            cp16(As + (size_t)r * SAF + 2 * c2, ok ? w + (size_t)n * g.NRH + i : w, ok);
        }
        for (int e = tid; e < 2 * KCF * (CT / 2); e += NW * 32) {
            const int rr = e / (CT / 2), c2 = e - rr * (CT / 2);
            const int j = rr % KCF, i = i0 + j;
            const int src_row = rr < KCF ? i : g.NR - 1 - i;
            const int c = c0 + 2 * c2;
            const bool ok = i < g.NRH && c < ncol;
            cp16(Xs + (size_t)rr * SXF + 2 * c2, ok ? x + (size_t)src_row * ncol + c : x, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    double acc[MTW][4][2];
#pragma unroll
    for (int t = 0; t < MTW; ++t)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[t][j][0] = acc[t][j][1] = 0.0;
    stage(0);
    for (int ch = 0; ch < nch; ++ch) {
        if (ch + 1 < nch) {
            stage(ch + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const double* As = smd + (ch & 1) * (stA + stX);
        const double* Xs = As + stA;
        for (int e = tid; e < KCF * CT; e += NW * 32) {
            const int j = e / CT, c = e - j * CT;
            Bs[(size_t)j * SXF + c] = (Xs[(size_t)j * SXF + c] + sgn * Xs[(size_t)(KCF + j) * SXF + c]) * ws[ch * KCF + j];
        }
        __syncthreads();
        for (int kk = 0; kk < KCF; kk += 4) {
            const int j = kk + q;
            double af[MTW], bf[4];
#pragma unroll
            for (int t = 0; t < MTW; ++t) {
                const int mt = warp * MTW + t;
                af[t] = (mt < RT) ? As[(size_t)(mt * 8 + gq) * SAF + j] : 0.0;
            }
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) bf[jj] = Bs[(size_t)j * SXF + jj * 8 + gq];
#pragma unroll
            for (int t = 0; t < MTW; ++t)
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) dmma(acc[t][jj], af[t], bf[jj]);
        }
        __syncthreads();  // the stage is refilled by the next iteration's prefetch
    }
    double* o = out + (size_t)m * g.NRCHOPDIM * ncol;
#pragma unroll
    for (int t = 0; t < MTW; ++t) {
        const int r = (warp * MTW + t) * 8 + gq;
        const int n = 2 * r + pr;
        if (r >= rows || n >= g.NRCHOPDIM) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j * 8 + 2 * q;  // even: real part of mode k = c / 2
            if (c >= ncol) continue;
            const double re = acc[t][j][0], im = acc[t][j][1];
            const int kk = c >> 1;
            double sr = re, si = im;
            switch (scale) {
                case 1: sr = -re; si = -im; break;
                case 2: { const double f = -(double)m; sr = -im * f; si = re * f; } break;  // -i m v
                case 3: { const double f = g.ak[kk]; sr = -im * f; si = re * f; } break;    //  i k v
                case 4: { const double f = (double)m * g.ak[kk]; sr = re * f; si = im * f; } break;
                default: break;
            }
            double2* dst = (double2*)(o + (size_t)n * ncol + c);
            if (n >= nn) {
                if (!accumulate) *dst = make_double2(0.0, 0.0);
            } else if (accumulate) {
                const double2 v = *dst;
                *dst = make_double2(v.x + sr, v.y + si);
            } else {
                *dst = make_double2(sr, si);
            }
        }
    }
}

// PROJECT's five EOMUL/OEMUL products (mod_legops.f90:2497-2535) as two
// K-concatenated GEMMs per (m, parity of n) and 32-column tile:
//   PSI = [V | D] . [-i m F0(RUR); -F1(RUP)]                       K = 2 NRH
//   CHI = [D | V | T] . [i k F1(RUR); m k F0(RUP); -F0(UZ)]         K = 3 NRH
// F0 / F1 are the EO / OE folds x_i +/- x_{NR-1-i} of the input rows for the
// output parity; the complex column factors are applied to the folded chunk,
// before the products (the weights are real).  All 5 NRH / 32 chunks go
// through one two-stage cp.async ring; PSI is written after the first 2 NRH,
// CHI at the end, each once and without a read-modify-write.  Segment sg of
// the K extent: 0 (V, RUR, EO, -i m), 1 (D, RUP, OE, -1), 2 (D, RUR, OE, i k),
// 3 (V, RUP, EO, m k), 4 (T, UZ, EO, -1).
template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32) project_dmma_kernel(DevGrid g, const double* __restrict__ V,
                                                           const double* __restrict__ D, const double* __restrict__ T,
                                                           const double* __restrict__ rur,
                                                           const double* __restrict__ rup,
                                                           const double* __restrict__ uz, double* __restrict__ psi,
                                                           double* __restrict__ chi, int RTmax) {
    extern __shared__ double smd[];
    const int m = blockIdx.z, pr = blockIdx.y, c0 = blockIdx.x * CT;
    const int ncol = 2 * g.NXCHOPDIM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, q = lane & 3;
    int nn = g.NRCHOP - m;
    if (nn < 0) nn = 0;
    const int rows = (g.NRCHOPDIM - pr + 1) / 2;
    const int RT = (rows + 7) / 8;
    const int nch = (g.NRH + KCF - 1) / KCF;
    const int total = 5 * nch;
    const size_t stA = (size_t)RTmax * 8 * SAF, stX = (size_t)2 * KCF * SXF;
    double* Bs = smd + 2 * (stA + stX);  // [KCF][SXF] folded, scaled chunk
    const size_t wofs = (size_t)m * g.NRCHOPDIM * g.NRH, xofs = (size_t)m * g.NR * ncol;

    auto stage = [&](int gc) {
        const int sg = gc / nch, i0 = (gc - sg * nch) * KCF;
        const double* w = (sg == 0 || sg == 3 ? V : (sg == 4 ? T : D)) + wofs;
        const double* x = (sg == 0 || sg == 2 ? rur : (sg == 4 ? uz : rup)) + xofs;
        double* As = smd + (gc & 1) * (stA + stX);
        double* Xs = As + stA;
        for (int e = tid; e < RT * 8 * (KCF / 2); e += NW * 32) {
            const int r = e / (KCF / 2), c2 = e - r * (KCF / 2);
            const int n = 2 * r + pr, i = i0 + 2 * c2;
            const bool ok = n < nn && i < g.NRH;
            cp16(As + (size_t)r * SAF + 2 * c2, ok ? w + (size_t)n * g.NRH + i : w, ok);
        }
        for (int e = tid; e < 2 * KCF * (CT / 2); e += NW * 32) {
            const int rr = e / (CT / 2), c2 = e - rr * (CT / 2);
            const int j = rr % KCF, i = i0 + j;
            const int src_row = rr < KCF ? i : g.NR - 1 - i;
            const int c = c0 + 2 * c2;
            const bool ok = i < g.NRH && c < ncol;
            cp16(Xs + (size_t)rr * SXF + 2 * c2, ok ? x + (size_t)src_row * ncol + c : x, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    auto epilogue = [&](double (&acc)[MTW][4][2], double* out) {
        double* o = out + (size_t)m * g.NRCHOPDIM * ncol;
#pragma unroll
        for (int t = 0; t < MTW; ++t) {
            const int r = (warp * MTW + t) * 8 + gq;
            const int n = 2 * r + pr;
            if (r >= rows || n >= g.NRCHOPDIM) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = c0 + j * 8 + 2 * q;
                if (c >= ncol) continue;
                *(double2*)(o + (size_t)n * ncol + c) =
                    n < nn ? make_double2(acc[t][j][0], acc[t][j][1]) : make_double2(0.0, 0.0);
                acc[t][j][0] = acc[t][j][1] = 0.0;
            }
        }
    };

    double acc[MTW][4][2];
#pragma unroll
    for (int t = 0; t < MTW; ++t)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[t][j][0] = acc[t][j][1] = 0.0;
    stage(0);
    for (int gc = 0; gc < total; ++gc) {
        if (gc + 1 < total) {
            stage(gc + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const int sg = gc / nch;
        const double* As = smd + (gc & 1) * (stA + stX);
        const double* Xs = As + stA;
        // fold sign for (parity, EO/OE) and the complex column factor of the segment
        const double sgn = (pr ^ (sg == 1 || sg == 2 ? 1 : 0)) ? -1.0 : 1.0;
        for (int e = tid; e < KCF * (CT / 2); e += NW * 32) {
            const int j = e / (CT / 2), c = 2 * (e - j * (CT / 2));
            const double re = Xs[(size_t)j * SXF + c] + sgn * Xs[(size_t)(KCF + j) * SXF + c];
            const double im = Xs[(size_t)j * SXF + c + 1] + sgn * Xs[(size_t)(KCF + j) * SXF + c + 1];
            const int kk = (c0 + c) >> 1;
            const double ak = (c0 + c < ncol) ? g.ak[kk] : 0.0;
            double sr, si;
            switch (sg) {
                case 0: sr = im * m; si = -re * m; break;                    // -i m v
                case 2: sr = -im * ak; si = re * ak; break;                  //  i k v
                case 3: { const double f = m * ak; sr = re * f; si = im * f; } break;  // m k v
                default: sr = -re; si = -im; break;                          // -v
            }
            Bs[(size_t)j * SXF + c] = sr;
            Bs[(size_t)j * SXF + c + 1] = si;
        }
        __syncthreads();
        for (int kk = 0; kk < KCF; kk += 4) {
            const int j = kk + q;
            double af[MTW], bf[4];
#pragma unroll
            for (int t = 0; t < MTW; ++t) {
                const int mt = warp * MTW + t;
                af[t] = (mt < RT) ? As[(size_t)(mt * 8 + gq) * SAF + j] : 0.0;
            }
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) bf[jj] = Bs[(size_t)j * SXF + jj * 8 + gq];
#pragma unroll
            for (int t = 0; t < MTW; ++t)
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) dmma(acc[t][jj], af[t], bf[jj]);
        }
        if (gc == 2 * nch - 1) epilogue(acc, psi);
        if (gc == total - 1) epilogue(acc, chi);
        __syncthreads();  // the stage is refilled by the next iteration's prefetch
    }
}

// ---------------------------------------------------------------------------

static int pad16_8(int v) { return v + ((8 - v % 16) + 16) % 16; }  // smallest >= v that is 8 mod 16

bool dmma_supported(const DevGrid& g) { return g.NRH <= 128 && g.NRH % 2 == 0 && g.NRCHOPDIM <= 256; }

template <int MTW>
static void b2p_launch(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    const int SA = pad16_8(((g.NRH + 7) / 8) * 8);
    const int KPmax = ((g.NRCHOPDIM + 1) / 2 + 3) & ~3;
    const size_t smem = (size_t)KPmax * (SA + SBS) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(b2p_dmma_kernel<MTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    dim3 grid((2 * g.NXCHOPDIM + CT - 1) / CT, g.NTCHOPDIM);
    b2p_dmma_kernel<MTW><<<grid, 128, smem, s>>>(g, (const double*)a, (double*)b, ln, pad, SA, KPmax);
    count_launch();
}

void k_rtran_b2p_dmma(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    const int RT = (g.NRH + 7) / 8;
    switch ((RT + 3) / 4) {
        case 1: b2p_launch<1>(g, a, b, ln, pad, s); break;
        case 2: b2p_launch<2>(g, a, b, ln, pad, s); break;
        case 3: b2p_launch<3>(g, a, b, ln, pad, s); break;
        default: b2p_launch<4>(g, a, b, ln, pad, s); break;
    }
}

template <int NW, int MTW>
static void fold_launch(const DevGrid& g, const double* Wt, int wt_rows, const double2* in, double2* out, int mode,
                        int scale, int accumulate, int pad, int use_w, cudaStream_t s) {
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    const int nch = (g.NRH + KCF - 1) / KCF;
    const size_t smem =
        (2 * ((size_t)RT * 8 * SAF + (size_t)2 * KCF * SXF) + (size_t)nch * KCF + (size_t)KCF * SXF) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(fold_dmma_kernel<NW, MTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    dim3 grid((2 * g.NXCHOPDIM + CT - 1) / CT, 2, g.NTCHOPDIM);
    fold_dmma_kernel<NW, MTW><<<grid, NW * 32, smem, s>>>(g, Wt, wt_rows, (const double*)in, (double*)out, mode,
                                                          scale, accumulate, pad, use_w, RT);
    count_launch();
}

void k_fold_gemm_dmma(const DevGrid& g, const double* Wt, int wt_rows, const double2* in, double2* out, int mode,
                      int scale, int accumulate, int pad, cudaStream_t s) {
    // m-tiles of the output rows of one parity split over 3 or 4 warps with the least idle tiles
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    const int use_w = (mode & 2) ? 1 : 0;
    const int m4 = (RT + 3) / 4, m3 = (RT + 2) / 3;
    const bool three = 3 * m3 - RT < 4 * m4 - RT && m3 <= 4;
#define FOLD_CASE(NW, MTW) fold_launch<NW, MTW>(g, Wt, wt_rows, in, out, mode & 1, scale, accumulate, pad, use_w, s)
    if (three) {
        switch (m3) {
            case 1: FOLD_CASE(3, 1); break;
            case 2: FOLD_CASE(3, 2); break;
            case 3: FOLD_CASE(3, 3); break;
            default: FOLD_CASE(3, 4); break;
        }
    } else {
        switch (m4) {
            case 1: FOLD_CASE(4, 1); break;
            case 2: FOLD_CASE(4, 2); break;
            case 3: FOLD_CASE(4, 3); break;
            default: FOLD_CASE(4, 4); break;
        }
    }
#undef FOLD_CASE
}

template <int NW, int MTW>
static void project_launch(const DevGrid& g, const double* V, const double* D, const double* T, const double2* rur,
                           const double2* rup, const double2* uz, double2* psi, double2* chi, cudaStream_t s) {
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    const size_t smem = (2 * ((size_t)RT * 8 * SAF + (size_t)2 * KCF * SXF) + (size_t)KCF * SXF) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(project_dmma_kernel<NW, MTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    dim3 grid((2 * g.NXCHOPDIM + CT - 1) / CT, 2, g.NTCHOPDIM);
    project_dmma_kernel<NW, MTW><<<grid, NW * 32, smem, s>>>(g, V, D, T, (const double*)rur, (const double*)rup,
                                                             (const double*)uz, (double*)psi, (double*)chi, RT);
    count_launch();
}

void k_project_dmma(const DevGrid& g, const double* V, const double* D, const double* T, const double2* rur,
                    const double2* rup, const double2* uz, double2* psi, double2* chi, cudaStream_t s) {
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    const int m4 = (RT + 3) / 4, m3 = (RT + 2) / 3;
    const bool three = 3 * m3 - RT < 4 * m4 - RT && m3 <= 4;
#define PROJ_CASE(NW, MTW) project_launch<NW, MTW>(g, V, D, T, rur, rup, uz, psi, chi, s)
    if (three) {
        switch (m3) {
            case 1: PROJ_CASE(3, 1); break;
            case 2: PROJ_CASE(3, 2); break;
            case 3: PROJ_CASE(3, 3); break;
            default: PROJ_CASE(3, 4); break;
        }
    } else {
        switch (m4) {
            case 1: PROJ_CASE(4, 1); break;
            case 2: PROJ_CASE(4, 2); break;
            case 3: PROJ_CASE(4, 3); break;
            default: PROJ_CASE(4, 4); break;
        }
    }
#undef PROJ_CASE
}

}  // namespace mlegs
