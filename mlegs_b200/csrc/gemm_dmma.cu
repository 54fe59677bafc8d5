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

}  // namespace

// RTRAN(+1).  Per m, the K rows of both parities (t < kp_p, n = 2t + p) go in
// chunks of KCB = 16 through an NST_B2P-stage cp.async ring: A [KCB][SA] (PF rows
// n, i contiguous) and B [KCB][SBS] (A(n, c0 .. c0+31)).  The even- and
// odd-parity products accumulate in separate registers; the epilogue forms
// B(i) = C_0 + C_1 and B(NR-1-i) = C_0 - C_1.  The output-row m-tiles go
// round-robin over NW warps.
constexpr int KCB = 16;
constexpr int NST_B2P = 2;   // ring stages of b2p_dmma_kernel
constexpr int NST_FOLD = 2;  // ring stages of legfold_dmma_kernel
constexpr int NST_PFFF = 2;  // ring stages of projfff_dmma_kernel

// One (m, 8 NJ-column) tile of RTRAN(+1): the body of b2p_dmma_kernel (NJ = 4),
// also run per work item by the grouped ensemble kernel (ensemble.cu).
template <int NW, int MTW, int NJ = 4>
__device__ __forceinline__ void b2p_tile(const DevGrid& g, const double* __restrict__ A, double* __restrict__ out,
                                         const double* ln, int pad, int SA, int m, int c0, double* smd) {
    const size_t stg = (size_t)KCB * (SA + SBS);
    const int ncol = 2 * g.NXCHOPDIM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, q = lane & 3;
    const int RT = (g.NRH + 7) / 8;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    const int kp0 = (nn + 1) / 2, kp1 = nn / 2;
    const int nc0 = (kp0 + KCB - 1) / KCB, nc1 = (kp1 + KCB - 1) / KCB;
    const int total = nc0 + nc1;
    const int ne = g.NRCHOPDIM + 1;
    const double* pf = g.pf + (size_t)m * ne * g.NRH;
    const double* a = A + (size_t)m * g.NRCHOPDIM * ncol;
    const int ach = g.NRH / 2;  // 16-byte chunks per PF row (NRH is even)
    // (row, chunk) of this thread's first PF element and the step per pass, so
    // the staging loop needs no division
    const int tt0 = tid / ach, ch0 = tid - tt0 * ach;
    const int dtt = (NW * 32) / ach, dch = (NW * 32) - dtt * ach;

    auto stage = [&](int cidx) {
        const int p = cidx < nc0 ? 0 : 1;
        const int t0 = (cidx - (p ? nc0 : 0)) * KCB, kp = p ? kp1 : kp0;
        double* As = smd + (cidx % NST_B2P) * stg;
        double* Bs = As + (size_t)KCB * SA;
        int tt = tt0, ch = ch0;
        for (int e = tid; e < KCB * ach; e += NW * 32) {
            const int t = t0 + tt;
            const bool ok = t < kp;
            cp16(As + (size_t)tt * SA + 2 * ch, ok ? pf + (size_t)(2 * t + p) * g.NRH + 2 * ch : pf, ok);
            tt += dtt;
            ch += dch;
            if (ch >= ach) {
                ch -= ach;
                ++tt;
            }
        }
        for (int e = tid; e < KCB * (4 * NJ); e += NW * 32) {
            const int tt = e / (4 * NJ), ch = e - tt * (4 * NJ);
            const int t = t0 + tt, c = c0 + 2 * ch;
            const bool ok = t < kp && c < ncol;
            cp16(Bs + (size_t)tt * SBS + 2 * ch, ok ? a + (size_t)(2 * t + p) * ncol + c : a, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    auto mma_chunk = [&](double (&acc)[MTW][NJ][2], const double* As, const double* Bs, int ksteps) {
#pragma unroll
        for (int s4 = 0; s4 < KCB / 4; ++s4) {
            if (s4 < ksteps) {
                const int k = 4 * s4 + q;
                double bf[NJ];
#pragma unroll
                for (int j = 0; j < NJ; ++j) bf[j] = Bs[(size_t)k * SBS + j * 8 + gq];
#pragma unroll
                for (int i = 0; i < MTW; ++i) {
                    const int mt = warp + NW * i;
                    if (mt < RT) {
                        const double af = As[(size_t)k * SA + mt * 8 + gq];
#pragma unroll
                        for (int j = 0; j < NJ; ++j) dmma(acc[i][j], af, bf[j]);
                    }
                }
            }
        }
    };

    double acc0[MTW][NJ][2], acc1[MTW][NJ][2];
#pragma unroll
    for (int i = 0; i < MTW; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc0[i][j][0] = acc0[i][j][1] = acc1[i][j][0] = acc1[i][j][1] = 0.0;
    // ring: NST_B2P - 1 chunks in flight ahead of the one computed; every
    // iteration commits one group (empty past the end), so the wait count is fixed
#pragma unroll
    for (int c = 0; c < NST_B2P - 1; ++c) {
        if (c < total) stage(c);
        else asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int cidx = 0; cidx < total; ++cidx) {
        if (cidx + NST_B2P - 1 < total) stage(cidx + NST_B2P - 1);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" ::"n"(NST_B2P - 1) : "memory");
        __syncthreads();
        const double* As = smd + (cidx % NST_B2P) * stg;
        const double* Bs = As + (size_t)KCB * SA;
        const int p = cidx < nc0 ? 0 : 1;
        const int t0 = (cidx - (p ? nc0 : 0)) * KCB, kp = p ? kp1 : kp0;
        const int ksteps = (min(KCB, kp - t0) + 3) / 4;
        if (p == 0) mma_chunk(acc0, As, Bs, ksteps);
        else mma_chunk(acc1, As, Bs, ksteps);
        __syncthreads();  // the stage is refilled by the next iteration's prefetch
    }
    // butterfly + log term
    const double lnv = (m == 0 && ln) ? *ln : 0.0;
    double* o = out + (size_t)m * g.NR * ncol;
#pragma unroll
    for (int i = 0; i < MTW; ++i) {
        const int row = (warp + NW * i) * 8 + gq;
        if (row >= g.NRH) continue;
        const int rh = g.NR - 1 - row;
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const int c = c0 + j * 8 + 2 * q;
            if (c >= ncol) continue;
            double2 lo = make_double2(acc0[i][j][0] + acc1[i][j][0], acc0[i][j][1] + acc1[i][j][1]);
            double2 hi = make_double2(acc0[i][j][0] - acc1[i][j][0], acc0[i][j][1] - acc1[i][j][1]);
            if (c == 0 && lnv != 0.0) {
                lo.x += lnv * g.lnx[row];
                hi.x += lnv * g.lnx[rh];
            }
            *(double2*)(o + (size_t)row * ncol + c) = lo;
            *(double2*)(o + (size_t)rh * ncol + c) = hi;
        }
    }
}

template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32) b2p_dmma_kernel(DevGrid g, const double* __restrict__ A,
                                                           double* __restrict__ out, const double* ln, int pad,
                                                           int SA) {
    extern __shared__ double smd[];
    b2p_tile<NW, MTW>(g, A, out, ln, pad, SA, blockIdx.y, blockIdx.x * CT, smd);
}

// Fold GEMMs: RTRAN(-1) and PROJECT's five EOMUL/OEMUL products.  One CTA
// computes the output rows n = 2r + pr of one parity, one m and 32 columns,
// over a K extent of nseg segments of NRH rows each:
//   out0 = sum_{seg < split} Wt_seg . (s_seg F_seg),  out1 = sum_{seg >= split} ...
// where F_seg is the EO or OE fold x_i +/- x_{NR-1-i} of the segment's input
// rows (times w_i for RTRAN(-1)) and s_seg a complex column factor, applied to
// the folded chunk before the products (the weights are real).  PROJECT
// (mod_legops.f90:2497-2535) is
//   PSI = [V | D] . [-i m F0(RUR); -F1(RUP)],
//   CHI = [D | V | T] . [i k F1(RUR); m k F0(RUP); -F0(UZ)].
// The K rows go in chunks of KC2 = 16 through a two-stage cp.async ring (the
// weight rows of the chunk and the input rows x_i, x_{NR-1-i} of the 32
// columns); the folded, scaled chunk is formed once in shared memory for all
// warps.  The m-tiles (8 output rows) go round-robin over the warps, and tiles
// whose rows all lie at n >= NRCHOPS(m) issue no MMAs.  About 49 KB of shared
// memory lets four CTAs share an SM.
constexpr int KC2 = 16;       // K rows per chunk
constexpr int SA2 = KC2 + 4;  // weight row stride (doubles), = 4 mod 16
constexpr int SX2 = CT + 8;   // input / folded row stride (doubles), = 8 mod 16


template <class T>
__device__ __forceinline__ T pick5(const T (&a)[5], int i) {
    T v = a[0];
#pragma unroll
    for (int j = 1; j < 5; ++j)
        if (i == j) v = a[j];
    return v;
}

// One (m, output parity, 8 NJ-column) tile of the fold GEMMs: the body of
// legfold_dmma_kernel (NJ = 4), also run per work item by the grouped ensemble
// kernel.
template <int NW, int MTW, int NJ = 4>
__device__ __forceinline__ void legfold_tile(const DevGrid& g, const FoldArgs& fa, int RTmax, int m, int pr, int c0,
                                             double* smd) {
    const int ncol = 2 * g.NXCHOPDIM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, q = lane & 3;
    int nn = g.NRCHOP + fa.pad - m;
    if (nn < 0) nn = 0;
    const int nw = min(nn, fa.wt_rows);                    // rows with weights
    const int rows = (g.NRCHOPDIM - pr + 1) / 2;           // output rows n = 2r + pr < NRCHOPDIM
    const int rv = min(rows, max(0, (nw - pr + 1) / 2));   // of them with weights
    const int RTv = (rv + 7) / 8;
    const int nch = (g.NRH + KC2 - 1) / KC2;
    const int total = fa.nseg * nch;
    const size_t stA = (size_t)RTmax * 8 * SA2, stX = (size_t)2 * KC2 * SX2;
    double* Bs = smd + NST_FOLD * (stA + stX);  // [KC2][SX2] folded, scaled chunk
    double* ws = Bs + KC2 * SX2;         // [nch * KC2] fold weights (w_i, or 1), 0 past NRH
    const size_t wofs = (size_t)m * fa.wt_rows * g.NRH, xofs = (size_t)m * g.NR * ncol;
    for (int i = tid; i < nch * KC2; i += NW * 32) ws[i] = (i < g.NRH) ? (fa.use_w ? g.w[i] : 1.0) : 0.0;
    // fold pass: thread -> column pair p2 (fixed), rows j = tid / (4 NJ) + (NW * 32 / (4 NJ)) t
    constexpr int NP2 = 4 * NJ;
    const int p2 = tid % NP2;
    const int cp = c0 + 2 * p2;
    const double akv = (cp < ncol) ? g.ak[cp >> 1] : 0.0;

    auto stage = [&](int gc) {
        const int sg = gc / nch, i0 = (gc - sg * nch) * KC2;
        const double* w = pick5(fa.w, sg) + wofs;
        const double* x = pick5(fa.x, sg) + xofs;
        double* As = smd + (gc % NST_FOLD) * (stA + stX);
        double* Xs = As + stA;
        for (int e = tid; e < RTv * 8 * (KC2 / 2); e += NW * 32) {
            const int r = e / (KC2 / 2), c2 = e - r * (KC2 / 2);
            const int n = 2 * r + pr, i = i0 + 2 * c2;
            const bool ok = n < nw && i < g.NRH;
            cp16(As + (size_t)r * SA2 + 2 * c2, ok ? w + (size_t)n * g.NRH + i : w, ok);
        }
        for (int e = tid; e < 2 * KC2 * (4 * NJ); e += NW * 32) {
            const int rr = e / (4 * NJ), c2 = e - rr * (4 * NJ);
            const int j = rr % KC2, i = i0 + j;
            const int src_row = rr < KC2 ? i : g.NR - 1 - i;
            const int c = c0 + 2 * c2;
            const bool ok = i < g.NRH && c < ncol;
            cp16(Xs + (size_t)rr * SX2 + 2 * c2, ok ? x + (size_t)src_row * ncol + c : x, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    auto epilogue = [&](double (&acc)[MTW][NJ][2], double* out) {
        double* o = out + (size_t)m * g.NRCHOPDIM * ncol;
#pragma unroll
        for (int t = 0; t < MTW; ++t) {
            const int r = (warp + NW * t) * 8 + gq;
            const int n = 2 * r + pr;
            if (r >= rows || n >= g.NRCHOPDIM) continue;
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const int c = c0 + j * 8 + 2 * q;
                double2 v = make_double2(acc[t][j][0], acc[t][j][1]);
                acc[t][j][0] = acc[t][j][1] = 0.0;
                if (c >= ncol) continue;
                double2* dst = (double2*)(o + (size_t)n * ncol + c);
                if (n >= nn) {
                    if (!fa.accumulate) *dst = make_double2(0.0, 0.0);
                } else if (fa.accumulate) {
                    const double2 u = *dst;
                    *dst = make_double2(u.x + v.x, u.y + v.y);
                } else {
                    *dst = v;
                }
            }
        }
    };

    double acc[MTW][NJ][2];
#pragma unroll
    for (int t = 0; t < MTW; ++t)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc[t][j][0] = acc[t][j][1] = 0.0;
#pragma unroll
    for (int c = 0; c < NST_FOLD - 1; ++c) {
        if (c < total) stage(c);
        else asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int gc = 0; gc < total; ++gc) {
        if (gc + NST_FOLD - 1 < total) stage(gc + NST_FOLD - 1);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" ::"n"(NST_FOLD - 1) : "memory");
        __syncthreads();
        const int sg = gc / nch, ch = gc - sg * nch;
        const double* As = smd + (gc % NST_FOLD) * (stA + stX);
        const double* Xs = As + stA;
        const double sgn = (pr ^ pick5(fa.mode, sg)) ? -1.0 : 1.0;
        const int sc = pick5(fa.scale, sg);
        for (int j = tid / NP2; j < KC2; j += (NW * 32) / NP2) {
            const double2 top = *(const double2*)(Xs + (size_t)j * SX2 + 2 * p2);
            const double2 bot = *(const double2*)(Xs + (size_t)(KC2 + j) * SX2 + 2 * p2);
            const double wv = ws[ch * KC2 + j];
            const double re = (top.x + sgn * bot.x) * wv, im = (top.y + sgn * bot.y) * wv;
            double2 v;
            switch (sc) {
                case 1: v = make_double2(-re, -im); break;
                case 2: v = make_double2(im * m, -re * m); break;  // -i m v
                case 3: v = make_double2(-im * akv, re * akv); break;  // i k v
                case 4: { const double f = m * akv; v = make_double2(re * f, im * f); } break;  // m k v
                default: v = make_double2(re, im); break;
            }
            *(double2*)(Bs + (size_t)j * SX2 + 2 * p2) = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC2; kk += 4) {
            const int j = kk + q;
            double bf[NJ];
#pragma unroll
            for (int jj = 0; jj < NJ; ++jj) bf[jj] = Bs[(size_t)j * SX2 + jj * 8 + gq];
#pragma unroll
            for (int t = 0; t < MTW; ++t) {
                const int mt = warp + NW * t;
                if (mt < RTv) {
                    const double af = As[(size_t)(mt * 8 + gq) * SA2 + j];
#pragma unroll
                    for (int jj = 0; jj < NJ; ++jj) dmma(acc[t][jj], af, bf[jj]);
                }
            }
        }
        if (gc == fa.split * nch - 1 || gc == total - 1) epilogue(acc, gc < fa.split * nch ? fa.out0 : fa.out1);
        __syncthreads();  // the stage is refilled by the next iteration's prefetch
    }
}

template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32, 4) legfold_dmma_kernel(DevGrid g, FoldArgs fa, int RTmax) {
    extern __shared__ double smd[];
    legfold_tile<NW, MTW>(g, fa, RTmax, blockIdx.z, blockIdx.y, blockIdx.x * CT, smd);
}

// PROJECT of velocity fields given as FFF coefficients, as one FFF -> FFF
// product per m.  RTRAN(+1) followed by the EO/OE fold is, for output parity
// pr and fold mode, 2 C_p with p = pr ^ mode (C_p the parity-p half of the
// RTRAN(+1) product), so each fold product W . F(RTRAN(x)) equals
//   Comp_W(n, n') x(n'),  Comp_W(n, n') = 2 sum_{i < NRH} W(n, i) PF(n', i),
// over input rows n' of parity p (n, n' < NRCHOPS(m) at pad 0).  The
// composite matrices are formed once per context (proj_comp_kernel), stored
// [m][pr][r][t] for n = 2r + pr, n' = 2t + p; PROJECT then costs a third of
// the FLOPs of RTRAN(+1) x 3 plus the five fold products and never writes PFF.
// The complex column factors (-i m, -1, i k, m k, -1) are applied to each B
// fragment as it is read (a re/im swap and a per-lane real factor).
__global__ void proj_comp_kernel(DevGrid g, const double* __restrict__ W, int p_flip, double* __restrict__ Cm,
                                 int RC, int KPC) {
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t total = (size_t)g.NTCHOPDIM * 2 * RC * KPC;
    if (idx >= total) return;
    const int t = (int)(idx % KPC);
    const int r = (int)((idx / KPC) % RC);
    const int pr = (int)((idx / ((size_t)KPC * RC)) % 2);
    const int m = (int)(idx / ((size_t)KPC * RC * 2));
    int nn = g.NRCHOP - m;
    if (nn < 0) nn = 0;
    const int n = 2 * r + pr, np = 2 * t + (pr ^ p_flip);
    double v = 0.0;
    if (n < nn && n < g.NRCHOPDIM && np < nn) {
        const double* w = W + ((size_t)m * g.NRCHOPDIM + n) * g.NRH;
        const double* pf = g.pf + ((size_t)m * (g.NRCHOPDIM + 1) + np) * g.NRH;
        for (int i = 0; i < g.NRH; ++i) v += w[i] * pf[i];
        v *= 2.0;
    }
    Cm[idx] = v;
}

struct ProjFffArgs {
    const double* C[5];  // composite per segment: CV, CD, CD, CV, CT
    const double* x[5];  // FFF inputs: RUR, RUP, RUR, RUP, UZ
    double* psi;
    double* chi;
};

template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32, 5) projfff_dmma_kernel(DevGrid g, ProjFffArgs pa, int RC, int KPC,
                                                                 int RTmax) {
    extern __shared__ double smd[];
    const int m = blockIdx.z, pr = blockIdx.y, c0 = blockIdx.x * CT;
    const int ncol = 2 * g.NXCHOPDIM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, q = lane & 3;
    int nn = g.NRCHOP - m;
    if (nn < 0) nn = 0;
    const int rows = (g.NRCHOPDIM - pr + 1) / 2;
    const int rv = min(rows, max(0, (nn - pr + 1) / 2));
    const int RTv = (rv + 7) / 8;
    // input-row parity of the segments: p = pr for EO (0, 3, 4), pr ^ 1 for OE (1, 2)
    const int kpS = max(0, (nn - pr + 1) / 2), kpO = max(0, (nn - (pr ^ 1) + 1) / 2);
    const int nS = (kpS + KC2 - 1) / KC2, nO = (kpO + KC2 - 1) / KC2;
    const int npsi = nS + nO, total = npsi + nO + 2 * nS;
    const size_t stA = (size_t)RTmax * 8 * SA2, stB = (size_t)KC2 * SX2;
    const size_t cofs = (((size_t)m * 2 + pr) * RC) * KPC, xofs = (size_t)m * g.NRCHOPDIM * ncol;

    auto locate = [&](int gc, int& sg, int& ch) {  // chunk -> (segment, chunk in segment)
        int b = gc;
        sg = 0;
        if (b >= nS) {
            b -= nS;
            sg = 1;
            if (b >= nO) {
                b -= nO;
                sg = 2;
                if (b >= nO) {
                    b -= nO;
                    sg = 3;
                    if (b >= nS) {
                        b -= nS;
                        sg = 4;
                    }
                }
            }
        }
        ch = b;
    };
    auto stage = [&](int gc) {
        int sg, ch;
        locate(gc, sg, ch);
        const bool odd = (sg == 1 || sg == 2);
        const int kp = odd ? kpO : kpS, p = pr ^ (odd ? 1 : 0), t0 = ch * KC2;
        const double* cm = pick5(pa.C, sg) + cofs;
        const double* x = pick5(pa.x, sg) + xofs;
        double* As = smd + (gc % NST_PFFF) * (stA + stB);
        double* Bs = As + stA;
        for (int e = tid; e < RTv * 8 * (KC2 / 2); e += NW * 32) {
            const int r = e / (KC2 / 2), c2 = e - r * (KC2 / 2);
            const int t = t0 + 2 * c2;
            const bool ok = r < rv && t < kp;
            cp16(As + (size_t)r * SA2 + 2 * c2, ok ? cm + (size_t)r * KPC + t : cm, ok);
        }
        for (int e = tid; e < KC2 * (CT / 2); e += NW * 32) {
            const int tt = e / (CT / 2), c2 = e - tt * (CT / 2);
            const int t = t0 + tt, c = c0 + 2 * c2;
            const bool ok = t < kp && c < ncol;
            cp16(Bs + (size_t)tt * SX2 + 2 * c2, ok ? x + (size_t)(2 * t + p) * ncol + c : x, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    auto epilogue = [&](double (&acc)[MTW][4][2], double* out) {
        double* o = out + (size_t)m * g.NRCHOPDIM * ncol;
#pragma unroll
        for (int t = 0; t < MTW; ++t) {
            const int r = (warp + NW * t) * 8 + gq;
            const int n = 2 * r + pr;
            if (r >= rows || n >= g.NRCHOPDIM) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = c0 + j * 8 + 2 * q;
                const double2 v = n < nn ? make_double2(acc[t][j][0], acc[t][j][1]) : make_double2(0.0, 0.0);
                acc[t][j][0] = acc[t][j][1] = 0.0;
                if (c < ncol) *(double2*)(o + (size_t)n * ncol + c) = v;
            }
        }
    };

    // per-lane B-fragment factors: lane column c = c0 + 8 jj + gq (gq even: real part)
    double akv[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const int c = c0 + jj * 8 + gq;
        akv[jj] = (c < ncol) ? g.ak[c >> 1] : 0.0;
    }
    const double md = (double)m, ev = (gq & 1) ? -1.0 : 1.0;  // ev: +1 on the real lanes

    double acc[MTW][4][2];
#pragma unroll
    for (int t = 0; t < MTW; ++t)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[t][j][0] = acc[t][j][1] = 0.0;
    if (npsi == 0) epilogue(acc, pa.psi);
    if (total == npsi) epilogue(acc, pa.chi);
#pragma unroll
    for (int c = 0; c < NST_PFFF - 1; ++c) {
        if (c < total) stage(c);
        else asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int gc = 0; gc < total; ++gc) {
        if (gc + NST_PFFF - 1 < total) stage(gc + NST_PFFF - 1);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" ::"n"(NST_PFFF - 1) : "memory");
        __syncthreads();
        int sg, ch;
        locate(gc, sg, ch);
        const bool odd = (sg == 1 || sg == 2);
        const int kp = odd ? kpO : kpS;
        const int ksteps = (min(KC2, kp - ch * KC2) + 3) / 4;
        // B factor: -i m (swap, +m on real lanes), -1, i k (swap, -k on real lanes), m k, -1
        const bool swap = (sg == 0 || sg == 2);
        double f[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            switch (sg) {
                case 0: f[jj] = ev * md; break;
                case 2: f[jj] = -ev * akv[jj]; break;
                case 3: f[jj] = md * akv[jj]; break;
                default: f[jj] = -1.0; break;
            }
        }
        const int bcol = swap ? (gq ^ 1) : gq;
        const double* As = smd + (gc % NST_PFFF) * (stA + stB);
        const double* Bs = As + stA;
#pragma unroll
        for (int s4 = 0; s4 < KC2 / 4; ++s4) {
            if (s4 < ksteps) {
                const int j = 4 * s4 + q;
                double bf[4];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) bf[jj] = Bs[(size_t)j * SX2 + jj * 8 + bcol] * f[jj];
#pragma unroll
                for (int t = 0; t < MTW; ++t) {
                    const int mt = warp + NW * t;
                    if (mt < RTv) {
                        const double af = As[(size_t)(mt * 8 + gq) * SA2 + j];
#pragma unroll
                        for (int jj = 0; jj < 4; ++jj) dmma(acc[t][jj], af, bf[jj]);
                    }
                }
            }
        }
        if (gc == npsi - 1) epilogue(acc, pa.psi);
        if (gc == total - 1) epilogue(acc, pa.chi);
        __syncthreads();  // the stage is refilled by the next iteration's prefetch
    }
}

// ---------------------------------------------------------------------------

static int pad16_8(int v) { return v + ((8 - v % 16) + 16) % 16; }  // smallest >= v that is 8 mod 16

bool dmma_supported(const DevGrid& g) { return g.NRH <= 128 && g.NRH % 2 == 0 && g.NRCHOPDIM <= 256; }

template <int NW, int MTW>
static void b2p_launch(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    const int SA = pad16_8(((g.NRH + 7) / 8) * 8);
    const size_t smem = NST_B2P * (size_t)KCB * (SA + SBS) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(b2p_dmma_kernel<NW, MTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    dim3 grid((2 * g.NXCHOPDIM + CT - 1) / CT, g.NTCHOPDIM);
    b2p_dmma_kernel<NW, MTW><<<grid, NW * 32, smem, s>>>(g, (const double*)a, (double*)b, ln, pad, SA);
    count_launch();
}

// The NRH / 8 output m-tiles go round-robin over 6 warps.
void k_rtran_b2p_dmma(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    // 4 warps per CTA: the small CTAs (about 140 registers a thread, 36 KB of
    // shared memory) run three to an SM; the m-tiles go round-robin over the warps
    const int RT = (g.NRH + 7) / 8;
    switch ((RT + 3) / 4) {
        case 1: b2p_launch<4, 1>(g, a, b, ln, pad, s); break;
        case 2: b2p_launch<4, 2>(g, a, b, ln, pad, s); break;
        case 3: b2p_launch<4, 3>(g, a, b, ln, pad, s); break;
        default: b2p_launch<4, 4>(g, a, b, ln, pad, s); break;
    }
}

template <int NW, int MTW>
static void legfold_launch(const DevGrid& g, const FoldArgs& fa, cudaStream_t s) {
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    const int nch = (g.NRH + KC2 - 1) / KC2;
    const size_t smem =
        (NST_FOLD * ((size_t)RT * 8 * SA2 + (size_t)2 * KC2 * SX2) + (size_t)KC2 * SX2 + (size_t)nch * KC2) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(legfold_dmma_kernel<NW, MTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    dim3 grid((2 * g.NXCHOPDIM + CT - 1) / CT, 2, g.NTCHOPDIM);
    legfold_dmma_kernel<NW, MTW><<<grid, NW * 32, smem, s>>>(g, fa, RT);
    count_launch();
}

// The output-row m-tiles of one parity go round-robin over 4 warps.
static void legfold(const DevGrid& g, const FoldArgs& fa, cudaStream_t s) {
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    switch ((RT + 3) / 4) {
        case 1: legfold_launch<4, 1>(g, fa, s); break;
        case 2: legfold_launch<4, 2>(g, fa, s); break;
        case 3: legfold_launch<4, 3>(g, fa, s); break;
        default: legfold_launch<4, 4>(g, fa, s); break;
    }
}

void k_fold_gemm_dmma(const DevGrid& g, const double* Wt, int wt_rows, const double2* in, double2* out, int mode,
                      int scale, int accumulate, int pad, cudaStream_t s) {
    FoldArgs fa{};
    fa.w[0] = Wt;
    fa.x[0] = (const double*)in;
    fa.mode[0] = mode & 1;
    fa.scale[0] = scale;
    fa.nseg = fa.split = 1;
    fa.out0 = fa.out1 = (double*)out;
    fa.wt_rows = wt_rows;
    fa.pad = pad;
    fa.use_w = (mode & 2) ? 1 : 0;
    fa.accumulate = accumulate;
    legfold(g, fa, s);
}

void k_project_dmma(const DevGrid& g, const double* V, const double* D, const double* T, const double2* rur,
                    const double2* rup, const double2* uz, double2* psi, double2* chi, cudaStream_t s) {
    FoldArgs fa{};
    const double* w[5] = {V, D, D, V, T};
    const double2* x[5] = {rur, rup, rur, rup, uz};
    const int mode[5] = {0, 1, 1, 0, 0}, scale[5] = {2, 1, 3, 4, 1};
    for (int q = 0; q < 5; ++q) {
        fa.w[q] = w[q];
        fa.x[q] = (const double*)x[q];
        fa.mode[q] = mode[q];
        fa.scale[q] = scale[q];
    }
    fa.nseg = 5;
    fa.split = 2;
    fa.out0 = (double*)psi;
    fa.out1 = (double*)chi;
    fa.wt_rows = g.NRCHOPDIM;
    fa.pad = 0;
    fa.use_w = 0;
    fa.accumulate = 0;
    legfold(g, fa, s);
}

size_t proj_comp_doubles(const DevGrid& g) {
    const int RC = (g.NRCHOPDIM + 1) / 2, KPC = (((g.NRCHOP + 1) / 2) + KC2 - 1) / KC2 * KC2;
    return (size_t)g.NTCHOPDIM * 2 * RC * KPC;
}

void k_proj_comp(const DevGrid& g, const double* W, int p_flip, double* Cm, cudaStream_t s) {
    const int RC = (g.NRCHOPDIM + 1) / 2, KPC = (((g.NRCHOP + 1) / 2) + KC2 - 1) / KC2 * KC2;
    const size_t n = (size_t)g.NTCHOPDIM * 2 * RC * KPC;
    proj_comp_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, W, p_flip, Cm, RC, KPC);
    count_launch();
}

template <int NW, int MTW>
static void projfff_launch(const DevGrid& g, const ProjFffArgs& pa, cudaStream_t s) {
    const int RC = (g.NRCHOPDIM + 1) / 2, KPC = (((g.NRCHOP + 1) / 2) + KC2 - 1) / KC2 * KC2;
    const int RT = (RC + 7) / 8;
    const size_t smem = NST_PFFF * ((size_t)RT * 8 * SA2 + (size_t)KC2 * SX2) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(projfff_dmma_kernel<NW, MTW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    dim3 grid((2 * g.NXCHOPDIM + CT - 1) / CT, 2, g.NTCHOPDIM);
    projfff_dmma_kernel<NW, MTW><<<grid, NW * 32, smem, s>>>(g, pa, RC, KPC, RT);
    count_launch();
}

void k_project_fff_dmma(const DevGrid& g, const double* CV, const double* CD, const double* CT_, double2* rur,
                        double2* rup, double2* uz, double2* psi, double2* chi, double* psi_ln, const double* Lfff,
                        cudaStream_t s, double* chi_ln) {
    // VEL2PLN on RUP's (0, 0) column first: it changes RUP's input to the products
    launch_vel2pln_fff(g, rup, psi_ln, Lfff, s, chi_ln);
    ProjFffArgs pa;
    const double* C[5] = {CV, CD, CD, CV, CT_};
    const double2* x[5] = {rur, rup, rur, rup, uz};
    for (int q = 0; q < 5; ++q) {
        pa.C[q] = C[q];
        pa.x[q] = (const double*)x[q];
    }
    pa.psi = (double*)psi;
    pa.chi = (double*)chi;
    const int RT = ((g.NRCHOPDIM + 1) / 2 + 7) / 8;
    switch ((RT + 3) / 4) {
        case 1: projfff_launch<4, 1>(g, pa, s); break;
        case 2: projfff_launch<4, 2>(g, pa, s); break;
        case 3: projfff_launch<4, 3>(g, pa, s); break;
        default: projfff_launch<4, 4>(g, pa, s); break;
    }
}


// ---------------------------------------------------------------------------
// Grouped persistent Legendre GEMMs for ensembles of instances of different
// grids (ensemble.cu).  One launch covers every RTRAN(+1) (or every fold
// product) of every instance: the work items are (problem, m[, parity],
// column tile) tiles numbered consecutively problem by problem; persistent
// CTAs take the next tile from a global counter (atomicAdd, no waiting on
// other CTAs) and run the same tile bodies as the single-grid kernels, with
// the problem's own grid and a per-problem column-tile width (8 * nj columns,
// nj = 2 or 4, chosen per class by the ensemble's autotuner).
namespace {

__device__ __forceinline__ int find_problem(const int* __restrict__ first, int np, int tile) {
    int lo = 0, hi = np - 1;  // largest i with first[i] <= tile
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32) grouped_b2p_kernel(const GroupB2P* __restrict__ pr,
                                                              const int* __restrict__ first, int np, int total,
                                                              int* next) {
    extern __shared__ double smd[];
    __shared__ int tile_s;
    for (;;) {
        if (threadIdx.x == 0) tile_s = atomicAdd(next, 1);
        __syncthreads();
        const int tile = tile_s;
        __syncthreads();
        if (tile >= total) break;
        const GroupB2P P = pr[find_problem(first, np, tile)];
        const int local = tile - P.first;
        const int m = local / P.ntx, cx = local - m * P.ntx;
        if (P.nj == 2) b2p_tile<NW, MTW, 2>(P.g, P.in, P.out, P.ln, P.pad, P.SA, m, cx * 16, smd);
        else b2p_tile<NW, MTW, 4>(P.g, P.in, P.out, P.ln, P.pad, P.SA, m, cx * 32, smd);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

template <int NW, int MTW>
__global__ void __launch_bounds__(NW * 32) grouped_fold_kernel(const GroupFold* __restrict__ pr,
                                                               const int* __restrict__ first, int np, int total,
                                                               int* next) {
    extern __shared__ double smd[];
    __shared__ int tile_s;
    for (;;) {
        if (threadIdx.x == 0) tile_s = atomicAdd(next, 1);
        __syncthreads();
        const int tile = tile_s;
        __syncthreads();
        if (tile >= total) break;
        const GroupFold P = pr[find_problem(first, np, tile)];
        const int local = tile - P.first;
        const int mp = local / P.ntx, cx = local - mp * P.ntx;
        const int m = mp >> 1, par = mp & 1;
        if (P.nj == 2) legfold_tile<NW, MTW, 2>(P.g, P.fa, P.RTmax, m, par, cx * 16, smd);
        else legfold_tile<NW, MTW, 4>(P.g, P.fa, P.RTmax, m, par, cx * 32, smd);
        __syncthreads();
    }
}

}  // namespace

// the grouped kernels also hold a static work-item slot in shared memory
constexpr int kGroupedSmemMax = 227 * 1024 - 128;

int group_b2p_prepare(GroupB2P& p) {
    p.SA = pad16_8(((p.g.NRH + 7) / 8) * 8);
    const int ct = 8 * p.nj;
    p.ntx = (2 * p.g.NXCHOPDIM + ct - 1) / ct;
    return p.ntx * p.g.NTCHOPDIM;
}
size_t group_b2p_smem(const GroupB2P& p) { return NST_B2P * (size_t)KCB * (p.SA + SBS) * sizeof(double); }

int group_fold_prepare(GroupFold& p) {
    p.RTmax = ((p.g.NRCHOPDIM + 1) / 2 + 7) / 8;
    const int ct = 8 * p.nj;
    p.ntx = (2 * p.g.NXCHOPDIM + ct - 1) / ct;
    return p.ntx * 2 * p.g.NTCHOPDIM;
}
size_t group_fold_smem(const GroupFold& p) {
    const int nch = (p.g.NRH + KC2 - 1) / KC2;
    return (NST_FOLD * ((size_t)p.RTmax * 8 * SA2 + (size_t)2 * KC2 * SX2) + (size_t)KC2 * SX2 + (size_t)nch * KC2) *
           sizeof(double);
}
bool group_supported(const DevGrid& g) { return dmma_supported(g) && (g.NRH + 7) / 8 <= 12 && ((g.NRCHOPDIM + 1) / 2 + 7) / 8 <= 12; }

void k_grouped_b2p(const GroupB2P* d, const int* first, int np, int total, size_t smem, int ctas, int* next,
                   cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(grouped_b2p_kernel<4, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupedSmemMax);
        attr = true;
    }
    cudaMemsetAsync(next, 0, sizeof(int), s);
    grouped_b2p_kernel<4, 3><<<ctas, 128, smem, s>>>(d, first, np, total, next);
    count_launch();
}

void k_grouped_fold(const GroupFold* d, const int* first, int np, int total, size_t smem, int ctas, int* next,
                    cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(grouped_fold_kernel<4, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupedSmemMax);
        attr = true;
    }
    cudaMemsetAsync(next, 0, sizeof(int), s);
    grouped_fold_kernel<4, 3><<<ctas, 128, smem, s>>>(d, first, np, total, next);
    count_launch();
}

}  // namespace mlegs
