// RTRAN(A, +1) on the FP64 tensor path with bulk-copy staging and a
// warp-specialised pipeline (FP64 contexts).
//
// Same contract as b2p_dmma_kernel (gemm_dmma.cu, mod_fft.f90:1264-1336): per
// m and parity p of n,
//     C_p(i, c) = sum_t PF(i, 2t+p) A(2t+p, c),  B(i) = C_0 + C_1,
//     B(NR-1-i) = C_0 - C_1,  plus the (m, k) = (0, 0) log term.
// One CTA computes a 32-column tile of one m for all NRH output rows:
//   warps 0..3   consumers: m8n8k4 FP64 MMAs over their MTW m-tiles x four
//                n-tiles, both parities' accumulators in registers;
//   warp 4       producer: per 16-row K chunk, one 1-D bulk copy
//                (cp.async.bulk) per PF row and per field row into a ring of
//                NST shared-memory stages, completing on the stage's
//                mbarrier.
// The consumers' fragment loads are shared-memory loads at fixed offsets from
// a per-thread base (row strides = 8 mod 16 doubles: the minimum two
// wavefronts per load); no address arithmetic runs per MMA.  K rows past the
// parity's extent are not copied; their B fragments are zeroed in registers
// (the stale A rows there are finite: the ring starts zeroed).  Every
// mbarrier wait is bounded (about a second); on a timeout the CTA raises the
// module's error word and its roles stop, the producer first waiting (again
// bounded) for the copies it issued.
#include "mlegs_internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>

namespace mlegs {

namespace {

constexpr uint64_t WAIT_CYCLES = 2000000000ull;  // about one second of SM cycles
constexpr int BK = 16;                           // K rows per chunk
constexpr int BCT = 32;                          // output columns per CTA
constexpr int BSB = BCT + 8;                     // field row stride (doubles), = 8 mod 16
constexpr int BNW = 4;                           // consumer warps

__device__ int g_bulk_err = 0;

__device__ __forceinline__ uint32_t sa_of(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa_of(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa_of(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa_of(bar)) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(sa_of(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of `parity`; false after WAIT_CYCLES.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
    if (bar_try(bar, parity)) return true;
    const uint64_t t0 = (uint64_t)clock64();
    while (!bar_try(bar, parity))
        if ((uint64_t)clock64() - t0 > WAIT_CYCLES) return false;
    return true;
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(sa_of(dst)),
        "l"(src), "r"(bytes), "r"(sa_of(bar))
        : "memory");
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// 16 K rows of one parity: four k-steps of MTW x 4 MMAs.  As/Bs point at the
// thread's fragment base (row q, column gq, plus the warp's first m-tile);
// rows with k >= kvalid read as zero in B.
template <int MTW, int SA, bool MASK>
__device__ __forceinline__ void chunk_mma(double (&acc)[MTW][4][2], const double* __restrict__ As,
                                          const double* __restrict__ Bs, int kvalid, int q) {
#pragma unroll
    for (int s4 = 0; s4 < BK / 4; ++s4) {
        if (MASK && 4 * s4 >= kvalid) break;  // warp-uniform: no row of this k-step is valid
        double bf[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = Bs[s4 * 4 * BSB + j * 8];
        if (MASK) {
            if (4 * s4 + q >= kvalid) {
#pragma unroll
                for (int j = 0; j < 4; ++j) bf[j] = 0.0;
            }
        }
#pragma unroll
        for (int i = 0; i < MTW; ++i) {
            const double af = As[s4 * 4 * SA + i * BNW * 8];
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma(acc[i][j], af, bf[j]);
        }
    }
}

// Per-stage work description the producer hands to the consumers with the
// stage's data (written before the stage's arrive, read after its wait).
struct StageInfo {
    int tile;    // tile index (m * ntx + column tile), -1: no more work
    int p;       // parity of the K rows
    int kvalid;  // valid K rows in this chunk (0: a tile without K rows)
    int last;    // 1: the tile's last chunk (the consumers write the tile out)
};

template <int MTW, int NST>
__global__ void __launch_bounds__((BNW + 1) * 32, MTW <= 3 ? 3 : 2) b2p_bulk_kernel(DevGrid g, const double* __restrict__ A,
                                                                               double* __restrict__ out,
                                                                               const double* ln, int pad) {
    constexpr int SA = BNW * MTW * 8 + (((BNW * MTW) & 1) ? 0 : 8);  // PF row stride, = 8 mod 16
    constexpr int STG = BK * SA + BK * BSB;                          // doubles per stage
    extern __shared__ __align__(128) double smd[];
    uint64_t* full = (uint64_t*)(smd + NST * STG);
    uint64_t* empty = full + NST;
    __shared__ StageInfo info[NST];
    __shared__ int abort_f;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntx = (ncol + BCT - 1) / BCT, ntiles = ntx * g.NTCHOPDIM;
    // zeroed ring (rows that are never copied stay finite), barriers
    for (int e = tid; e < NST * STG; e += blockDim.x) smd[e] = 0.0;
    if (tid == 0) {
        abort_f = 0;
        for (int st = 0; st < NST; ++st) {
            bar_init(full + st, 1);
            bar_init(empty + st, BNW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    if (warp == BNW) {
        // ---------------------------------------------------------------- producer
        // The CTA's tiles are blockIdx.x, + gridDim.x, ... (m ascending: the
        // largest K first); their chunks form one stream through the ring, so
        // the next tile's rows arrive while the current one is finishing.
        const int ne = g.NRCHOPDIM + 1;
        const uint32_t abytes = (uint32_t)g.NRH * 8u;
        int seq = 0;  // chunks handed over so far
        bool ok = true;
        auto acquire = [&](int st) -> bool {  // the stage's previous contents consumed
            if (seq < NST) return true;
            bool w = true;
            if (lane == 0) w = bar_wait(empty + st, (uint32_t)((seq / NST - 1) & 1));
            w = __shfl_sync(0xffffffffu, w ? 1 : 0, 0) != 0;
            return w && !*(volatile int*)&abort_f;
        };
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const int m = tile / ntx, c0 = (tile - m * ntx) * BCT;
            int nn = g.NRCHOP + pad - m;
            if (nn < 0) nn = 0;
            const int kp0 = (nn + 1) / 2, kp1 = nn / 2;
            const int nc0 = (kp0 + BK - 1) / BK, nc1 = (kp1 + BK - 1) / BK;
            const int total = max(1, nc0 + nc1);  // a tile without K rows still hands over one empty chunk
            const double* pf = g.pf + (size_t)m * ne * g.NRH;
            const double* a = A + (size_t)m * g.NRCHOPDIM * ncol;
            const uint32_t bbytes = (uint32_t)min(BCT, ncol - c0) * 8u;
            for (int c = 0; c < total; ++c) {
                const int st = seq % NST;
                if (!acquire(st)) {
                    ok = false;
                    break;
                }
                int p = 0, t0 = 0, rows = 0;
                if (nc0 + nc1 > 0) {
                    p = c < nc0 ? 0 : 1;
                    t0 = (c - (p ? nc0 : 0)) * BK;
                    rows = min(BK, (p ? kp1 : kp0) - t0);
                }
                double* As = smd + (size_t)st * STG;
                double* Bs = As + BK * SA;
                if (lane == 0) {
                    info[st] = StageInfo{tile, p, rows, c == total - 1 ? 1 : 0};
                    bar_expect_tx(full + st, (uint32_t)rows * (abytes + bbytes));
                }
                __syncwarp();
                if (lane < rows) {
                    const int n = 2 * (t0 + lane) + p;
                    bulk_copy(As + lane * SA, pf + (size_t)n * g.NRH, abytes, full + st);
                } else if (lane >= 16 && lane - 16 < rows) {
                    const int n = 2 * (t0 + lane - 16) + p;
                    bulk_copy(Bs + (lane - 16) * BSB, a + (size_t)n * ncol + c0, bbytes, full + st);
                }
                ++seq;
            }
        }
        if (ok) {  // end of work
            const int st = seq % NST;
            if (acquire(st)) {
                if (lane == 0) {
                    info[st] = StageInfo{-1, 0, 0, 0};
                    bar_expect_tx(full + st, 0u);
                }
                ++seq;
            } else {
                ok = false;
            }
        }
        if (!ok && lane == 0) {
            // drain: the copies of stages handed over and possibly unconsumed land
            // before the CTA's shared memory is released (bounded waits)
            for (int c = max(0, seq - NST); c < seq; ++c) bar_wait(full + (c % NST), (uint32_t)((c / NST) & 1));
            atomicExch(&g_bulk_err, 1);
        }
        return;
    }

    // -------------------------------------------------------------------- consumers
    const int gq = lane >> 2, q = lane & 3;
    double acc0[MTW][4][2], acc1[MTW][4][2];
#pragma unroll
    for (int i = 0; i < MTW; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc0[i][j][0] = acc0[i][j][1] = acc1[i][j][0] = acc1[i][j][1] = 0.0;
    const int fa = q * SA + warp * 8 + gq;  // A fragment base within a stage
    const int fb = q * BSB + gq;            // B fragment base
    for (int seq = 0;; ++seq) {
        const int st = seq % NST;
        if (!bar_wait(full + st, (uint32_t)((seq / NST) & 1))) {
            if (lane == 0) {
                abort_f = 1;
                atomicExch(&g_bulk_err, 1);
            }
            return;
        }
        const StageInfo inf = info[st];
        if (inf.tile < 0) return;
        const double* As = smd + (size_t)st * STG;
        const double* Bs = As + BK * SA;
        if (inf.kvalid >= BK) {
            if (inf.p == 0) chunk_mma<MTW, SA, false>(acc0, As + fa, Bs + fb, inf.kvalid, q);
            else chunk_mma<MTW, SA, false>(acc1, As + fa, Bs + fb, inf.kvalid, q);
        } else if (inf.kvalid > 0) {
            if (inf.p == 0) chunk_mma<MTW, SA, true>(acc0, As + fa, Bs + fb, inf.kvalid, q);
            else chunk_mma<MTW, SA, true>(acc1, As + fa, Bs + fb, inf.kvalid, q);
        }
        __syncwarp();
        if (lane == 0) bar_arrive(empty + st);
        if (!inf.last) continue;
        // the tile's butterfly + log term, then fresh accumulators
        const int m = inf.tile / ntx, c0 = (inf.tile - m * ntx) * BCT;
        const double lnv = (m == 0 && ln) ? *ln : 0.0;
        double* o = out + (size_t)m * g.NR * ncol;
#pragma unroll
        for (int i = 0; i < MTW; ++i) {
            const int row = (warp + BNW * i) * 8 + gq;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = c0 + j * 8 + 2 * q;
                if (row < g.NRH && c < ncol) {
                    const int rh = g.NR - 1 - row;
                    double2 lo = make_double2(acc0[i][j][0] + acc1[i][j][0], acc0[i][j][1] + acc1[i][j][1]);
                    double2 hi = make_double2(acc0[i][j][0] - acc1[i][j][0], acc0[i][j][1] - acc1[i][j][1]);
                    if (c == 0 && lnv != 0.0) {
                        lo.x += lnv * g.lnx[row];
                        hi.x += lnv * g.lnx[rh];
                    }
                    *(double2*)(o + (size_t)row * ncol + c) = lo;
                    *(double2*)(o + (size_t)rh * ncol + c) = hi;
                }
                acc0[i][j][0] = acc0[i][j][1] = acc1[i][j][0] = acc1[i][j][1] = 0.0;
            }
        }
    }
}

// Fold GEMMs (RTRAN(-1), mod_fft.f90:1189-1261, and PROJECT's EOMUL/OEMUL
// products, mod_legops.f90:2497-2535, 2548-2648) with the same pipeline:
//   out(n, c) (+)= sum_seg sum_{i < NRH} W_seg(n, i) s_seg(c) F_seg(i, c),
//   F = x(i) +/- x(NR-1-i), the sign by output-row parity xor the segment's mode.
// One CTA tile = (m, output parity pr, 64 columns): each of four consumer
// warps folds its own 16 columns once per chunk and multiplies them by every
// valid output-row tile (8 rows) of the weights, so the fold work is not
// repeated across warps.  A K chunk (16 rows i of one
// segment) is one bulk copy of the segment's weight block and two tensor-map
// (TMA) boxes of the input field: rows i0 .. i0+15 and NR-16-i0 .. NR-1-i0,
// 72 columns each (the tile's 64 and 8 more, so that the box rows land at a
// stride of 8 mod 16 doubles; columns past the field read as zero).  The
// weights come from a table laid out per (m, pr, chunk) as [row r][20]
// (n = 2r + pr, i = 16 chunk + kk for kk < 16, zero padded: row stride = 4 mod
// 16 doubles, the minimum two wavefronts per fragment load), so a chunk's
// weights are one contiguous copy; RTRAN(-1)'s table has the Gauss weights
// w_i folded in.  The fold and the complex column factor s_seg are applied to
// each B fragment as it is read: -1, m k and the fold sign are real factors,
// -i m and i k read the partner column (re <-> im) with a per-lane sign.
struct FoldBulkArgs {
    const double* wc[5];  // chunked weight tables
    int mode[5];          // 0: EO fold, 1: OE fold
    int scale[5];         // 0 none, 1 -v, 2 -i m v, 3 i k v, 4 m k v
    int nseg, split;      // segments [0, split) -> out0, [split, nseg) -> out1
    double* out0;
    double* out1;
    int wt_rows, pad, accumulate, RB;  // RB: rows per (m, pr) block of the tables
};
// The segments' input fields as 2-D tensor maps: columns (2 NXCHOPDIM) x rows (NTCHOPDIM NR).
struct alignas(64) FoldMaps {
    CUtensorMap x[5];
};
constexpr int WCS = 20;           // chunked weight row stride (doubles), = 4 mod 16
constexpr int FNW = 4;            // consumer warps, 16 columns each
constexpr int FCT = 16 * FNW;     // columns per tile
constexpr int XW = FCT + 8;       // field box width (doubles), = 8 mod 16

template <class T>
__device__ __forceinline__ T sel5(const T (&a)[5], int i) {
    T v = a[0];
#pragma unroll
    for (int j = 1; j < 5; ++j)
        if (i == j) v = a[j];
    return v;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(sa_of(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(sa_of(bar))
        : "memory");
}

struct FoldInfo {
    int tile;    // (m, pr, column tile) index, -1: no more work
    int gc;      // chunk index within the tile (segment * nch + chunk)
    int kvalid;  // valid K rows in the chunk
    int last;    // 1: the tile's last chunk
};

// Xt / Xb: the thread's B base in the top rows (row q) and bottom rows (row
// 31 - q; row 31 - k holds x(NR-1-i0-k)); As: the A base (row gq, column q);
// rtv: valid output-row tiles (warp-uniform).
template <int MT, bool MASK>
__device__ __forceinline__ void fold_chunk_mma(double (&acc)[MT][2][2], const double* __restrict__ As,
                                               const double* __restrict__ Xt, const double* __restrict__ Xb,
                                               const double (&fac)[2], const double (&fsg)[2], int kvalid, int q,
                                               int rtv) {
#pragma unroll
    for (int s4 = 0; s4 < BK / 4; ++s4) {
        if (MASK && 4 * s4 >= kvalid) break;
        double bf[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double top = Xt[s4 * 4 * XW + j * 8], bot = Xb[-s4 * 4 * XW + j * 8];
            bf[j] = fma(fsg[j], bot, fac[j] * top);
        }
        if (MASK) {
            if (4 * s4 + q >= kvalid) bf[0] = bf[1] = 0.0;
        }
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            if (i < rtv) {
                const double af = As[i * 8 * WCS + s4 * 4];
                dmma(acc[i][0], af, bf[0]);
                dmma(acc[i][1], af, bf[1]);
            }
        }
    }
}

template <int MT, int NST>
__global__ void __launch_bounds__((FNW + 1) * 32, 3) fold_bulk_kernel(DevGrid g, FoldBulkArgs fa,
                                                                      const __grid_constant__ FoldMaps tm) {
    extern __shared__ __align__(128) double smd[];
    const int STG = fa.RB * WCS + 2 * BK * XW;  // doubles per stage (a multiple of 16)
    uint64_t* full = (uint64_t*)(smd + NST * STG);
    uint64_t* empty = full + NST;
    __shared__ FoldInfo info[NST];
    __shared__ int abort_f;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntx = (ncol + FCT - 1) / FCT, ntiles = ntx * 2 * g.NTCHOPDIM;
    const int nch = (g.NRH + BK - 1) / BK, nchunks = fa.nseg * nch;
    for (int e = tid; e < NST * STG; e += blockDim.x) smd[e] = 0.0;
    if (tid == 0) {
        abort_f = 0;
        for (int st = 0; st < NST; ++st) {
            bar_init(full + st, 1);
            bar_init(empty + st, FNW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    // per tile: m, parity, first column, valid row tiles (rows n < min(NRCHOPS(m), wt_rows))
    auto decode = [&](int tile, int& m, int& pr, int& c0, int& nn, int& RTv) {
        m = tile / (2 * ntx);
        const int rem = tile - m * 2 * ntx;
        pr = rem / ntx;
        c0 = (rem - pr * ntx) * FCT;
        nn = g.NRCHOP + fa.pad - m;
        if (nn < 0) nn = 0;
        const int nw = min(nn, fa.wt_rows);
        const int rows = (g.NRCHOPDIM - pr + 1) / 2;
        const int rv = min(rows, max(0, (nw - pr + 1) / 2));
        RTv = (rv + 7) / 8;
    };

    if (warp == FNW) {
        // ---------------------------------------------------------------- producer
        int seq = 0;
        bool ok = true;
        auto acquire = [&](int st) -> bool {
            if (seq < NST) return true;
            bool w = true;
            if (lane == 0) w = bar_wait(empty + st, (uint32_t)((seq / NST - 1) & 1));
            w = __shfl_sync(0xffffffffu, w ? 1 : 0, 0) != 0;
            return w && !*(volatile int*)&abort_f;
        };
        constexpr uint32_t xbytes = (uint32_t)(BK * XW * 8);
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            int m, pr, c0, nn, RTv;
            decode(tile, m, pr, c0, nn, RTv);
            const uint32_t abytes = (uint32_t)RTv * 8u * WCS * 8u;
            for (int gc = 0; gc < nchunks; ++gc) {
                const int st = seq % NST;
                if (!acquire(st)) {
                    ok = false;
                    break;
                }
                const int sg = gc / nch, ch = gc - sg * nch, i0 = ch * BK;
                const int kv = min(BK, g.NRH - i0);
                double* As = smd + (size_t)st * STG;
                double* Xs = As + fa.RB * WCS;
                if (lane == 0) {
                    info[st] = FoldInfo{tile, gc, kv, gc == nchunks - 1 ? 1 : 0};
                    bar_expect_tx(full + st, abytes + 2u * xbytes);
                    if (abytes) {
                        const double* wc = sel5(fa.wc, sg) + (((size_t)m * 2 + pr) * nch + ch) * fa.RB * WCS;
                        bulk_copy(As, wc, abytes, full + st);
                    }
                    const CUtensorMap* map = &tm.x[0];
                    for (int j = 1; j < 5; ++j)
                        if (sg == j) map = &tm.x[j];
                    tma_load_2d(Xs, map, c0, m * g.NR + i0, full + st);
                    tma_load_2d(Xs + BK * XW, map, c0, m * g.NR + g.NR - BK - i0, full + st);
                }
                __syncwarp();
                ++seq;
            }
        }
        if (ok) {
            const int st = seq % NST;
            if (acquire(st)) {
                if (lane == 0) {
                    info[st] = FoldInfo{-1, 0, 0, 0};
                    bar_expect_tx(full + st, 0u);
                }
                ++seq;
            } else {
                ok = false;
            }
        }
        if (!ok && lane == 0) {
            for (int c = max(0, seq - NST); c < seq; ++c) bar_wait(full + (c % NST), (uint32_t)((c / NST) & 1));
            atomicExch(&g_bulk_err, 1);
        }
        return;
    }

    // -------------------------------------------------------------------- consumers
    const int gq = lane >> 2, q = lane & 3;
    double acc[MT][2][2];
#pragma unroll
    for (int i = 0; i < MT; ++i) acc[i][0][0] = acc[i][0][1] = acc[i][1][0] = acc[i][1][1] = 0.0;
    const int fa_ofs = gq * WCS + q;  // A fragment base within a stage
    double fac[2] = {1.0, 1.0}, fsg[2] = {1.0, 1.0};
    int gsel = gq;
    int cur_tile = -2, cur_sg = -1;
    int m = 0, pr = 0, c0 = 0, nn = 0, RTv = 0;
    auto epilogue = [&](double* out) {
        double* o = out + (size_t)m * g.NRCHOPDIM * ncol;
#pragma unroll
        for (int t = 0; t < MT; ++t) {
            const int n = 2 * (t * 8 + gq) + pr;
            const bool rok = n < g.NRCHOPDIM;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int c = c0 + warp * 16 + j * 8 + 2 * q;
                const double2 v = make_double2(acc[t][j][0], acc[t][j][1]);
                acc[t][j][0] = acc[t][j][1] = 0.0;
                if (!rok || c >= ncol) continue;
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
    for (int seq = 0;; ++seq) {
        const int st = seq % NST;
        if (!bar_wait(full + st, (uint32_t)((seq / NST) & 1))) {
            if (lane == 0) {
                abort_f = 1;
                atomicExch(&g_bulk_err, 1);
            }
            return;
        }
        const FoldInfo inf = info[st];
        if (inf.tile < 0) return;
        if (inf.tile != cur_tile) {
            cur_tile = inf.tile;
            cur_sg = -1;
            decode(inf.tile, m, pr, c0, nn, RTv);
        }
        const int sg = inf.gc / nch;
        if (sg != cur_sg) {  // the segment's fold sign, column factors and column selection
            cur_sg = sg;
            const int sc = sel5(fa.scale, sg);
            const double sgn = (pr ^ sel5(fa.mode, sg)) ? -1.0 : 1.0;
            const bool rot = sc == 2 || sc == 3;
            const double odd = (gq & 1) ? 1.0 : -1.0;  // lanes on imaginary columns
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int c = c0 + warp * 16 + j * 8 + gq;
                const double kv = c < ncol ? g.ak[c >> 1] : 0.0;
                double f = 1.0;
                switch (sc) {
                    case 1: f = -1.0; break;
                    case 2: f = -odd * (double)m; break;  // -i m v: re <- m im, im <- -m re
                    case 3: f = odd * kv; break;          // i k v: re <- -k im, im <- k re
                    case 4: f = (double)m * kv; break;
                    default: break;
                }
                fac[j] = f;
                fsg[j] = f * sgn;
            }
            gsel = rot ? (gq ^ 1) : gq;
        }
        const double* As = smd + (size_t)st * STG;
        const double* Xs = As + fa.RB * WCS;
        const double* Xt = Xs + q * XW + warp * 16 + gsel;
        const double* Xb = Xs + (2 * BK - 1 - q) * XW + warp * 16 + gsel;
        if (inf.kvalid >= BK) fold_chunk_mma<MT, false>(acc, As + fa_ofs, Xt, Xb, fac, fsg, inf.kvalid, q, RTv);
        else fold_chunk_mma<MT, true>(acc, As + fa_ofs, Xt, Xb, fac, fsg, inf.kvalid, q, RTv);
        __syncwarp();
        if (lane == 0) bar_arrive(empty + st);
        const int ch_last = (inf.gc % nch) == nch - 1;
        if (ch_last && sg == fa.split - 1) epilogue(fa.out0);
        else if (inf.last) epilogue(fa.out1);
    }
}

// Chunked weight table of a fold GEMM: Wc[m][pr][chunk][r][WCS] = W(n = 2r + pr,
// i = 16 chunk + kk) (times w_i when use_w), zero past NRH, wt_rows and kk >= 16.
__global__ void fold_table_kernel(DevGrid g, const double* __restrict__ W, int wt_rows, int use_w, int RB,
                                  double* __restrict__ Wc) {
    const int nch = (g.NRH + BK - 1) / BK;
    const size_t total = (size_t)g.NTCHOPDIM * 2 * nch * RB * WCS;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int kk = (int)(t % WCS);
    const int r = (int)((t / WCS) % RB);
    const int ch = (int)((t / ((size_t)WCS * RB)) % nch);
    const int pr = (int)((t / ((size_t)WCS * RB * nch)) % 2);
    const int m = (int)(t / ((size_t)WCS * RB * nch * 2));
    const int n = 2 * r + pr, i = ch * BK + kk;
    double v = 0.0;
    if (kk < BK && n < wt_rows && i < g.NRH) {
        v = W[((size_t)m * wt_rows + n) * g.NRH + i];
        if (use_w) v *= g.w[i];
    }
    Wc[t] = v;
}

int bulk_sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

template <int MTW, int NST>
void launch_b2p_bulk_n(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, int per_sm,
                       cudaStream_t s) {
    constexpr int SA = BNW * MTW * 8 + (((BNW * MTW) & 1) ? 0 : 8);
    constexpr size_t smem = (size_t)NST * (BK * SA + BK * BSB) * sizeof(double) + 2 * NST * sizeof(uint64_t);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(b2p_bulk_kernel<MTW, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntiles = ((ncol + BCT - 1) / BCT) * g.NTCHOPDIM;
    const int grid = std::min(ntiles, bulk_sm_count() * per_sm);
    b2p_bulk_kernel<MTW, NST><<<grid, (BNW + 1) * 32, smem, s>>>(g, (const double*)a, (double*)b, ln, pad);
    count_launch();
}

// Three stages at three CTAs per SM (55 KB each at MTW = 3) leave room on every
// SM for a VERFFT(+1) CTA, which runs beside the GEMM on the other stream in
// TOFP; four stages filled the SM (545 vs 541 steps/s at 192x128x256).
template <int MTW>
void launch_b2p_bulk(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    launch_b2p_bulk_n<MTW, 3>(g, a, b, ln, pad, MTW <= 3 ? 3 : 2, s);
}

template <int MT>
void launch_fold_bulk(const DevGrid& g, const FoldBulkArgs& fa, const FoldMaps& tm, cudaStream_t s) {
    constexpr int NST = 2;
    const size_t smem = (size_t)NST * (fa.RB * WCS + 2 * BK * XW) * sizeof(double) + 2 * NST * sizeof(uint64_t);
    static size_t attr = 0;  // the opt-in size set so far (the kernel also has static shared memory)
    if (smem > attr) {
        if (cudaFuncSetAttribute(fold_bulk_kernel<MT, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) == cudaSuccess)
            attr = smem;
    }
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntiles = ((ncol + FCT - 1) / FCT) * 2 * g.NTCHOPDIM;
    const int grid = std::min(ntiles, bulk_sm_count() * 3);
    fold_bulk_kernel<MT, NST><<<grid, (FNW + 1) * 32, smem, s>>>(g, fa, tm);
    count_launch();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// A PFF field [m][r][2 NXCHOPDIM] as a 2-D map (columns, rows), box XW x 16, zero fill.
bool field_map(const DevGrid& g, const double* x, CUtensorMap* map) {
    auto enc = tmap_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)(2 * g.NXCHOPDIM), (cuuint64_t)g.NTCHOPDIM * g.NR};
    const cuuint64_t strides[1] = {(cuuint64_t)(2 * g.NXCHOPDIM) * 8};
    const cuuint32_t box[2] = {(cuuint32_t)XW, (cuuint32_t)BK};
    const cuuint32_t es[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)x, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Register-only ceiling of the FP64 tensor path: every warp issues DPK_ITER
// rounds of eight independent mma.sync.m8n8k4.f64 on register fragments (no
// memory traffic but one store per thread at the end), DPK_CTAS CTAs of eight
// warps per SM.  The GEMMs' tensor-pipe fractions are read against it.
constexpr int DPK_ITER = 4096, DPK_CTAS = 4;
__global__ void __launch_bounds__(256) dmma_peak_kernel(double* out, double seed) {
    double acc[8][2];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = 0.0;
    const double a = seed * (1 + (threadIdx.x & 3)), b = seed * (2 + (threadIdx.x >> 5));
    for (int it = 0; it < DPK_ITER; ++it) {
#pragma unroll
        for (int j = 0; j < 8; ++j) dmma(acc[j], a, b);
    }
    double v = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) v += acc[j][0] + acc[j][1];
    out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = v;
}

}  // namespace

// FLOPs of one k_dmma_peak launch: CTAs x warps x rounds x MMAs x (8 x 8 x 4 x 2)
double dmma_peak_flops() { return (double)bulk_sm_count() * DPK_CTAS * 8 * DPK_ITER * 8 * 512.0; }

// out: at least SMs x DPK_CTAS x 256 doubles
double k_dmma_peak(double* out, cudaStream_t s) {
    dmma_peak_kernel<<<bulk_sm_count() * DPK_CTAS, 256, 0, s>>>(out, 1e-3);
    count_launch();
    return dmma_peak_flops();
}

bool b2p_bulk_supported(const DevGrid& g) {
    const int RT = (g.NRH + 7) / 8;
    return (g.NRH % 2) == 0 && RT <= 4 * BNW;
}

void k_rtran_b2p_bulk(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s) {
    const int RT = (g.NRH + 7) / 8;
    switch ((RT + BNW - 1) / BNW) {
        case 1: launch_b2p_bulk<1>(g, a, b, ln, pad, s); break;
        case 2: launch_b2p_bulk<2>(g, a, b, ln, pad, s); break;
        case 3: launch_b2p_bulk<3>(g, a, b, ln, pad, s); break;
        default: launch_b2p_bulk<4>(g, a, b, ln, pad, s); break;
    }
}

int bulk_gemm_error(bool reset) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_bulk_err, sizeof(int)) != cudaSuccess) return -1;
    if (reset && v) {
        const int z = 0;
        cudaMemcpyToSymbol(g_bulk_err, &z, sizeof(int));
    }
    return v;
}

// ---------------------------------------------------------------- fold GEMMs
int fold_table_rows(const DevGrid& g, int wt_rows) { return ((wt_rows + 1) / 2 + 7) / 8 * 8; }

size_t fold_table_doubles(const DevGrid& g, int wt_rows) {
    const int nch = (g.NRH + BK - 1) / BK;
    return (size_t)g.NTCHOPDIM * 2 * nch * fold_table_rows(g, wt_rows) * WCS;
}

void k_fold_table(const DevGrid& g, const double* W, int wt_rows, int use_w, double* Wc, cudaStream_t s) {
    const size_t n = fold_table_doubles(g, wt_rows);
    fold_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, W, wt_rows, use_w, fold_table_rows(g, wt_rows),
                                                                   Wc);
    count_launch();
}

bool fold_bulk_supported(const DevGrid& g, int wt_rows) {
    const int RB = fold_table_rows(g, wt_rows);
    const size_t smem = (size_t)2 * (RB * WCS + 2 * BK * XW) * sizeof(double) + 32;
    // at most 12 output-row tiles (the accumulators stay in registers), two CTAs per SM
    // fit, a chunk's bottom box starts at row NR - 16 - i0 >= 0, and the tensor maps encode
    return RB <= 12 * 8 && smem <= 227 * 1024 / 2 - 1024 && g.NRH >= BK && tmap_encoder() != nullptr;
}

// out (+)= sum over segments; wc: chunked tables of k_fold_table (wt_rows rows).
void k_fold_bulk(const DevGrid& g, const double* const* wc, const double2* const* x, const int* mode,
                 const int* scale, int nseg, int split, double2* out0, double2* out1, int wt_rows, int pad,
                 int accumulate, cudaStream_t s) {
    FoldBulkArgs fa{};
    FoldMaps tm;
    memset(&tm, 0, sizeof(tm));
    for (int q = 0; q < 5; ++q) {
        const int src = q < nseg ? q : 0;
        fa.wc[q] = wc[src];
        fa.mode[q] = q < nseg ? mode[q] : 0;
        fa.scale[q] = q < nseg ? scale[q] : 0;
        if (q < nseg && !field_map(g, (const double*)x[q], &tm.x[q]))
            throw std::runtime_error("fold GEMM: cuTensorMapEncodeTiled failed");
    }
    for (int q = nseg; q < 5; ++q) tm.x[q] = tm.x[0];
    fa.nseg = nseg;
    fa.split = split;
    fa.out0 = (double*)out0;
    fa.out1 = (double*)(out1 ? out1 : out0);
    fa.wt_rows = wt_rows;
    fa.pad = pad;
    fa.accumulate = accumulate;
    fa.RB = fold_table_rows(g, wt_rows);
    const int RT = fa.RB / 8;  // output-row tiles of a block
    if (RT <= 2) launch_fold_bulk<2>(g, fa, tm, s);
    else if (RT <= 4) launch_fold_bulk<4>(g, fa, tm, s);
    else if (RT <= 6) launch_fold_bulk<6>(g, fa, tm, s);
    else if (RT <= 9) launch_fold_bulk<9>(g, fa, tm, s);
    else launch_fold_bulk<12>(g, fa, tm, s);
}

}  // namespace mlegs
