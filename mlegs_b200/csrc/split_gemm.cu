// Split-BF16 (Ozaki) Legendre GEMMs on the fifth-generation tensor cores.
//
// Two GEMM families of the path run here when a context is created with
// MLEGS_PREC_SPLIT:
//   RTRAN(A, +1)  (mod_fft.f90:1264-1336), per m and parity p of n:
//       C_p(i, c) = sum_t PF(i, 2t+p) A(2t+p, c),  B(i) = C_0 + C_1,  B(NR-1-i) = C_0 - C_1,
//       plus the (m, k) = (0, 0) log term;
//   fold GEMMs    RTRAN(A, -1) (mod_fft.f90:1189-1261) and the EOMUL/OEMUL
//       products of PROJECT (mod_legops.f90:2497-2535, 2548-2648):
//       out(n, c) (+)= s(m, k) sum_{i < NRH} Wt(n, i) F(i, c),
//       F = x(i) +/- x(NR-1-i) (times w_i for RTRAN(-1)); the fold of row n is
//       parity(n) xor mode.
//
// Slicing.  Each row of the weight operand (per m and parity) and each column
// of the field operand (per m) is scaled by a power of two into (-1, 1) and
// written as v = sum_q a_q 2^{-8(q+1)}, a_q integer, |a_0| <= 256,
// |a_q| <= 128 (q > 0); a_q is stored in BF16 pre-multiplied by 2^{-8q}, which
// is exact.  The products a_qa b_qb with qa + qb <= S-1 go to S FP32
// accumulators in tensor memory, one per level L = qa + qb.  For K <= 128
// every partial sum of levels 0..3 is a multiple of 2^{-8L} below 2^{24-8L},
// so those four are exact; levels 4 and 5 round near 2^-56 of the row x
// column scale.  The epilogue adds the levels in FP64 and applies the two
// power-of-two scales.
//
// Kernel (persistent, one CTA per SM, 288 threads):
//   warps 0-3  epilogue: TMEM lane = output row, tcgen05.ld, FP64 combine, stores;
//   warps 4-7  producers: stage the work item's FP64 field columns (32 wide,
//              all K rows) in shared memory with 16-byte cp.async copies one
//              item ahead, take the column maxima there, and split 16-row
//              chunks into a ring of shared-memory stages; in RTRAN(+1) mode
//              one of them also brings the matching weight-slice chunk (one
//              contiguous bulk copy of the L2-resident slice image) onto the
//              stage's mbarrier, in fold mode the weight chunks of one
//              (m, parity) stay resident across its column tiles;
//   warp 8     one thread issues tcgen05.mma (M=128, K=16, BF16 x BF16 -> F32):
//              per chunk and weight slice qa a single MMA against the field
//              slices 0..S-1-qa stacked along N, whose products land in the
//              consecutive level accumulators qa..S-1; commits free the ring
//              stage and, per tile, hand the accumulators to the epilogue
//              (double-buffered in tensor memory in fold mode).
// Shared-memory operands use the K-major no-swizzle canonical layout: core
// matrices of 8 rows x 16 bytes, LBO = 128 B between the two K halves of a
// K=16 step, SBO = 256 B between 8-row groups.  Every wait is bounded (about
// one second of SM cycles); on a timeout the kernel raises *err, lets every
// role drain, waits (bounded) for what it issued, frees its tensor memory and
// returns.
#include "mlegs_internal.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

namespace mlegs {

namespace {

constexpr uint64_t WAIT_NS = 2000000000ull;  // cycles

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// SM cycle counter; the wait limits below are in cycles (2e9 cycles is about
// one second at the B200's clocks).
__device__ __forceinline__ uint64_t gtimer() { return (uint64_t)clock64(); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `parity` to complete; false after WAIT_NS cycles.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    while (!mbar_try(bar, parity))
        if (gtimer() - t0 > WAIT_NS) return false;
    return true;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar))
        : "memory");
}

// 16-byte asynchronous global -> shared copy (zero fill when src_bytes = 0).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
// Arrive on `bar` once this thread's earlier cp.async copies have landed.
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: BF16 x BF16 -> F32, both operands K-major.
constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ int scale_exp(double mx) {
    if (!(mx > 0.0)) return 0;
    int e;
    frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1)
    return e < -990 ? -990 : e;  // keeps 2^{8-e} finite; such columns hold no significant value
}

// One slicing step on v (|v| < 256 on entry, an FP64 value): returns the BF16
// bits of rint(v) * 2^{-8q} and leaves the remainder (v - rint(v)) * 256 in v.
// Exact arithmetic without conversion instructions: adding 1.5 * 2^52 rounds
// to the nearest integer and leaves it in the low word of the sum; adding
// 1.5 * 2^23 to it as a float and subtracting again gives the FP32 value; a
// value with at most 8 significant bits has its BF16 bits in the FP32's upper half.
__device__ __forceinline__ uint32_t slice_step(double& v, float sc) {
    const double t = v + 6755399441055744.0;         // 1.5 * 2^52
    const double a = t - 6755399441055744.0;         // rint(v)
    v = (v - a) * 256.0;
    const int ai = __double2loint(t);                // rint(v) as an integer
    const float fa = __int_as_float(0x4B400000 + ai) - 12582912.0f;  // (float) ai, exact for |ai| < 2^22
    return __float_as_uint(fa * sc) >> 16;
}

// Slices of 8 values (already multiplied by 2^{8-e}, |x| < 256) -> S packed
// rows of 8 BF16 each; slice q holds a_q 2^{-8q}.
template <int S>
__device__ __forceinline__ void split8(double (&x)[8], uint4 (&out)[S]) {
    uint32_t w[S][4];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        double v = x[u];
        float sc = 1.0f;
#pragma unroll
        for (int q = 0; q < S; ++q) {
            const uint32_t b = slice_step(v, sc);
            sc *= 0.00390625f;
            if (u & 1) w[q][u >> 1] |= b << 16;
            else w[q][u >> 1] = b;
        }
    }
#pragma unroll
    for (int q = 0; q < S; ++q) out[q] = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
}

}  // namespace


// ---------------------------------------------------------------------------
namespace {

constexpr int NT2 = 32;     // output columns per tile (per slice: the MMA's N is a multiple)
constexpr int NTH2 = 288;   // 9 warps
constexpr int NPROD = 128;  // producer threads (warps 4-7)
constexpr uint32_t BSLICE = (NT2 / 8) * 256;  // one B slice of a chunk

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}

// Bounded wait of the pipeline roles (limit in SM cycles) that gives up at
// once when another role has aborted.  The drain waits after an abort use
// mbar_wait with the full WAIT_NS, so a short role limit (set by the host to
// exercise the error path) still lets every copy and MMA in flight land.
__device__ bool wait_ab(uint64_t* bar, uint32_t parity, volatile int* abort_f, uint64_t limit) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    while (!mbar_try(bar, parity)) {
        if (*abort_f) return false;
        if (gtimer() - t0 > limit) {
            *abort_f = 1;
            return false;
        }
    }
    return true;
}

// Same for 4 values -> S packed half rows (4 BF16 each).
template <int S>
__device__ __forceinline__ void split4(double (&x)[4], uint2 (&out)[S]) {
    uint32_t w[S][2];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        double v = x[u];
        float sc = 1.0f;
#pragma unroll
        for (int q = 0; q < S; ++q) {
            const uint32_t b = slice_step(v, sc);
            sc *= 0.00390625f;
            if (u & 1) w[q][u >> 1] |= b << 16;
            else w[q][u >> 1] = b;
        }
    }
#pragma unroll
    for (int q = 0; q < S; ++q) out[q] = make_uint2(w[q][0], w[q][1]);
}

}  // namespace

// Weight slice images, chunk-contiguous:
//   img[((mp * NCH + c) * S + q) * RG * 256 + rg * 256 + kc2 * 128 + row8 * 16]
// mp = m * 2 + parity, chunk c = 16 K values, rg = row / 8; eA[mp * 128 + row].
// MODE 0 (RTRAN +1): rows i < NRH, K index t with n = 2t + parity (table PF).
// MODE 1 (fold):     rows r with n = 2r + parity < wt_rows, K index i < NRH.
template <int S, int MODE>
__global__ void slice_image_kernel(DevGrid g, const double* W, int wt_rows, uint8_t* img, int* eA, int RG,
                                   int NCH) {
    const int m = blockIdx.x, p = blockIdx.y, row = threadIdx.x;
    if (row >= RG * 8) return;
    const int mp = m * 2 + p;
    double mx = 0.0;
    int kt = 0;
    const double* base = nullptr;
    bool ok;
    if (MODE == 0) {
        const int ne = g.NRCHOPDIM + 1;
        kt = (ne - p + 1) / 2;
        base = W + (size_t)m * ne * g.NRH;
        ok = row < g.NRH;
        if (ok)
            for (int t = 0; t < kt; ++t) mx = fmax(mx, fabs(base[(size_t)(2 * t + p) * g.NRH + row]));
    } else {
        const int n = 2 * row + p;
        kt = g.NRH;
        ok = n < wt_rows;
        base = W + ((size_t)m * wt_rows + (ok ? n : 0)) * g.NRH;
        if (ok)
            for (int i = 0; i < g.NRH; ++i) mx = fmax(mx, fabs(base[i]));
    }
    const int e = scale_exp(mx);
    eA[mp * 128 + row] = e;
    const double sc = ldexp(1.0, 8 - e);
    for (int c = 0; c < NCH; ++c)
        for (int kc2 = 0; kc2 < 2; ++kc2) {
            double x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int t = 16 * c + 8 * kc2 + u;
                double v = 0.0;
                if (ok && t < kt) v = (MODE == 0) ? base[(size_t)(2 * t + p) * g.NRH + row] : base[t];
                x[u] = v * sc;
            }
            uint4 o[S];
            split8<S>(x, o);
            uint8_t* dst = img + ((size_t)(mp * NCH + c) * S) * RG * 256 + (row >> 3) * 256 + kc2 * 128 + (row & 7) * 16;
#pragma unroll
            for (int q = 0; q < S; ++q) *(uint4*)(dst + (size_t)q * RG * 256) = o[q];
        }
}

__device__ __forceinline__ void bar_producers() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Collective OR over the 128 producer threads (named barrier 1).
// Exact 2^e for -1022 <= e <= 1023.
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

__device__ __forceinline__ bool bar_producers_or(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

struct SplitArgs {
    const uint8_t* img;
    const int* eA;
    const double* in;
    double* out;
    const double* ln;  // MODE 0: A%LN of the input (may be null)
    int* err;
    unsigned long long wlim;  // role wait limit in SM cycles
    int pad, RG, NCH, trows;
    int mode, scale, accumulate, use_w;  // MODE 1
};

// One work item = (m[, parity of n], 48-column tile).  Per item the producers
// stage the item's FP64 field columns in shared memory (one bulk copy per
// row, double-buffered one item ahead), take the column maxima there, and
// split 16-row chunks into the ring.
// STREAM: the weight chunks come with each ring stage by one bulk copy (MODE 0
// always; MODE 1 when one (m, parity)'s chunks do not fit in shared memory
// beside the staged field tile, e.g. NR = 256) instead of staying resident.
template <int S, int MODE, int NS, bool STREAM>
__global__ void __launch_bounds__(NTH2, 1) split_gemm_kernel(DevGrid g, SplitArgs P) {
    constexpr int NL = S;  // one accumulator per level qa + qb
    constexpr uint32_t TCOLS = 512;
    constexpr int NBUF = (MODE == 0) ? 1 : 2;  // accumulator sets in tensor memory (MODE 1: 2 x 240 columns)
    constexpr uint32_t TROWB = NT2 * 8;  // bytes of one staged field row
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntiles = (ncol + NT2 - 1) / NT2;
    const int nitems = (MODE == 0 ? 1 : 2) * g.NTCHOPDIM * ntiles;
    // MODE 1: a contiguous item range per CTA, so consecutive items share (m,
    // parity) and its resident weight chunks; MODE 0: items dealt round-robin.
    const int per = (nitems + gridDim.x - 1) / gridDim.x;
    const int ib = (MODE == 1) ? blockIdx.x * per : blockIdx.x;
    const int ie = (MODE == 1) ? min(nitems, ib + per) : nitems;
    const int istep = (MODE == 1) ? 1 : gridDim.x;

    // MODE 0 streams one weight chunk per ring stage (SA bytes incl. the tail
    // rows up to 128); MODE 1 keeps all NCH chunks of one (m, parity) resident.
    const uint32_t SA = (uint32_t)(S * P.RG + 16 - P.RG) * 256;
    const uint32_t SB = (uint32_t)S * BSLICE;
    const uint32_t CB = (uint32_t)S * P.RG * 256;  // one chunk image
    const uint32_t TB = (uint32_t)P.trows * TROWB;  // one staged field tile
    uint8_t* tile_s = sm;                           // [2][trows][32] doubles
    uint8_t* stA = sm + 2 * TB;
    const uint32_t A_bytes = STREAM ? NS * SA : (uint32_t)P.NCH * CB + (uint32_t)(16 - P.RG) * 256;
    uint8_t* stB = stA + A_bytes;
    int* ebs = (int*)(stB + NS * SB);               // [2][32] column exponents
    double* cmax = (double*)(ebs + 2 * NT2);        // [4][32]
    double* wsm = cmax + 4 * NT2;                   // [128] Gauss weights
    uint64_t* full = (uint64_t*)(wsm + 128);
    uint64_t* empty = full + NS;
    uint64_t* tfull = empty + NS;     // [2]
    uint64_t* tempty = tfull + 2;     // [2]
    uint64_t* done = tempty + 2;
    uint64_t* a_full = done + 1;       // MODE 1: resident weight chunks landed
    uint64_t* a_free = a_full + 1;     // MODE 1: MMAs reading them completed
    uint64_t* tile_full = a_free + 1;  // [2]
    uint64_t* eb_ready = tile_full + 2;  // [2]
    uint64_t* eb_free = eb_ready + 2;    // [2]
    uint32_t* tslot = (uint32_t*)(eb_free + 2);
    volatile int* abort_f = (volatile int*)(tslot + 1);

    if (warp == 0) tmem_alloc(tslot, TCOLS);
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], STREAM ? NPROD + 1 : NPROD);
            mbar_init(&empty[s], 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&tfull[q], 1);
            mbar_init(&tempty[q], 128);
        }
        mbar_init(done, 1);
        mbar_init(a_full, 1);
        mbar_init(a_free, 1);
        for (int q = 0; q < 2; ++q) {
            mbar_init(&tile_full[q], NPROD);
            mbar_init(&eb_ready[q], NPROD);
            mbar_init(&eb_free[q], 128);
        }
        *abort_f = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < g.NRH; i += NTH2) wsm[i] = g.w[i];
    __syncthreads();
    tc_after();
    const uint32_t tbase = *tslot;

    auto item_info = [&](int item, int& m, int& pr, int& tile, int& nn, int& n0, int& n1) {
        tile = item % ntiles;
        const int mp = item / ntiles;
        m = (MODE == 0) ? mp : mp / 2;
        pr = (MODE == 0) ? 0 : mp % 2;
        nn = g.NRCHOP + P.pad - m;
        if (nn < 0) nn = 0;
        if (MODE == 0) {
            n0 = ((nn + 1) / 2 + 15) / 16;
            n1 = (nn / 2 + 15) / 16;
        } else {
            n0 = (pr < nn) ? P.NCH : 0;
            n1 = 0;
        }
    };

    if (warp >= 4 && warp < 8) {
        // ------------------------------------------------------------ producers
        const int pt = tid - 128, j = pt % NT2, h = pt / NT2;  // h: quarter of the 16 K rows
        // Stage the field columns of item `it` (local index k) into tile buffer k & 1:
        // 16-byte cp.async copies by all producers (columns past the last are
        // zero-filled), completing on tile_full[k & 1].
        auto issue_tile = [&](int it, int k) {
            int m, pr, tile, nn, n0, n1;
            item_info(it, m, pr, tile, nn, n0, n1);
            const int rows = (MODE == 0) ? nn : (n0 > 0 ? g.NR : 0);
            const int c0 = tile * NT2;
            const double* base = P.in + (size_t)m * P.trows * ncol + c0;
            uint8_t* dst = tile_s + (k & 1) * TB;
            for (int idx = pt; idx < rows * (NT2 / 2); idx += NPROD) {
                const int r = idx / (NT2 / 2), q = idx % (NT2 / 2);
                const bool ok = c0 + 2 * q < ncol;
                cp_async16(dst + r * TROWB + q * 16, ok ? (const void*)(base + (size_t)r * ncol + 2 * q) : (const void*)base,
                           ok ? 16u : 0u);
            }
            cp_async_arrive(&tile_full[k & 1]);
        };
        uint32_t gch = 0, issued = 0;
        int k = 0;
        int cur_mp = -1;
        uint32_t a_loads = 0;
        if (ib < ie) issue_tile(ib, 0);
        for (int item = ib; item < ie; item += istep, ++k) {
            // all producers are done with item k-1 (its tile buffer is reused below)
            if (bar_producers_or(*abort_f != 0)) break;
            const bool ab = *abort_f != 0;
            int m, pr, tile, nn, n0, n1;
            item_info(item, m, pr, tile, nn, n0, n1);
            if (item + istep < ie) issue_tile(item + istep, k + 1);
            if (MODE == 1 && !STREAM && m * 2 + pr != cur_mp) {
                // bring the weight chunks of the new (m, parity) once the MMAs on the old ones are done
                if (warp == 4) {
                    if (lane == 0 && !ab) {
                        if (a_loads > 0) wait_ab(a_free, (a_loads - 1) & 1, abort_f, P.wlim);
                        mbar_expect_tx(a_full, (uint32_t)P.NCH * CB);
                        const uint8_t* src = P.img + (size_t)((m * 2 + pr) * P.NCH) * CB;
                        for (int c = 0; c < P.NCH; ++c) bulk_g2s(stA + c * CB, src + (size_t)c * CB, CB, a_full);
                    }
                    __syncwarp();
                }
                cur_mp = m * 2 + pr;
                ++a_loads;
            }
            const double* T = (const double*)(tile_s + (k & 1) * TB);
            if (!ab) wait_ab(&tile_full[k & 1], (k >> 1) & 1, abort_f, P.wlim);
            if (k >= 2 && !*abort_f) wait_ab(&eb_free[k & 1], ((k >> 1) - 1) & 1, abort_f, P.wlim);
            const int col = tile * NT2 + j;
            const bool cok = col < ncol;
            const int fp = pr ^ P.mode;
            // column maxima from the staged tile
            double mx = 0.0;
            if (cok) {
                double m1 = 0.0;
                if (MODE == 0) {
                    int n = h;
                    for (; n + 4 < nn; n += 8) {
                        mx = fmax(mx, fabs(T[n * NT2 + j]));
                        m1 = fmax(m1, fabs(T[(n + 4) * NT2 + j]));
                    }
                    for (; n < nn; n += 4) mx = fmax(mx, fabs(T[n * NT2 + j]));
                } else if (n0 > 0) {
                    const double sgn = fp ? -1.0 : 1.0;
                    int i = h;
                    for (; i + 4 < g.NRH; i += 8) {
                        const double w0 = P.use_w ? wsm[i] : 1.0, w1 = P.use_w ? wsm[i + 4] : 1.0;
                        mx = fmax(mx, fabs((T[i * NT2 + j] + sgn * T[(g.NR - 1 - i) * NT2 + j]) * w0));
                        m1 = fmax(m1, fabs((T[(i + 4) * NT2 + j] + sgn * T[(g.NR - 5 - i) * NT2 + j]) * w1));
                    }
                    for (; i < g.NRH; i += 4) {
                        const double w0 = P.use_w ? wsm[i] : 1.0;
                        mx = fmax(mx, fabs((T[i * NT2 + j] + sgn * T[(g.NR - 1 - i) * NT2 + j]) * w0));
                    }
                }
                mx = fmax(mx, m1);
            }
            cmax[h * NT2 + j] = mx;
            bar_producers();
            if (h == 0)
                ebs[(k & 1) * NT2 + j] =
                    cok ? scale_exp(fmax(fmax(cmax[j], cmax[NT2 + j]), fmax(cmax[2 * NT2 + j], cmax[3 * NT2 + j]))) : 0;
            bar_producers();
            const int eb = ebs[(k & 1) * NT2 + j];
            mbar_arrive(&eb_ready[k & 1]);
            const double bsc = ldexp(1.0, 8 - eb);
            for (int ci = 0; ci < n0 + n1; ++ci) {
                const int p = (MODE == 0) ? (ci < n0 ? 0 : 1) : pr;
                const int c = (MODE == 0 && ci >= n0) ? ci - n0 : ci;
                double x[4];
                if (MODE == 0) {
                    const int kp = p ? nn / 2 : (nn + 1) / 2;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int t = 16 * c + 4 * h + u;
                        x[u] = (cok && t < kp) ? T[(2 * t + p) * NT2 + j] * bsc : 0.0;
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int i = 16 * c + 4 * h + u;
                        double f = 0.0;
                        if (cok && i < g.NRH) {
                            const double lo = T[i * NT2 + j], hi = T[(g.NR - 1 - i) * NT2 + j];
                            f = fp ? lo - hi : lo + hi;
                            if (P.use_w) f *= wsm[i];
                        }
                        x[u] = f * bsc;
                    }
                }
                const uint32_t s = gch % NS, rnd = gch / NS;
                if (rnd > 0 && !*abort_f) wait_ab(&empty[s], (rnd - 1) & 1, abort_f, P.wlim);
                if (STREAM && pt == 0 && !*abort_f) {
                    mbar_expect_tx(&full[s], CB);
                    bulk_g2s(stA + s * SA, P.img + (size_t)((m * 2 + p) * P.NCH + c) * CB, CB, &full[s]);
                    ++issued;
                }
                uint2 o[S];
                split4<S>(x, o);
                uint8_t* dst = stB + s * SB + (j >> 3) * 256 + (h >> 1) * 128 + (j & 7) * 16 + (h & 1) * 8;
#pragma unroll
                for (int q = 0; q < S; ++q) *(uint2*)(dst + q * BSLICE) = o[q];
                fence_async_smem();
                mbar_arrive(&full[s]);
                ++gch;
            }
        }
        // on an abort, let what this thread issued land before the CTA exits
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (pt == 0 && *abort_f) {
            const uint32_t first = issued > (uint32_t)NS ? issued - NS : 0;
            for (uint32_t q = first; q < issued; ++q) mbar_wait(&full[q % NS], (q / NS) & 1);
            if (MODE == 1 && !STREAM && a_loads > 0) mbar_wait(a_full, (a_loads - 1) & 1);
        }
    } else if (warp == 8) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t a0 = saddr(stA), b0 = saddr(stB);
            uint32_t gch = 0, tt = 0, a_uses = 0;
            int cur_mp = -1;
            for (int item = ib; item < ie && !*abort_f; item += istep) {
                int m, pr, tile, nn, n0, n1;
                item_info(item, m, pr, tile, nn, n0, n1);
                if (MODE == 1 && !STREAM && m * 2 + pr != cur_mp) {
                    if (a_uses > 0) mma_commit(a_free);
                    if (!wait_ab(a_full, a_uses & 1, abort_f, P.wlim)) break;
                    cur_mp = m * 2 + pr;
                    ++a_uses;
                }
                const int buf = tt % NBUF;
                if (tt >= (uint32_t)NBUF && !wait_ab(&tempty[buf], ((tt / NBUF) - 1) & 1, abort_f, P.wlim)) break;
                tc_after();
                bool ok = true;
                for (int ci = 0; ci < n0 + n1; ++ci) {
                    const int p = (MODE == 0) ? (ci < n0 ? 0 : 1) : 0;
                    const int c = (MODE == 0 && ci >= n0) ? ci - n0 : ci;
                    const uint32_t s = gch % NS, rnd = gch / NS;
                    if (!wait_ab(&full[s], rnd & 1, abort_f, P.wlim)) {
                        ok = false;
                        break;
                    }
                    tc_after();
                    // A slice qa against B slices 0..S-1-qa stacked along N: the products
                    // of levels qa..S-1 land in consecutive accumulators.
#pragma unroll
                    for (int qa = 0; qa < S; ++qa) {
                        const uint32_t abase = STREAM ? a0 + s * SA : a0 + c * CB;
                        const uint64_t ad = sdesc(abase + qa * P.RG * 256, 128, 256);
                        const uint64_t bd = sdesc(b0 + s * SB, 128, 256);
                        const uint32_t idesc = idesc_bf16(128, (S - qa) * NT2);
                        const uint32_t acc = (c > 0 || qa > 0) ? 1u : 0u;
                        mma_bf16(tbase + (uint32_t)(buf * 256 + (p * NL + qa) * NT2), ad, bd, idesc, acc);
                    }
                    mma_commit(&empty[s]);
                    ++gch;
                }
                if (!ok) break;
                mma_commit(&tfull[buf]);
                ++tt;
            }
            // every MMA issued has completed before the CTA frees its tensor memory
            mma_commit(done);
            mbar_wait(done, 0);
        }
    } else if (warp < 4) {
        // ------------------------------------------------------------ epilogue
        const int r = tid;  // TMEM lane
        const uint32_t tl = tbase + ((uint32_t)(warp * 32) << 16);
        uint32_t tt = 0;
        for (int item = ib; item < ie; item += istep, ++tt) {
            if (__any_sync(0xffffffffu, *abort_f != 0)) break;
            int m, pr, tile, nn, n0, n1;
            item_info(item, m, pr, tile, nn, n0, n1);
            const int buf = tt % NBUF;
            const bool w1 = wait_ab(&tfull[buf], (tt / NBUF) & 1, abort_f, P.wlim);
            const bool w2 = wait_ab(&eb_ready[tt & 1], (tt >> 1) & 1, abort_f, P.wlim);
            if (!__all_sync(0xffffffffu, w1 && w2)) break;
            tc_after();
            const int c0 = tile * NT2;
            const int* eb = ebs + (tt & 1) * NT2;
            if (MODE == 0) {
                const int i = r;
                const bool row_ok = i < g.NRH;
                const double sA0 = pow2((row_ok ? P.eA[(m * 2 + 0) * 128 + i] : 0) - 8);
                const double sA1 = pow2((row_ok ? P.eA[(m * 2 + 1) * 128 + i] : 0) - 8);
                const double lnv = (m == 0 && P.ln) ? *P.ln : 0.0;
                double* out = P.out + (size_t)m * g.NR * ncol;
                for (int cc = 0; cc < NT2 / 16; ++cc) {
                    double cp[2][16];
#pragma unroll
                    for (int p = 0; p < 2; ++p) {
                        const int np = p ? n1 : n0;
#pragma unroll
                        for (int q = 0; q < 16; ++q) cp[p][q] = 0.0;
                        if (np > 0) {
                            float a[NL][16];
#pragma unroll
                            for (int lv = 0; lv < NL; ++lv) tmem_ld16(tl + (uint32_t)((p * NL + lv) * NT2 + cc * 16), a[lv]);
                            tmem_ld_wait();
#pragma unroll
                            for (int lv = 0; lv < NL; ++lv)
#pragma unroll
                                for (int q = 0; q < 16; ++q) cp[p][q] += (double)a[lv][q];
                        }
                    }
                    if (!row_ok) continue;
                    double lo[16], hi[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const double sb = pow2(eb[cc * 16 + q] - 8);
                        const double ce = cp[0][q] * sA0 * sb;
                        const double co = cp[1][q] * sA1 * sb;
                        lo[q] = ce + co;
                        hi[q] = ce - co;
                    }
                    if (c0 + cc * 16 == 0 && lnv != 0.0) {
                        lo[0] += lnv * g.lnx[i];
                        hi[0] += lnv * g.lnx[g.NR - 1 - i];
                    }
                    double* o1 = out + (size_t)i * ncol + c0 + cc * 16;
                    double* o2 = out + (size_t)(g.NR - 1 - i) * ncol + c0 + cc * 16;
                    const int nq = min(16, ncol - (c0 + cc * 16));
                    if (nq == 16) {
#pragma unroll
                        for (int q = 0; q < 16; q += 2) {
                            *(double2*)(o1 + q) = make_double2(lo[q], lo[q + 1]);
                            *(double2*)(o2 + q) = make_double2(hi[q], hi[q + 1]);
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < 16; ++q)
                            if (q < nq) {
                                o1[q] = lo[q];
                                o2[q] = hi[q];
                            }
                    }
                }
            } else {
                const int n = 2 * r + pr;
                const bool row_out = n < g.NRCHOPDIM, row_val = n < nn;
                const double sA = pow2(((row_val && n0 > 0) ? P.eA[(m * 2 + pr) * 128 + r] : 0) - 8);
                double* out = P.out + (size_t)m * g.NRCHOPDIM * ncol;
                for (int cc = 0; cc < NT2 / 16; ++cc) {
                    double cp[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) cp[q] = 0.0;
                    if (n0 > 0) {
                        float a[NL][16];
#pragma unroll
                        for (int lv = 0; lv < NL; ++lv) tmem_ld16(tl + (uint32_t)(buf * 256 + lv * NT2 + cc * 16), a[lv]);
                        tmem_ld_wait();
#pragma unroll
                        for (int lv = 0; lv < NL; ++lv)
#pragma unroll
                            for (int q = 0; q < 16; ++q) cp[q] += (double)a[lv][q];
                    }
                    if (!row_out) continue;
#pragma unroll
                    for (int q = 0; q < 16; q += 2) {
                        const int cl = c0 + cc * 16 + q;  // even: real part of mode k = cl / 2
                        if (cl >= ncol) continue;
                        double re = 0.0, im = 0.0;
                        if (row_val && n0 > 0) {
                            re = cp[q] * sA * pow2(eb[cc * 16 + q] - 8);
                            im = cp[q + 1] * sA * pow2(eb[cc * 16 + q + 1] - 8);
                        }
                        const int k = cl >> 1;
                        double sr = re, si = im;
                        switch (P.scale) {
                            case 1: sr = -re; si = -im; break;
                            case 2: { const double f = -(double)m; sr = -im * f; si = re * f; } break;  // -i m v
                            case 3: { const double f = g.ak[k]; sr = -im * f; si = re * f; } break;     //  i k v
                            case 4: { const double f = (double)m * g.ak[k]; sr = re * f; si = im * f; } break;
                            default: break;
                        }
                        double2* dst = (double2*)(out + (size_t)n * ncol + cl);
                        if (!row_val) {
                            if (!P.accumulate) *dst = make_double2(0.0, 0.0);
                        } else if (P.accumulate) {
                            const double2 v = *dst;
                            *dst = make_double2(v.x + sr, v.y + si);
                        } else {
                            *dst = make_double2(sr, si);
                        }
                    }
                }
            }
            tc_before();
            mbar_arrive(&tempty[buf]);
            mbar_arrive(&eb_free[tt & 1]);
        }
    }
    __syncthreads();
    if (tid == 0 && *abort_f) atomicExch(P.err, 1);
    if (warp == 0) tmem_dealloc(tbase, TCOLS);
}

// ---------------------------------------------------------------------------
// Host side.

static int sm_count_split() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Geometry of one slice image: RG row groups, NCH chunks of 16 K values.
void split_geometry(const DevGrid& g, int mode, int wt_rows, int* RG, int* NCH) {
    if (mode == 0) {
        const int kt = (g.NRCHOPDIM + 2) / 2;  // t < ceil((NRCHOPDIM+1)/2)
        *RG = (g.NRH + 7) / 8;
        *NCH = (kt + 15) / 16;
    } else {
        *RG = ((wt_rows + 1) / 2 + 7) / 8;
        *NCH = (g.NRH + 15) / 16;
    }
}

static int tile_rows(const DevGrid& g, int mode) { return mode == 0 ? g.NRCHOPDIM : g.NR; }

size_t split_smem(int S, int RG, int NCH, int trows, int ns, bool stream) {
    const size_t sa = (size_t)(S * RG + 16 - RG) * 256, sb = (size_t)S * BSLICE;
    const size_t a = stream ? ns * sa : (size_t)NCH * S * RG * 256 + (size_t)(16 - RG) * 256;
    return 2 * (size_t)trows * NT2 * 8 + a + ns * sb + 2 * NT2 * 4 + 4 * NT2 * 8 + 128 * 8 + 8 * (2 * ns + 13) + 16 + 64;
}

// Ring depth and weight placement per mode: resident weight chunks (MODE 1)
// with 4, 3 or 2 stages where they fit, else streamed weights with 4, 3 or 2.
static int split_stages(const DevGrid& g, int S, int mode, int wt_rows, bool* stream) {
    int RG, NCH;
    split_geometry(g, mode, wt_rows, &RG, &NCH);
    for (int st = (mode == 0) ? 1 : 0; st < 2; ++st)
        for (int ns = 4; ns >= 2; --ns)
            if (split_smem(S, RG, NCH, tile_rows(g, mode), ns, st != 0) <= 227 * 1024) {
                *stream = st != 0;
                return ns;
            }
    return 0;
}

size_t split_image_bytes(const DevGrid& g, int S, int mode, int wt_rows) {
    int RG, NCH;
    split_geometry(g, mode, wt_rows, &RG, &NCH);
    return (size_t)g.NTCHOPDIM * 2 * NCH * S * RG * 256;
}

bool split_supported(const DevGrid& g, int S, int wt_rows) {
    if (S < 3 || S > 6 || g.NRH > 128 || g.NRH < 1) return false;
    for (int mode = 0; mode < 2; ++mode) {
        int RG, NCH;
        split_geometry(g, mode, wt_rows, &RG, &NCH);
        bool st;
        if (RG > 16 || split_stages(g, S, mode, wt_rows, &st) == 0) return false;
    }
    return true;
}

template <int S>
static void prep(const DevGrid& g, int mode, const double* W, int wt_rows, uint8_t* img, int* eA, cudaStream_t s) {
    int RG, NCH;
    split_geometry(g, mode, wt_rows, &RG, &NCH);
    if (mode == 0)
        slice_image_kernel<S, 0><<<dim3(g.NTCHOPDIM, 2), RG * 8, 0, s>>>(g, W, wt_rows, img, eA, RG, NCH);
    else
        slice_image_kernel<S, 1><<<dim3(g.NTCHOPDIM, 2), RG * 8, 0, s>>>(g, W, wt_rows, img, eA, RG, NCH);
    count_launch();
}

void k_split_prepare(const DevGrid& g, int S, int mode, const double* W, int wt_rows, uint8_t* img, int* eA,
                     cudaStream_t s) {
    switch (S) {
        case 3: prep<3>(g, mode, W, wt_rows, img, eA, s); break;
        case 4: prep<4>(g, mode, W, wt_rows, img, eA, s); break;
        case 5: prep<5>(g, mode, W, wt_rows, img, eA, s); break;
        default: prep<6>(g, mode, W, wt_rows, img, eA, s); break;
    }
}

template <int S, int MODE, int NS, bool STREAM>
static void launch_ns(const DevGrid& g, const SplitArgs& A, size_t smem, int grid, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(split_gemm_kernel<S, MODE, NS, STREAM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024);
        attr = true;
    }
    split_gemm_kernel<S, MODE, NS, STREAM><<<grid, NTH2, smem, s>>>(g, A);
}

template <int S, int MODE>
static void launch_split(const DevGrid& g, const SplitArgs& P, int wt_rows, cudaStream_t s) {
    int RG, NCH;
    split_geometry(g, MODE, wt_rows, &RG, &NCH);
    bool stream = true;
    const int ns = split_stages(g, S, MODE, wt_rows, &stream);
    SplitArgs A = P;
    A.RG = RG;
    A.NCH = NCH;
    A.trows = tile_rows(g, MODE);
    // at least 120 KB: one CTA per SM, so no CTA waits in tcgen05.alloc for another's columns
    const size_t smem = std::max(split_smem(S, RG, NCH, A.trows, ns, stream), (size_t)120 * 1024);
    const int ncol = 2 * g.NXCHOPDIM;
    const int nitems = (MODE == 0 ? 1 : 2) * g.NTCHOPDIM * ((ncol + NT2 - 1) / NT2);
    const int grid = std::min(nitems, sm_count_split());
    if constexpr (MODE == 0) {
        if (ns >= 4) launch_ns<S, MODE, 4, true>(g, A, smem, grid, s);
        else if (ns == 3) launch_ns<S, MODE, 3, true>(g, A, smem, grid, s);
        else launch_ns<S, MODE, 2, true>(g, A, smem, grid, s);
    } else if (stream) {
        if (ns >= 4) launch_ns<S, MODE, 4, true>(g, A, smem, grid, s);
        else if (ns == 3) launch_ns<S, MODE, 3, true>(g, A, smem, grid, s);
        else launch_ns<S, MODE, 2, true>(g, A, smem, grid, s);
    } else {
        if (ns >= 4) launch_ns<S, MODE, 4, false>(g, A, smem, grid, s);
        else if (ns == 3) launch_ns<S, MODE, 3, false>(g, A, smem, grid, s);
        else launch_ns<S, MODE, 2, false>(g, A, smem, grid, s);
    }
    count_launch();
}

template <int MODE>
static void launch_any(const DevGrid& g, int S, const SplitArgs& P, int wt_rows, cudaStream_t s) {
    switch (S) {
        case 3: launch_split<3, MODE>(g, P, wt_rows, s); break;
        case 4: launch_split<4, MODE>(g, P, wt_rows, s); break;
        case 5: launch_split<5, MODE>(g, P, wt_rows, s); break;
        default: launch_split<6, MODE>(g, P, wt_rows, s); break;
    }
}

void k_split_b2p(const DevGrid& g, int S, const uint8_t* img, const int* eA, const double2* a, double2* b,
                 const double* ln, int pad, int* err, uint64_t wait_cycles, cudaStream_t s) {
    SplitArgs P{};
    P.wlim = wait_cycles ? wait_cycles : WAIT_NS;
    P.img = img;
    P.eA = eA;
    P.in = (const double*)a;
    P.out = (double*)b;
    P.ln = ln;
    P.err = err;
    P.pad = pad;
    launch_any<0>(g, S, P, 0, s);
}

void k_split_fold(const DevGrid& g, int S, const uint8_t* img, const int* eA, int wt_rows, const double2* in,
                  double2* out, int mode, int scale, int accumulate, int pad, int use_w, int* err,
                  uint64_t wait_cycles, cudaStream_t s) {
    SplitArgs P{};
    P.wlim = wait_cycles ? wait_cycles : WAIT_NS;
    P.img = img;
    P.eA = eA;
    P.in = (const double*)in;
    P.out = (double*)out;
    P.err = err;
    P.pad = pad;
    P.mode = mode & 1;
    P.scale = scale;
    P.accumulate = accumulate;
    P.use_w = use_w;
    launch_any<1>(g, S, P, wt_rows, s);
}

}  // namespace mlegs
