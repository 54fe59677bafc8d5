// Split-BF16 (Ozaki) Legendre GEMMs on the fifth-generation tensor cores.
//
// RTRAN(A, +1) (mod_fft.f90:1264-1336) per m and parity p:
//     C_p(i, c) = sum_t PF(i, 2t+p) A(2t+p, c),   B(i) = C_0 + C_1, B(NR-1-i) = C_0 - C_1
// is computed from S slices per operand.  Each row i of PF (per m, p) and each
// column c of A (per m) is scaled by a power of two into (-1, 1) and written as
//     v = sum_q a_q 2^{-8(q+1)},  a_q integer, |a_0| <= 256, |a_q| <= 128 (q > 0),
// each a_q stored in BF16 pre-multiplied by 2^{-8q} (exact).  The products
// a_qa b_qb with qa + qb <= S-1 go to four FP32 accumulators in tensor memory:
//     level 0 (qa+qb = 0), level 1, level 2, levels >= 3,
// so levels 0..2 are exact (every partial sum is a multiple of the level's
// unit 2^{-8L} and below 2^{24-8L}: K <= 128) and the rounded fourth level
// sits near 2^-48 of the row x column scale.  The epilogue adds the four in FP64 and
// applies the two power-of-two scales, the parity butterfly and the
// (m, k) = (0, 0) log term.
//
// Kernel structure (one CTA = one m and a range of 64-column tiles):
//   - the PF slices of both parities for this m sit in shared memory for the
//     whole CTA (one bulk copy per slice, completion on an mbarrier);
//   - the A-column slices are made by all threads from the FP64 field, 16
//     K-rows at a time, into a 3-stage ring;
//   - one thread issues tcgen05.mma (M=128, N=64, K=16, BF16 x BF16 -> F32)
//     for the S(S+1)/2 slice pairs of each K-chunk and commits them to the
//     ring stage's mbarrier;
//   - the epilogue reads the accumulators with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = output rows i).
// Shared-memory operands use the K-major no-swizzle canonical layout: core
// matrices of 8 rows x 16 bytes, LBO = 128 B between the two K halves of a
// K=16 step, SBO between 8-row groups.  Every wait is bounded (1 s); on a
// timeout the kernel raises *err, drains what it issued and frees its tensor
// memory before returning.
#include "mlegs_internal.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

namespace mlegs {

namespace {

constexpr int NT = 64;    // output columns per tile (MMA N)
constexpr int NST = 3;    // B ring stages
constexpr int NTHR = 128;
constexpr uint64_t WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

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

// Waits for the phase of `parity` to complete; false after WAIT_NS.
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

// Slices of 8 values (already multiplied by 2^{8-e}, |x| < 256) -> S packed
// rows of 8 BF16 each; slice q holds a_q 2^{-8q}.
template <int S>
__device__ __forceinline__ void split8(double (&x)[8], uint4 (&out)[S]) {
    uint32_t w[S][4];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        double v = x[u];
        double sc = 1.0;
#pragma unroll
        for (int q = 0; q < S; ++q) {
            const double a = rint(v);
            v = (v - a) * 256.0;
            const unsigned short b = __bfloat16_as_ushort(__float2bfloat16_rn((float)(a * sc)));
            sc *= 0.00390625;
            if (u & 1) w[q][u >> 1] |= (uint32_t)b << 16;
            else w[q][u >> 1] = b;
        }
    }
#pragma unroll
    for (int q = 0; q < S; ++q) out[q] = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
}

}  // namespace

// ---------------------------------------------------------------------------
// PF slices for RTRAN(+1): image[(m*2+p)][q][rg][kc][row%8][8 bf16], row = i,
// K index t (n = 2t+p), one row-group slab = KC*128 bytes; eA[(m*2+p)*128+i].
template <int S>
__global__ void pf_split_kernel(DevGrid g, uint8_t* img, int* eA, int RG, int KC) {
    const int m = blockIdx.x, p = blockIdx.y, i = threadIdx.x;
    if (i >= RG * 8) return;
    const int ne = g.NRCHOPDIM + 1;
    const int kt = (ne - p + 1) / 2;
    const double* pf = g.pf + (size_t)m * ne * g.NRH;
    double mx = 0.0;
    if (i < g.NRH)
        for (int t = 0; t < kt; ++t) mx = fmax(mx, fabs(pf[(size_t)(2 * t + p) * g.NRH + i]));
    const int e = scale_exp(mx);
    eA[(m * 2 + p) * 128 + i] = e;
    const double sc = ldexp(1.0, 8 - e);
    const size_t sbo = (size_t)KC * 128;
    uint8_t* base = img + (size_t)(m * 2 + p) * S * RG * sbo;
    for (int kc = 0; kc < KC; ++kc) {
        double x[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int t = kc * 8 + u;
            x[u] = (i < g.NRH && t < kt) ? pf[(size_t)(2 * t + p) * g.NRH + i] * sc : 0.0;
        }
        uint4 o[S];
        split8<S>(x, o);
#pragma unroll
        for (int q = 0; q < S; ++q)
            *(uint4*)(base + (size_t)q * RG * sbo + (size_t)(i >> 3) * sbo + kc * 128 + (i & 7) * 16) = o[q];
    }
}

struct B2PArgs {
    const uint8_t* img;
    const int* eA;
    const double* in;   // FFF as doubles [m][n][2*NXCHOPDIM]
    double* out;        // PFF as doubles [m][r][2*NXCHOPDIM]
    const double* ln;
    int* err;
    int pad, RG, KC, tiles_per_cta;
};

template <int S>
__global__ void __launch_bounds__(NTHR, 1) split_b2p_kernel(DevGrid g, B2PArgs P) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = blockIdx.x;
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntiles = (ncol + NT - 1) / NT;
    const int tile0 = blockIdx.y * P.tiles_per_cta;
    const int tile1 = min(tile0 + P.tiles_per_cta, ntiles);
    if (tile0 >= tile1) return;

    const uint32_t SBO_A = P.KC * 128;
    const uint32_t A_par = S * P.RG * SBO_A;
    const uint32_t A_tot = ((2 * A_par + (16 - P.RG) * SBO_A) + 1023) & ~1023u;
    constexpr uint32_t B_slice = (NT / 8) * 256;
    constexpr uint32_t B_stage = S * B_slice;
    uint8_t* Asm = sm;
    uint8_t* Bsm = sm + A_tot;
    uint64_t* bars = (uint64_t*)(Bsm + NST * B_stage);  // [0] A full, [1..NST] MMA done
    uint32_t* tslot = (uint32_t*)(bars + 1 + NST);
    int* abort_f = (int*)(tslot + 1);
    int* eB = abort_f + 1;                               // [NT]
    double* cmax = (double*)(((uintptr_t)(eB + NT) + 15) & ~(uintptr_t)15);  // [2][NT]

    int nn = g.NRCHOP + P.pad - m;
    if (nn < 0) nn = 0;
    const int kp[2] = {(nn + 1) / 2, nn / 2};
    const int nch[2] = {(kp[0] + 15) / 16, (kp[1] + 15) / 16};
    const double* in = P.in + (size_t)m * g.NRCHOPDIM * ncol;
    double* out = P.out + (size_t)m * g.NR * ncol;

    if (warp == 0) tmem_alloc(tslot, 512);
    if (tid == 0) {
        for (int q = 0; q < 1 + NST; ++q) mbar_init(&bars[q], 1);
        *abort_f = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    tc_after();
    const uint32_t tbase = *tslot;
    bool a_issued = false;
    if (tid == 0 && nn > 0) {
        const uint8_t* src = P.img + (size_t)(m * 2) * A_par;
        mbar_expect_tx(&bars[0], 2 * A_par);
        for (int q = 0; q < 2 * S; ++q) bulk_g2s(Asm + q * (A_par / S), src + (size_t)q * (A_par / S), A_par / S, &bars[0]);
        a_issued = true;
    }
    bool a_ready = false;
    uint32_t gchunk = 0;
    constexpr uint32_t IDESC = idesc_bf16(128, NT);
    const uint32_t a_base = saddr(Asm), b_base = saddr(Bsm);

    for (int tile = tile0; tile < tile1; ++tile) {
        const int c0 = tile * NT;
        const int j = tid % NT, h = tid / NT;
        const int col = c0 + j;
        // column scale over all n < nn of this column (parity h rows by this thread)
        double mx = 0.0;
        if (col < ncol)
            for (int t = 0; t < kp[h]; ++t) mx = fmax(mx, fabs(in[(size_t)(2 * t + h) * ncol + col]));
        cmax[h * NT + j] = mx;
        __syncthreads();
        if (tid < NT) eB[tid] = scale_exp(fmax(cmax[tid], cmax[NT + tid]));
        __syncthreads();
        const double bsc = ldexp(1.0, 8 - eB[j]);
        const int total = nch[0] + nch[1];
        for (int ci = 0; ci < total; ++ci) {
            const int p = ci < nch[0] ? 0 : 1;
            const int c = p ? ci - nch[0] : ci;
            const uint32_t stage = gchunk % NST, use = gchunk / NST;
            if (use > 0 && !mbar_wait(&bars[1 + stage], (use - 1) & 1)) atomicExch(abort_f, 1);
            // B chunk: K rows t = 16c + 8h + u of parity p, column j
            double x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int t = 16 * c + 8 * h + u;
                x[u] = (t < kp[p] && col < ncol) ? in[(size_t)(2 * t + p) * ncol + col] * bsc : 0.0;
            }
            uint4 o[S];
            split8<S>(x, o);
            uint8_t* bst = Bsm + stage * B_stage + (j >> 3) * 256 + h * 128 + (j & 7) * 16;
#pragma unroll
            for (int q = 0; q < S; ++q) *(uint4*)(bst + q * B_slice) = o[q];
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                if (!a_ready) {
                    if (!mbar_wait(&bars[0], 0)) atomicExch(abort_f, 1);
                    a_ready = true;
                }
                tc_after();
                if (*abort_f == 0) {
                    const uint32_t a_par = a_base + p * A_par + c * 256;
                    const uint32_t b_stg = b_base + stage * B_stage;
                    bool first = (c == 0);
                    uint32_t init_mask = 0;
                    for (int qa = 0; qa < S; ++qa)
                        for (int qb = 0; qb + qa < S; ++qb) {
                            const int lv = min(qa + qb, 3);
                            const uint32_t d = tbase + (uint32_t)((p * 4 + lv) * NT);
                            const uint64_t ad = sdesc(a_par + qa * P.RG * SBO_A, 128, SBO_A);
                            const uint64_t bd = sdesc(b_stg + qb * B_slice, 128, 256);
                            const uint32_t acc = (!first || (init_mask >> lv) & 1) ? 1u : 0u;
                            mma_bf16(d, ad, bd, IDESC, acc);
                            init_mask |= 1u << lv;
                        }
                }
                mma_commit(&bars[1 + stage]);
            }
            ++gchunk;
        }
        // all MMAs of this tile complete
        if (total > 0) {
            const uint32_t ls = (gchunk - 1) % NST, lu = (gchunk - 1) / NST;
            if (!mbar_wait(&bars[1 + ls], lu & 1)) atomicExch(abort_f, 1);
        }
        tc_after();
        __syncthreads();
        if (*abort_f) break;
        // epilogue: row i = TMEM lane
        const int i = warp * 32 + lane;
        const bool row_ok = i < g.NRH;
        const int eAe = row_ok ? P.eA[(m * 2 + 0) * 128 + i] : 0;
        const int eAo = row_ok ? P.eA[(m * 2 + 1) * 128 + i] : 0;
        const double lnv = (m == 0 && P.ln) ? *P.ln : 0.0;
        const uint32_t tl = tbase + ((uint32_t)(warp * 32) << 16);
        for (int cc = 0; cc < NT / 16; ++cc) {
            double cp[2][16];
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                float a[4][16];
#pragma unroll
                for (int lv = 0; lv < 4; ++lv) tmem_ld16(tl + (uint32_t)((p * 4 + lv) * NT + cc * 16), a[lv]);
                tmem_ld_wait();
#pragma unroll
                for (int q = 0; q < 16; ++q)  // level 3 exists only when S > 3
                    cp[p][q] = nch[p] ? ((double)a[0][q] + (double)a[1][q]) +
                                            ((double)a[2][q] + (S > 3 ? (double)a[3][q] : 0.0))
                                      : 0.0;
            }
            if (!row_ok) continue;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int jj = cc * 16 + q;
                const int cl = c0 + jj;
                if (cl >= ncol) continue;
                const double ce = ldexp(cp[0][q], eAe + eB[jj] - 16);
                const double co = ldexp(cp[1][q], eAo + eB[jj] - 16);
                double lo = ce + co, hi = ce - co;
                if (cl == 0 && lnv != 0.0) {
                    lo += lnv * g.lnx[i];
                    hi += lnv * g.lnx[g.NR - 1 - i];
                }
                out[(size_t)i * ncol + cl] = lo;
                out[(size_t)(g.NR - 1 - i) * ncol + cl] = hi;
            }
        }
        tc_before();
        __syncthreads();
    }
    // drain: nothing of ours may still be writing shared or tensor memory
    if (tid == 0) {
        if (a_issued && !a_ready) mbar_wait(&bars[0], 0);
        if (*abort_f) atomicExch(P.err, 1);
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, 512);
}

// ---------------------------------------------------------------------------
// Fold GEMMs: RTRAN(A, -1) (mod_fft.f90:1189-1261) and the EOMUL/OEMUL
// products of PROJECT (mod_legops.f90:2497-2535, 2548-2648):
//     out(n, c) (+)= s(m, k) sum_{i < NRH} Wt(n, i) F(i, c),
//     F = x(i) + x(NR-1-i) (even fold) or x(i) - x(NR-1-i) (odd fold), times w_i
//     for RTRAN(-1); the fold of row n is parity(n) xor mode.
// One CTA computes the rows n = 2r + pr (r = TMEM lane) of one parity pr for
// one m and a group of 64-column tiles, so both operands and the four level
// accumulators (256 TMEM columns) fit twice per SM.  Wt slices: image
// [(m*2+pr)][q][rg][kc][r%8][8 bf16] with K = i; eA[(m*2+pr)*128 + r].
template <int S>
__global__ void wt_split_kernel(DevGrid g, const double* Wt, int wt_rows, uint8_t* img, int* eA, int RG, int KC) {
    const int m = blockIdx.x, pr = blockIdx.y, r = threadIdx.x;
    if (r >= RG * 8) return;
    const int n = 2 * r + pr;
    const double* w = Wt + ((size_t)m * wt_rows + n) * g.NRH;
    const bool ok = n < wt_rows;
    double mx = 0.0;
    if (ok)
        for (int i = 0; i < g.NRH; ++i) mx = fmax(mx, fabs(w[i]));
    const int e = scale_exp(mx);
    eA[(m * 2 + pr) * 128 + r] = e;
    const double sc = ldexp(1.0, 8 - e);
    const size_t sbo = (size_t)KC * 128;
    uint8_t* base = img + (size_t)(m * 2 + pr) * S * RG * sbo;
    for (int kc = 0; kc < KC; ++kc) {
        double x[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = kc * 8 + u;
            x[u] = (ok && i < g.NRH) ? w[i] * sc : 0.0;
        }
        uint4 o[S];
        split8<S>(x, o);
#pragma unroll
        for (int q = 0; q < S; ++q)
            *(uint4*)(base + (size_t)q * RG * sbo + (size_t)(r >> 3) * sbo + kc * 128 + (r & 7) * 16) = o[q];
    }
}

struct FoldArgs {
    const uint8_t* img;
    const int* eA;
    const double* in;   // PFF as doubles [m][r][2*NXCHOPDIM]
    double* out;        // FFF as doubles [m][n][2*NXCHOPDIM]
    int* err;
    int pad, RG, KC, tiles_per_cta, mode, scale, accumulate, use_w;
};

template <int S>
__global__ void __launch_bounds__(NTHR, 2) split_fold_kernel(DevGrid g, FoldArgs P) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = blockIdx.x, pr = blockIdx.y & 1;
    const int ncol = 2 * g.NXCHOPDIM;
    const int ntiles = (ncol + NT - 1) / NT;
    const int tile0 = (blockIdx.y >> 1) * P.tiles_per_cta;
    const int tile1 = min(tile0 + P.tiles_per_cta, ntiles);
    if (tile0 >= tile1) return;

    const uint32_t SBO_A = P.KC * 128;
    const uint32_t A_img = S * P.RG * SBO_A;
    const uint32_t A_tot = ((A_img + (16 - P.RG) * SBO_A) + 1023) & ~1023u;
    constexpr uint32_t B_slice = (NT / 8) * 256;
    constexpr uint32_t B_stage = S * B_slice;
    uint8_t* Asm = sm;
    uint8_t* Bsm = sm + A_tot;
    uint64_t* bars = (uint64_t*)(Bsm + NST * B_stage);
    uint32_t* tslot = (uint32_t*)(bars + 1 + NST);
    int* abort_f = (int*)(tslot + 1);
    int* eB = abort_f + 1;
    double* cmax = (double*)(((uintptr_t)(eB + NT) + 15) & ~(uintptr_t)15);

    int nn = g.NRCHOP + P.pad - m;
    if (nn < 0) nn = 0;
    const int fold = pr ^ P.mode;  // 0: x_i + x_{NR-1-i}, 1: x_i - x_{NR-1-i}
    const int nch = (g.NRH + 15) / 16;
    const bool any_rows = pr < nn;  // some n = 2r + pr < nn
    const double* x = P.in + (size_t)m * g.NR * ncol;
    double* out = P.out + (size_t)m * g.NRCHOPDIM * ncol;

    if (warp == 0) tmem_alloc(tslot, 256);
    if (tid == 0) {
        for (int q = 0; q < 1 + NST; ++q) mbar_init(&bars[q], 1);
        *abort_f = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    tc_after();
    const uint32_t tbase = *tslot;
    bool a_issued = false;
    if (tid == 0 && any_rows) {
        const uint8_t* src = P.img + (size_t)(m * 2 + pr) * A_img;
        mbar_expect_tx(&bars[0], A_img);
        for (int q = 0; q < S; ++q) bulk_g2s(Asm + q * (A_img / S), src + (size_t)q * (A_img / S), A_img / S, &bars[0]);
        a_issued = true;
    }
    bool a_ready = false;
    uint32_t gchunk = 0;
    constexpr uint32_t IDESC = idesc_bf16(128, NT);
    const uint32_t a_base = saddr(Asm), b_base = saddr(Bsm);

    for (int tile = tile0; tile < tile1; ++tile) {
        const int c0 = tile * NT;
        const int j = tid % NT, h = tid / NT;
        const int col = c0 + j;
        const int total = any_rows ? nch : 0;
        if (total > 0) {
            double mx = 0.0;
            if (col < ncol)
                for (int i = h; i < g.NRH; i += 2) {
                    double f = fold ? x[(size_t)i * ncol + col] - x[(size_t)(g.NR - 1 - i) * ncol + col]
                                    : x[(size_t)i * ncol + col] + x[(size_t)(g.NR - 1 - i) * ncol + col];
                    if (P.use_w) f *= g.w[i];
                    mx = fmax(mx, fabs(f));
                }
            cmax[h * NT + j] = mx;
            __syncthreads();
            if (tid < NT) eB[tid] = scale_exp(fmax(cmax[tid], cmax[NT + tid]));
            __syncthreads();
        }
        const double bsc = ldexp(1.0, 8 - (total > 0 ? eB[j] : 0));
        for (int c = 0; c < total; ++c) {
            const uint32_t stage = gchunk % NST, use = gchunk / NST;
            if (use > 0 && !mbar_wait(&bars[1 + stage], (use - 1) & 1)) atomicExch(abort_f, 1);
            double xv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = 16 * c + 8 * h + u;
                double f = 0.0;
                if (i < g.NRH && col < ncol) {
                    const double lo = x[(size_t)i * ncol + col], hi = x[(size_t)(g.NR - 1 - i) * ncol + col];
                    f = fold ? lo - hi : lo + hi;
                    if (P.use_w) f *= g.w[i];
                }
                xv[u] = f * bsc;
            }
            uint4 o[S];
            split8<S>(xv, o);
            uint8_t* bst = Bsm + stage * B_stage + (j >> 3) * 256 + h * 128 + (j & 7) * 16;
#pragma unroll
            for (int q = 0; q < S; ++q) *(uint4*)(bst + q * B_slice) = o[q];
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                if (!a_ready) {
                    if (!mbar_wait(&bars[0], 0)) atomicExch(abort_f, 1);
                    a_ready = true;
                }
                tc_after();
                if (*abort_f == 0) {
                    const uint32_t a_k = a_base + c * 256;
                    const uint32_t b_stg = b_base + stage * B_stage;
                    uint32_t init_mask = 0;
                    for (int qa = 0; qa < S; ++qa)
                        for (int qb = 0; qb + qa < S; ++qb) {
                            const int lv = min(qa + qb, 3);
                            const uint64_t ad = sdesc(a_k + qa * P.RG * SBO_A, 128, SBO_A);
                            const uint64_t bd = sdesc(b_stg + qb * B_slice, 128, 256);
                            const uint32_t acc = (c > 0 || (init_mask >> lv) & 1) ? 1u : 0u;
                            mma_bf16(tbase + (uint32_t)(lv * NT), ad, bd, IDESC, acc);
                            init_mask |= 1u << lv;
                        }
                }
                mma_commit(&bars[1 + stage]);
            }
            ++gchunk;
        }
        if (total > 0) {
            const uint32_t ls = (gchunk - 1) % NST, lu = (gchunk - 1) / NST;
            if (!mbar_wait(&bars[1 + ls], lu & 1)) atomicExch(abort_f, 1);
        }
        tc_after();
        __syncthreads();
        if (*abort_f) break;
        // epilogue: TMEM lane r -> row n = 2r + pr
        const int r = warp * 32 + lane;
        const int n = 2 * r + pr;
        const bool row_out = n < g.NRCHOPDIM;
        const bool row_val = n < nn;
        const int ea = (row_val && total > 0) ? P.eA[(m * 2 + pr) * 128 + r] : 0;
        const uint32_t tl = tbase + ((uint32_t)(warp * 32) << 16);
        for (int cc = 0; cc < NT / 16; ++cc) {
            float a[4][16];
            if (total > 0) {
#pragma unroll
                for (int lv = 0; lv < 4; ++lv) tmem_ld16(tl + (uint32_t)(lv * NT + cc * 16), a[lv]);
                tmem_ld_wait();
            }
            if (!row_out) continue;
#pragma unroll
            for (int q = 0; q < 16; q += 2) {
                const int cl = c0 + cc * 16 + q;  // even: real part of mode k = cl / 2
                if (cl >= ncol) continue;
                double re = 0.0, im = 0.0;
                if (row_val && total > 0) {
                    const double s0 = ((double)a[0][q] + (double)a[1][q]) +
                                      ((double)a[2][q] + (S > 3 ? (double)a[3][q] : 0.0));
                    const double s1 = ((double)a[0][q + 1] + (double)a[1][q + 1]) +
                                      ((double)a[2][q + 1] + (S > 3 ? (double)a[3][q + 1] : 0.0));
                    re = ldexp(s0, ea + eB[cc * 16 + q] - 16);
                    im = ldexp(s1, ea + eB[cc * 16 + q + 1] - 16);
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
                double* dst = out + (size_t)n * ncol + cl;
                if (!row_val) {
                    if (!P.accumulate) { dst[0] = 0.0; dst[1] = 0.0; }
                } else if (P.accumulate) {
                    dst[0] += sr;
                    dst[1] += si;
                } else {
                    dst[0] = sr;
                    dst[1] = si;
                }
            }
        }
        tc_before();
        __syncthreads();
    }
    if (tid == 0) {
        if (a_issued && !a_ready) mbar_wait(&bars[0], 0);
        if (*abort_f) atomicExch(P.err, 1);
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, 256);
}

// ---------------------------------------------------------------------------
// Host side.

size_t split_b2p_smem(int S, int RG, int KC) {
    const size_t sbo = (size_t)KC * 128;
    const size_t a_par = (size_t)S * RG * sbo;
    const size_t a_tot = ((2 * a_par + (16 - RG) * sbo) + 1023) & ~(size_t)1023;
    const size_t b = (size_t)NST * S * (NT / 8) * 256;
    return a_tot + b + 8 * (1 + NST) + 8 + 4 * NT + 16 + 16 * NT + 64;
}

void split_geometry(const DevGrid& g, int* RG, int* KC) {
    const int kt = (g.NRCHOPDIM + 1 + 1) / 2;
    const int kp = (kt + 15) / 16 * 16;
    *RG = (g.NRH + 7) / 8;
    *KC = kp / 8;
}

size_t split_b2p_image_bytes(const DevGrid& g, int S) {
    int RG, KC;
    split_geometry(g, &RG, &KC);
    return (size_t)g.NTCHOPDIM * 2 * S * RG * KC * 128;
}

bool split_supported(const DevGrid& g, int S) {
    if (S < 3 || S > 6 || g.NRH > 128 || g.NRH < 1) return false;
    int RG, KC;
    split_geometry(g, &RG, &KC);
    return split_b2p_smem(S, RG, KC) <= 227 * 1024;
}

template <int S>
static void launch_prepare(const DevGrid& g, uint8_t* img, int* eA, cudaStream_t s) {
    int RG, KC;
    split_geometry(g, &RG, &KC);
    pf_split_kernel<S><<<dim3(g.NTCHOPDIM, 2), RG * 8, 0, s>>>(g, img, eA, RG, KC);
    count_launch();
}

void k_split_prepare(const DevGrid& g, int S, uint8_t* img, int* eA, cudaStream_t s) {
    switch (S) {
        case 3: launch_prepare<3>(g, img, eA, s); break;
        case 4: launch_prepare<4>(g, img, eA, s); break;
        case 5: launch_prepare<5>(g, img, eA, s); break;
        default: launch_prepare<6>(g, img, eA, s); break;
    }
}

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

template <int S>
static void launch_b2p(const DevGrid& g, const uint8_t* img, const int* eA, const double2* a, double2* b,
                       const double* ln, int pad, int* err, cudaStream_t s) {
    int RG, KC;
    split_geometry(g, &RG, &KC);
    // at least 120 KB: one CTA per SM, so no CTA waits in tcgen05.alloc for another's 512 columns
    const size_t smem = std::max(split_b2p_smem(S, RG, KC), (size_t)120 * 1024);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(split_b2p_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    const int ntiles = (2 * g.NXCHOPDIM + NT - 1) / NT;
    int groups = std::max(1, std::min(ntiles, (2 * sm_count_split() + g.NTCHOPDIM - 1) / g.NTCHOPDIM));
    const int per = (ntiles + groups - 1) / groups;
    groups = (ntiles + per - 1) / per;
    B2PArgs P;
    P.img = img;
    P.eA = eA;
    P.in = (const double*)a;
    P.out = (double*)b;
    P.ln = ln;
    P.err = err;
    P.pad = pad;
    P.RG = RG;
    P.KC = KC;
    P.tiles_per_cta = per;
    split_b2p_kernel<S><<<dim3(g.NTCHOPDIM, groups), NTHR, smem, s>>>(g, P);
    count_launch();
}

void k_split_b2p(const DevGrid& g, int S, const uint8_t* img, const int* eA, const double2* a, double2* b,
                 const double* ln, int pad, int* err, cudaStream_t s) {
    switch (S) {
        case 3: launch_b2p<3>(g, img, eA, a, b, ln, pad, err, s); break;
        case 4: launch_b2p<4>(g, img, eA, a, b, ln, pad, err, s); break;
        case 5: launch_b2p<5>(g, img, eA, a, b, ln, pad, err, s); break;
        default: launch_b2p<6>(g, img, eA, a, b, ln, pad, err, s); break;
    }
}

// ---- fold GEMMs
void fold_geometry(const DevGrid& g, int wt_rows, int* RG, int* KC) {
    const int kp = (g.NRH + 15) / 16 * 16;
    *RG = ((wt_rows + 1) / 2 + 7) / 8;
    *KC = kp / 8;
}

size_t split_fold_smem(int S, int RG, int KC) {
    const size_t sbo = (size_t)KC * 128;
    const size_t a_tot = (((size_t)S * RG * sbo + (16 - RG) * sbo) + 1023) & ~(size_t)1023;
    const size_t b = (size_t)NST * S * (NT / 8) * 256;
    return a_tot + b + 8 * (1 + NST) + 8 + 4 * NT + 16 + 16 * NT + 64;
}

size_t split_fold_image_bytes(const DevGrid& g, int S, int wt_rows) {
    int RG, KC;
    fold_geometry(g, wt_rows, &RG, &KC);
    return (size_t)g.NTCHOPDIM * 2 * S * RG * KC * 128;
}

bool split_fold_supported(const DevGrid& g, int S, int wt_rows) {
    int RG, KC;
    fold_geometry(g, wt_rows, &RG, &KC);
    return RG <= 16 && g.NRH <= 128 && split_fold_smem(S, RG, KC) <= 227 * 1024;
}

template <int S>
static void launch_wt_prepare(const DevGrid& g, const double* Wt, int wt_rows, uint8_t* img, int* eA,
                              cudaStream_t s) {
    int RG, KC;
    fold_geometry(g, wt_rows, &RG, &KC);
    wt_split_kernel<S><<<dim3(g.NTCHOPDIM, 2), RG * 8, 0, s>>>(g, Wt, wt_rows, img, eA, RG, KC);
    count_launch();
}

void k_split_prepare_wt(const DevGrid& g, int S, const double* Wt, int wt_rows, uint8_t* img, int* eA,
                        cudaStream_t s) {
    switch (S) {
        case 3: launch_wt_prepare<3>(g, Wt, wt_rows, img, eA, s); break;
        case 4: launch_wt_prepare<4>(g, Wt, wt_rows, img, eA, s); break;
        case 5: launch_wt_prepare<5>(g, Wt, wt_rows, img, eA, s); break;
        default: launch_wt_prepare<6>(g, Wt, wt_rows, img, eA, s); break;
    }
}

template <int S>
static void launch_fold(const DevGrid& g, const uint8_t* img, const int* eA, int wt_rows, const double2* in,
                        double2* out, int mode, int scale, int accumulate, int pad, int use_w, int* err,
                        cudaStream_t s) {
    int RG, KC;
    fold_geometry(g, wt_rows, &RG, &KC);
    // at least 80 KB: at most two CTAs (2 x 256 TMEM columns) per SM
    const size_t smem = std::max(split_fold_smem(S, RG, KC), (size_t)80 * 1024);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(split_fold_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    const int ntiles = (2 * g.NXCHOPDIM + NT - 1) / NT;
    int groups = std::max(1, std::min(ntiles, (4 * sm_count_split() + 2 * g.NTCHOPDIM - 1) / (2 * g.NTCHOPDIM)));
    const int per = (ntiles + groups - 1) / groups;
    groups = (ntiles + per - 1) / per;
    FoldArgs P;
    P.img = img;
    P.eA = eA;
    P.in = (const double*)in;
    P.out = (double*)out;
    P.err = err;
    P.pad = pad;
    P.RG = RG;
    P.KC = KC;
    P.tiles_per_cta = per;
    P.mode = mode & 1;
    P.scale = scale;
    P.accumulate = accumulate;
    P.use_w = use_w;
    split_fold_kernel<S><<<dim3(g.NTCHOPDIM, 2 * groups), NTHR, smem, s>>>(g, P);
    count_launch();
}

void k_split_fold(const DevGrid& g, int S, const uint8_t* img, const int* eA, int wt_rows, const double2* in,
                  double2* out, int mode, int scale, int accumulate, int pad, int use_w, int* err, cudaStream_t s) {
    switch (S) {
        case 3: launch_fold<3>(g, img, eA, wt_rows, in, out, mode, scale, accumulate, pad, use_w, err, s); break;
        case 4: launch_fold<4>(g, img, eA, wt_rows, in, out, mode, scale, accumulate, pad, use_w, err, s); break;
        case 5: launch_fold<5>(g, img, eA, wt_rows, in, out, mode, scale, accumulate, pad, use_w, err, s); break;
        default: launch_fold<6>(g, img, eA, wt_rows, in, out, mode, scale, accumulate, pad, use_w, err, s); break;
    }
}

}  // namespace mlegs
