// Elementwise, banded-stencil and pointwise kernels of the hot path.
//
// Band operators restate mod_legops.f90 (DELSQH 76-133, MULXM 371-428,
// XXDX 680-748, DEL2 751-820, GRAD 1727-1786, PC2VEL 1789-1853,
// PC2VOR 1856-1919) on the FFF layout [m][n][k]; the truncation BANMUL
// applies (rows/columns beyond NN = NRCHOPS(m) dropped, mod_bandmat.f90:
// 1111-1153) is a mask on the column index.  Pointwise products restate
// VPRODSUB/VDOTPSUB (mod_legops.f90:2105-2130, 2207-2225) and the linear
// terms of CALC_BOUSSI_FORCE (mod_boussinesq.f90:385-391).
#include "mlegs_internal.h"

namespace mlegs {

thread_local int64_t* g_launch_counter = nullptr;

static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cmuli(double2 a, double s) { return make_double2(-a.y * s, a.x * s); }  // i s a

__device__ __forceinline__ int nrchops(const DevGrid& g, int m, int pad) {
    int nn = g.NRCHOP + pad - m;
    return nn < 0 ? 0 : nn;
}

// ---------------------------------------------------------------- fill/copy
__global__ void fill_kernel(double2* p, size_t n) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n) p[t] = make_double2(0.0, 0.0);
}
void k_fill(double2* p, size_t n, cudaStream_t s) {
    if (!n) return;
    fill_kernel<<<nblk(n, 256), 256, 0, s>>>(p, n);
    count_launch();
}
__global__ void copy_kernel(double2* d, const double2* a, size_t n) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n) d[t] = a[t];
}
void k_copy(double2* dst, const double2* src, size_t n, cudaStream_t s) {
    if (!n || dst == src) return;
    copy_kernel<<<nblk(n, 256), 256, 0, s>>>(dst, src, n);
    count_launch();
}

// dst = src over n entries and the field's LN slot (thread 0), in one launch.
__global__ void copy_ln_kernel(double2* d, const double2* a, size_t n, double* dln, const double* aln) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t == 0) *dln = *aln;
    if (t < n) d[t] = a[t];
}
void k_copy_ln(double2* dst, const double2* src, size_t n, double* dln, const double* sln, cudaStream_t s) {
    copy_ln_kernel<<<nblk(n > 0 ? n : 1, 256), 256, 0, s>>>(dst, src, n, dln, sln);
    count_launch();
}

// CHOPDO on FFF (mod_scalar3.f90:227-234): rows n >= NRCHOPS(m) -> 0.
__global__ void chopdo_fff_kernel(DevGrid g, double2* a, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    if (n >= nrchops(g, m, pad) || m >= g.NTCHOP) a[t] = make_double2(0.0, 0.0);
}
void k_chopdo_fff(const DevGrid& g, double2* a, int pad, cudaStream_t s) {
    size_t n = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    chopdo_fff_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, pad);
    count_launch();
}

// COPY0 of an FFF field in one pass: dst = src with the entries CHOPDO clears
// (rows n >= NRCHOPS(m) at pad, m >= NTCHOP) written as zero, LN copied.
__global__ void copy_chop_fff_kernel(DevGrid g, double2* d, const double2* a, double* dln, const double* aln,
                                     int pad) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t == 0) *dln = *aln;
    if (t >= total) return;
    const int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    const int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    d[t] = (n >= nrchops(g, m, pad) || m >= g.NTCHOP) ? make_double2(0.0, 0.0) : a[t];
}
void k_copy_chop_fff(const DevGrid& g, double2* dst, const double2* src, double* dln, const double* sln, int pad,
                     cudaStream_t s) {
    const size_t n = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    copy_chop_fff_kernel<<<nblk(n, 256), 256, 0, s>>>(g, dst, src, dln, sln, pad);
    count_launch();
}

// ------------------------------------------------------------ band operators
// DELSQH: b = -n(n+1)/L^2 a for n < NN; b(0,0,0) = LN/L^2/NORM(1,1).
__global__ void delsqh_kernel(DevGrid g, const double2* a, const double* ln, double2* b, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int k = (int)(t % g.NXCHOPDIM);
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    double2 v = make_double2(0.0, 0.0);
    if (n < nrchops(g, m, pad)) {
        int N = m + n;
        v = cscale(a[t], -(double)(N * (N + 1)) / g.ELL2);
    }
    if (m == 0 && n == 0 && k == 0) v = make_double2((ln ? *ln : 0.0) / g.ELL2 / g.norm0[0], 0.0);
    b[t] = v;
}
void k_delsqh(const DevGrid& g, const double2* a, const double* ln_a, double2* b, int pad, cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    delsqh_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, ln_a, b, pad);
    count_launch();
}

// IDELSQH (mod_legops.f90:136-241) without the log-term/far-field steps
// (done by k_ln / k_farfield_fix): a = -b L^2/(n(n+1)), a(n=0,m=0) = 0.
__global__ void idelsqh_kernel(DevGrid g, const double2* b, double2* a, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    double2 v = make_double2(0.0, 0.0);
    int N = m + n;
    if (n < nrchops(g, m, pad) && N != 0) v = cscale(b[t], -(g.ELL2 / (double)(N * (N + 1))));
    a[t] = v;
}
void k_idelsqh(const DevGrid& g, const double2* b, double2* a, int pad, cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    idelsqh_kernel<<<nblk(n, 256), 256, 0, s>>>(g, b, a, pad);
    count_launch();
}

// Tri-band apply: which 0 = XXDX (diag 0), 1 = MULXM (diag 1).
__global__ void band3_kernel(DevGrid g, const double2* a, double2* b, int which, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int k = (int)(t % g.NXCHOPDIM);
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    int nn = nrchops(g, m, pad);
    double2 v = make_double2(0.0, 0.0);
    if (n < nn) {
        const double* tb = (which == 0 ? g.xxdx : g.xm) + ((size_t)m * g.NB + n) * 2;
        const double2* col = a + ((size_t)m * g.NRCHOPDIM) * g.NXCHOPDIM + k;
        if (which == 1) v = col[(size_t)n * g.NXCHOPDIM];
        if (n >= 1) {
            double2 am = col[(size_t)(n - 1) * g.NXCHOPDIM];
            v.x += tb[0] * am.x;
            v.y += tb[0] * am.y;
        }
        if (n + 1 < nn) {
            double2 ap = col[(size_t)(n + 1) * g.NXCHOPDIM];
            v.x += tb[1] * ap.x;
            v.y += tb[1] * ap.y;
        }
    }
    b[t] = v;
}
void k_band3(const DevGrid& g, const double2* a, double2* b, int which, int pad, cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    band3_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, b, which, pad);
    count_launch();
}

// DEL2 without the log-term rows: b = DEL2H_m a - k^2 a (penta band).
__global__ void del2_kernel(DevGrid g, const double2* a, double2* b, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int k = (int)(t % g.NXCHOPDIM);
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    int nn = nrchops(g, m, pad);
    double2 v = make_double2(0.0, 0.0);
    if (n < nn) {
        const double* tb = g.del2h + ((size_t)m * g.NB + n) * 5;
        const double2* col = a + ((size_t)m * g.NRCHOPDIM) * g.NXCHOPDIM + k;
        for (int d = 0; d < 5; ++d) {
            int j = n + d - 2;
            if (j < 0 || j >= nn) continue;
            double2 aj = col[(size_t)j * g.NXCHOPDIM];
            v.x += tb[d] * aj.x;
            v.y += tb[d] * aj.y;
        }
        double k2 = g.ak[k] * g.ak[k];
        double2 an = col[(size_t)n * g.NXCHOPDIM];
        v.x -= k2 * an.x;
        v.y -= k2 * an.y;
    }
    b[t] = v;
}
void k_del2(const DevGrid& g, const double2* a, double2* b, int pad, cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    del2_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, b, pad);
    count_launch();
}

// Log-term rows of the (m,k) = (0,0) line:
//  which 0 (XXDX, 742-745):  b0 += LN/N0, b1 += LN/N1
//  which 1 (DEL2, 813-817):  b0 += 4/3 LN/L2/N0, b1 -= 2 LN/L2/N1, b2 += 2/3 LN/L2/N2
//  which 2 (IHELM, 1249-1255): b0 -= LN 4/3/L2/N0, b1 -= LN (-2/N1/L2), b2 -= LN (2/3/N2/L2)
// coef multiplies LN first (used for the IHELM LN = -B%LN/ALP form).
__global__ void logterm_kernel(DevGrid g, double2* b, const double* lnp, int which, double coef) {
    double ln = (*lnp) * coef;
    const double* n0 = g.norm0;
    size_t st = g.NXCHOPDIM;  // row stride of the (m=0) column
    if (which == 0) {
        b[0].x += ln / n0[0];
        b[st].x += ln / n0[1];
    } else if (which == 1) {
        b[0].x += 4.0 / 3 * ln / g.ELL2 / n0[0];
        b[st].x -= 2.0 * ln / g.ELL2 / n0[1];
        b[2 * st].x += 2.0 / 3 * ln / g.ELL2 / n0[2];
    } else {
        b[0].x -= ln * (4.0 / 3 / g.ELL2) / n0[0];
        b[st].x -= ln * (-2 / n0[1] / g.ELL2);
        b[2 * st].x -= ln * (+2.0 / 3 / n0[2] / g.ELL2);
    }
}
void k_logterm_rows(const DevGrid& g, double2* b, const double* ln, int which, double coef, cudaStream_t s) {
    logterm_kernel<<<1, 1, 0, s>>>(g, b, ln, which, coef);
    count_launch();
}

// m/k combinations of PC2VEL, PC2VOR and GRAD (rows n < NN, zero beyond):
//  op 0: i m x + i k y    op 1: -y - m k x    op 2: -i m x + i k y
//  op 3:  y - k m x       op 4: i m x         op 5: i k x          op 6: -x
//  and the conjugate factors of their transposes:
//  op 7: -i m x           op 8: -i k x        op 9: m k x          op 10: -m k x
__global__ void mk_kernel(DevGrid g, int op, const double2* x, const double2* y, double2* out, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int k = (int)(t % g.NXCHOPDIM);
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    double2 v = make_double2(0.0, 0.0);
    if (n < nrchops(g, m, pad)) {
        double mv = (double)m, kv = g.ak[k];
        double2 xv = x ? x[t] : make_double2(0.0, 0.0);
        double2 yv = y ? y[t] : make_double2(0.0, 0.0);
        switch (op) {
            case 0: v = cadd(cmuli(xv, mv), cmuli(yv, kv)); break;
            case 1: v = make_double2(-yv.x - (mv * kv) * xv.x, -yv.y - (mv * kv) * xv.y); break;
            case 2: v = cadd(cmuli(xv, -mv), cmuli(yv, kv)); break;
            case 3: v = make_double2(yv.x - (kv * mv) * xv.x, yv.y - (kv * mv) * xv.y); break;
            case 4: v = cmuli(xv, mv); break;
            case 5: v = cmuli(xv, kv); break;
            case 7: v = cmuli(xv, -mv); break;
            case 8: v = cmuli(xv, -kv); break;
            case 9: v = cscale(xv, mv * kv); break;
            case 10: v = cscale(xv, -(mv * kv)); break;
            default: v = make_double2(-xv.x, -xv.y); break;
        }
    }
    out[t] = v;
}
void k_mk_combine(const DevGrid& g, int op, const double2* x, const double2* y, double2* out, int pad,
                  cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    mk_kernel<<<nblk(n, 256), 256, 0, s>>>(g, op, x, y, out, pad);
    count_launch();
}

// a(n=0, m=0, k) -= sum_{n < nr_sum} AT1(n) a(n, 0, k) / AT1(0)   (CALCAT1 fix);
// by_pf: divided by TFM%PF(1,1,1) instead, as IHELMP writes it (mod_legops.f90:1586).
// One warp per k: lanes stride over n, shuffle reduction.
__global__ void farfield_kernel(DevGrid g, double2* a, int nr_sum, int by_pf) {
    int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (k >= g.NXCHOPDIM) return;
    double sx = 0.0, sy = 0.0;
    for (int n = lane; n < nr_sum; n += 32) {
        double2 v = a[(size_t)n * g.NXCHOPDIM + k];
        sx += g.at1[n] * v.x;
        sy += g.at1[n] * v.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (lane == 0) {
        const double den = by_pf ? g.pf[0] : g.at1[0];
        a[k].x -= sx / den;
        a[k].y -= sy / den;
    }
}
void k_farfield_fix(const DevGrid& g, double2* a, int nr_sum, cudaStream_t s, int by_pf) {
    farfield_kernel<<<nblk(g.NXCHOPDIM, 8), 256, 0, s>>>(g, a, nr_sum, by_pf);
    count_launch();
}

// VEL2PLN (mod_legops.f90:2277-2339) on the (m,k) = (0,0) radial line of a PFF
// field.  mode 0: PSI%LN <- extracted value; mode 1: PSI%LN <- ln.
// VEL2PLN's far-field value (mod_legops.f90:2277-2339) is a fixed linear
// functional of RUP's (m, k) = (0, 0) line:
//   PLN = -(1/2) sum_{n < NRCHOP} EXPLOG0(n) sum_i F_n(i) PF_0(n, i),
// F_n the even (n even) or odd fold of the PFF line times the Gauss weights.
// Its coefficients are formed once per context, for the PFF line (Lpff, NR
// entries) and for the FFF column whose RTRAN(+1) image that line is (Lfff,
// NRCHOP entries; the fold of the image is twice its parity half, so
// Lfff(n') = -sum_{n = n' mod 2} EXPLOG0(n) sum_i w_i PF_0(n, i) PF_0(n', i)).
// Each call is then one dot product.
__global__ void vel2pln_coef_kernel(DevGrid g, const double* explog0, int nn, double* Lpff, double* Lfff) {
    const double* pf = g.pf;  // m = 0 slice: [n][i]
    for (int i = threadIdx.x; i < g.NRH; i += blockDim.x) {
        double se = 0.0, so = 0.0;
        for (int n = 0; n < nn; ++n) {
            const double v = explog0[n] * pf[(size_t)n * g.NRH + i];
            if (n % 2 == 0) se += v;
            else so += v;
        }
        Lpff[i] = -0.5 * g.w[i] * (se + so);
        Lpff[g.NR - 1 - i] = -0.5 * g.w[i] * (se - so);
    }
    for (int np = threadIdx.x; np < nn; np += blockDim.x) {
        double acc = 0.0;
        for (int n = np % 2; n < nn; n += 2) {
            double gram = 0.0;
            for (int i = 0; i < g.NRH; ++i) gram += g.w[i] * pf[(size_t)n * g.NRH + i] * pf[(size_t)np * g.NRH + i];
            acc += explog0[n] * gram;
        }
        Lfff[np] = -acc;
    }
}
void k_vel2pln_coef(const DevGrid& g, const double* explog0, int nn, double* Lpff, double* Lfff, cudaStream_t s) {
    vel2pln_coef_kernel<<<1, 256, 0, s>>>(g, explog0, nn, Lpff, Lfff);
    count_launch();
}

// Block-wide sum of sum_j L[j] line[j * st].x over j < n (one block of 256).
__device__ double vel2pln_dot(const double* L, const double2* line, size_t st, int n, double* part) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) acc += L[j] * line[(size_t)j * st].x;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    double tot = 0.0;
    for (int w = 0; w < nw; ++w) tot += part[w];
    return tot;
}

__global__ void vel2pln_kernel(DevGrid g, double2* rup, double* psi_ln, int mode, double ln_in, const double* Lpff,
                               double* zero_ln) {
    __shared__ double part[8];
    const size_t st = g.NXCHOPDIM;  // PFF row stride for m = 0 ([0][r][k])
    const double pln = vel2pln_dot(Lpff, rup, st, g.NR, part);
    const double* pf = g.pf;
    for (int i = threadIdx.x; i < g.NRH; i += blockDim.x) {
        double e2 = -pf[i] * pln / g.norm0[0];
        double o2 = -pf[(size_t)g.NRH + i] * pln / g.norm0[1];
        rup[(size_t)i * st].x -= (e2 + o2);
        rup[(size_t)(g.NR - 1 - i) * st].x -= (e2 - o2);
    }
    if (threadIdx.x == 0) {
        *psi_ln = (mode == 1) ? ln_in : pln;
        if (zero_ln) *zero_ln = 0.0;
    }
}
void launch_vel2pln(const DevGrid& g, double2* rup_pff, double* psi_ln, int mode, double ln, const double* Lpff,
                    cudaStream_t s, double* zero_ln) {
    vel2pln_kernel<<<1, 256, 0, s>>>(g, rup_pff, psi_ln, mode, ln, Lpff, zero_ln);
    count_launch();
}

// VEL2PLN from RUP's FFF (0, 0) column; the subtraction of PLN times the
// n = 0, 1 functions from the PFF line is applied to the FFF column instead
// (rows 0 and 1 += PLN / NORM), the same change of the RTRAN(+1) image.
__global__ void vel2pln_fff_kernel(DevGrid g, double2* rup, double* psi_ln, const double* Lfff, double* zero_ln) {
    __shared__ double part[8];
    const size_t st = g.NXCHOPDIM;  // FFF row stride of the (0, 0) column
    const double pln = vel2pln_dot(Lfff, rup, st, g.NRCHOP, part);
    if (threadIdx.x == 0) {
        rup[0].x += pln / g.norm0[0];
        rup[st].x += pln / g.norm0[1];
        *psi_ln = pln;
        if (zero_ln) *zero_ln = 0.0;
    }
}
void launch_vel2pln_fff(const DevGrid& g, double2* rup_fff, double* psi_ln, const double* Lfff, cudaStream_t s,
                        double* zero_ln) {
    vel2pln_fff_kernel<<<1, 256, 0, s>>>(g, rup_fff, psi_ln, Lfff, zero_ln);
    count_launch();
}

// PRODCT_MK_ALLK / L2NORM_MK_ALLK (mod_scalar3.f90:470-526, 750-806) before
// their m = 0 halving: per (m, k) of PFF fields,
//   mode 0: scale * sum_{r < NR} Re(A conj B)(r) w_r
//   mode 1: scale * sum_{r < NR} |A(r)|^2 / (1 - x_r)^2 w_r
// summed in r order like DOT_PRODUCT.  out: [m][k], NTCHOPDIM x NXCHOPDIM.
__global__ void prodct_mk_kernel(DevGrid g, const double2* A, const double2* B, int mode, double scale,
                                 double* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.NTCHOPDIM * g.NXCHOPDIM) return;
    const int k = t % g.NXCHOPDIM, m = t / g.NXCHOPDIM;
    const size_t st = g.NXCHOPDIM, base = (size_t)m * g.NR * st + k;
    double acc = 0.0;
    if (mode == 0) {
        for (int r = 0; r < g.NR; ++r) {
            const double2 a = A[base + (size_t)r * st], b = B[base + (size_t)r * st];
            acc += (a.x * b.x + a.y * b.y) * g.w[r];
        }
    } else {
        for (int r = 0; r < g.NR; ++r) {
            const double2 a = A[base + (size_t)r * st];
            const double om = 1.0 - g.x[r];
            acc += (a.x * a.x + a.y * a.y) / (om * om) * g.w[r];
        }
    }
    out[t] = scale * acc;
}
void k_prodct_mk(const DevGrid& g, const double2* A, const double2* B, int mode, double scale, double* out,
                 cudaStream_t s) {
    const int n = g.NTCHOPDIM * g.NXCHOPDIM;
    prodct_mk_kernel<<<(n + 127) / 128, 128, 0, s>>>(g, A, B, mode, scale, out);
    count_launch();
}

// ------------------------------------------------------------ pointwise PPP
// VPRODSUB + VDOTPSUB (+ linear terms of CALC_BOUSSI_FORCE when linear = 1).
__global__ void force_pointwise_kernel(int nr, int plane, const double* rad, double2* rur, double2* rup,
                                       double2* uz, double2* ror, double2* rop, double2* oz,
                                       const double2* rbr, const double2* rbp, const double2* bz,
                                       double2* bn, const double2* bphys, double omega, double bv0,
                                       int linear) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)nr * plane;
    if (t >= total) return;
    int r = (int)(t / plane);
    double rr = rad[r];
    double r2 = rr * rr;
    double2 a1 = rur[t], a2 = rup[t], a3 = uz[t];
    double2 b1 = ror[t], b2 = rop[t], b3 = oz[t];
    double2 c1 = rbr[t], c2 = rbp[t], c3 = bz[t];
    double2 nr_ = make_double2(a2.x * b3.x - a3.x * b2.x, a2.y * b3.y - a3.y * b2.y);
    double2 np_ = make_double2(a3.x * b1.x - a1.x * b3.x, a3.y * b1.y - a1.y * b3.y);
    double2 nz_ = make_double2((a1.x * b2.x - a2.x * b1.x) / r2, (a1.y * b2.y - a2.y * b1.y) / r2);
    double2 d = make_double2((a1.x * c1.x + a2.x * c2.x) / r2 + a3.x * c3.x,
                             (a1.y * c1.y + a2.y * c2.y) / r2 + a3.y * c3.y);
    double2 bnv = make_double2(-d.x, -d.y);
    if (linear) {
        double2 bp = bphys[t];
        nr_.x += 2 * omega * a2.x;
        nr_.y += 2 * omega * a2.y;
        np_.x -= 2 * omega * a1.x;
        np_.y -= 2 * omega * a1.y;
        nz_.x -= bp.x;
        nz_.y -= bp.y;
        double n2 = bv0 * bv0;
        bnv.x += n2 * a3.x;
        bnv.y += n2 * a3.y;
    }
    ror[t] = nr_;
    rop[t] = np_;
    oz[t] = nz_;
    bn[t] = bnv;
}
void k_force_pointwise(const DevGrid& g, double2* rur, double2* rup, double2* uz, double2* ror,
                       double2* rop, double2* oz, const double2* rbr, const double2* rbp,
                       const double2* bz, double2* bn, const double2* bphys, double omega,
                       double bv0, int linear, cudaStream_t s) {
    size_t n = (size_t)g.NR * g.NX * g.NTH;
    force_pointwise_kernel<<<nblk(n, 256), 256, 0, s>>>(g.NR, g.NX * g.NTH, g.r, rur, rup, uz, ror,
                                                        rop, oz, rbr, rbp, bz, bn, bphys, omega, bv0,
                                                        linear);
    count_launch();
}

// ------------------------------------------------------------ FFF updates
// y = c*y + a*x1 + b*x2  (x2 may be null)
__global__ void axpby_kernel(double2* y, double a, const double2* x1, double b, const double2* x2,
                             double c, size_t n) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    double2 v = make_double2(0.0, 0.0);
    if (c != 0.0) v = cscale(y[t], c);
    if (x1) {
        double2 u = x1[t];
        v.x += a * u.x;
        v.y += a * u.y;
    }
    if (x2) {
        double2 u = x2[t];
        v.x += b * u.x;
        v.y += b * u.y;
    }
    y[t] = v;
}
void k_axpby(double2* y, double a, const double2* x1, double b, const double2* x2, double c, size_t n,
             cudaStream_t s) {
    axpby_kernel<<<nblk(n, 256), 256, 0, s>>>(y, a, x1, b, x2, c, n);
    count_launch();
}
// k_axpby and k_ln_axpby in one launch: the field's entries as axpby_kernel,
// its LN slot (thread 0) as ln_axpby_kernel.
__global__ void axpby_ln_kernel(double2* y, double a, const double2* x1, double b, const double2* x2, double c,
                                size_t n, double* yl, double la, const double* l1, double lb, const double* l2,
                                double lc) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t == 0) {
        double v = (lc != 0.0) ? lc * (*yl) : 0.0;
        if (l1) v += la * (*l1);
        if (l2) v += lb * (*l2);
        *yl = v;
    }
    if (t >= n) return;
    double2 v = make_double2(0.0, 0.0);
    if (c != 0.0) v = cscale(y[t], c);
    if (x1) {
        v.x += a * x1[t].x;
        v.y += a * x1[t].y;
    }
    if (x2) {
        v.x += b * x2[t].x;
        v.y += b * x2[t].y;
    }
    y[t] = v;
}
void k_axpby_ln(double2* y, double a, const double2* x1, double b, const double2* x2, double c, size_t n, double* yl,
                double la, const double* l1, double lb, const double* l2, double lc, cudaStream_t s) {
    axpby_ln_kernel<<<nblk(n > 0 ? n : 1, 256), 256, 0, s>>>(y, a, x1, b, x2, c, n, yl, la, l1, lb, l2, lc);
    count_launch();
}
__global__ void ln_axpby_kernel(double* y, double a, const double* x1, double b, const double* x2, double c) {
    double v = (c != 0.0) ? c * (*y) : 0.0;
    if (x1) v += a * (*x1);
    if (x2) v += b * (*x2);
    *y = v;
}
void k_ln_axpby(double* y, double a, const double* x1, double b, const double* x2, double c, cudaStream_t s) {
    ln_axpby_kernel<<<1, 1, 0, s>>>(y, a, x1, b, x2, c);
    count_launch();
}
__global__ void ln_set_kernel(double* y, double v) { *y = v; }
void k_ln_set(double* y, double v, cudaStream_t s) {
    ln_set_kernel<<<1, 1, 0, s>>>(y, v);
    count_launch();
}
__global__ void ln_copy_kernel(double* y, const double* x, double sc) { *y = (*x) * sc; }
void k_ln_copy(double* y, const double* x, double scale, cudaStream_t s) {
    ln_copy_kernel<<<1, 1, 0, s>>>(y, x, scale);
    count_launch();
}

// ETD update per FFF coefficient (CALC_BOUSSI_ETDFE_SUB 948-1047 with ab2 = 0,
// CALC_BOUSSI_ETDAB_SUB 1050-1139 with ab2 = 1).  E, NL: real parts, row-major 4x4.
__global__ void etd_kernel(DevGrid g, const double* Em, const double* Nm, double dt, int ab2,
                           double2* rur, double2* rup, double2* uz, double2* b, const double2* rnr,
                           const double2* rnp, const double2* nz, const double2* nb, const double2* hr,
                           const double2* hp, const double2* hz, const double2* onr,
                           const double2* onp, const double2* onz, const double2* onb) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int k = (int)(t % g.NXCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    double E[16], N[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        E[q] = Em[q];
        N[q] = Nm[q];
    }
    if (k == 0) {
        for (int q = 0; q < 4; ++q) {
            E[q] = 0.0;
            E[4 + q] = 0.0;
            N[q] = 0.0;
            N[4 + q] = 0.0;
        }
        E[0] = 1.0;
        E[5] = 1.0;
        N[0] = dt;
        N[5] = dt;
    }
    double2 ev[4], av[4];
    if (ab2) {
        double notm0 = (m == 0) ? 0.0 : 1.0, notk0 = (k == 0) ? 0.0 : 1.0;
        ev[0] = csub(rur[t], hr[t]);
        ev[1] = csub(rup[t], cscale(hp[t], notm0));
        ev[2] = csub(uz[t], cscale(hz[t], notk0));
        ev[3] = b[t];
        av[0] = csub(cscale(rnr[t], 1.5), cscale(onr[t], 0.5));
        av[1] = csub(cscale(rnp[t], 1.5), cscale(onp[t], 0.5));
        av[2] = csub(cscale(nz[t], 1.5), cscale(onz[t], 0.5));
        av[3] = csub(cscale(nb[t], 1.5), cscale(onb[t], 0.5));
    } else {
        ev[0] = rur[t];
        ev[1] = rup[t];
        ev[2] = uz[t];
        ev[3] = b[t];
        av[0] = rnr[t];
        av[1] = rnp[t];
        av[2] = nz[t];
        av[3] = nb[t];
    }
    double2 cv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double2 a = make_double2(0.0, 0.0), c = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a.x += E[i * 4 + j] * ev[j].x;
            a.y += E[i * 4 + j] * ev[j].y;
            c.x += N[i * 4 + j] * av[j].x;
            c.y += N[i * 4 + j] * av[j].y;
        }
        cv[i] = cadd(a, c);
    }
    rur[t] = cv[0];
    rup[t] = cv[1];
    uz[t] = cv[2];
    b[t] = cv[3];
}
void k_etd(const DevGrid& g, const double* E, const double* NL, double dt, int ab2, double2* rur,
           double2* rup, double2* uz, double2* b, const double2* rnr, const double2* rnp,
           const double2* nz, const double2* nb, const double2* hr, const double2* hp, const double2* hz,
           const double2* onr, const double2* onp, const double2* onz, const double2* onb, cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    etd_kernel<<<nblk(n, 256), 256, 0, s>>>(g, E, NL, dt, ab2, rur, rup, uz, b, rnr, rnp, nz, nb, hr, hp,
                                            hz, onr, onp, onz, onb);
    count_launch();
}

// HYPERV3 / CALC_BOUSSI_ETD_HYPERV filter (mod_march.f90:3521-3560, 1388-1408)
// followed by CHOPDO at pad.  hr: [NRCHOP][NTCHOPDIM] (column-major as HYPER_R).
__global__ void hyperv_kernel(DevGrid g, double2* a, const double* hr, const double* ht, const double* hx,
                              double tf, int pad) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return;
    int k = (int)(t % g.NXCHOPDIM);
    int n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    int m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    if (n < nrchops(g, m, pad)) {
        double f = hr[(size_t)m * g.NRCHOP + n] * ht[m] * hx[k];
        if (tf != 1.0) f = pow(f, tf);
        a[t] = cscale(a[t], f);
    } else {
        a[t] = make_double2(0.0, 0.0);
    }
}
void k_hyperv(const DevGrid& g, double2* a, const double* hr, const double* ht, const double* hx, double tf,
              int pad, cudaStream_t s) {
    size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    hyperv_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, hr, ht, hx, tf, pad);
    count_launch();
}

__global__ void finite_kernel(const double2* a, size_t n, int* flag) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    double2 v = a[t];
    if (!isfinite(v.x) || !isfinite(v.y)) atomicOr(flag, 1);
}
void k_finite(const double2* a, size_t n, int* flag, cudaStream_t s) {
    finite_kernel<<<nblk(n, 256), 256, 0, s>>>(a, n, flag);
    count_launch();
}

// ------------------------------------------------------ layout conversions
// ref index (Fortran column-major) -> device index, or -1 for padding.
__device__ __forceinline__ long long ref_to_dev(const DevGrid& g, int space, size_t t) {
    int ndimr = g.NR + 3, ndimth = g.NTH + 1;
    if (space == MLEGS_FFF) {
        int n = (int)(t % g.NRCHOPDIM);
        int m = (int)((t / g.NRCHOPDIM) % g.NTCHOPDIM);
        int k = (int)(t / ((size_t)g.NRCHOPDIM * g.NTCHOPDIM));
        return ((long long)m * g.NRCHOPDIM + n) * g.NXCHOPDIM + k;
    }
    if (space == MLEGS_PFF) {
        int r = (int)(t % ndimr);
        int m = (int)((t / ndimr) % g.NTCHOPDIM);
        int k = (int)(t / ((size_t)ndimr * g.NTCHOPDIM));
        if (r >= g.NR) return -1;
        return ((long long)m * g.NR + r) * g.NXCHOPDIM + k;
    }
    int r = (int)(t % ndimr);
    int j = (int)((t / ndimr) % ndimth);
    int z = (int)(t / ((size_t)ndimr * ndimth));
    if (r >= g.NR) return -1;
    if (space == MLEGS_PFP) {
        if (j >= g.NTCHOPDIM) return -1;
        return ((long long)r * g.NX + z) * g.NTCHOPDIM + j;
    }
    if (j >= g.NTH) return -1;
    return ((long long)r * g.NX + z) * g.NTH + j;
}
__global__ void from_ref_kernel(DevGrid g, int space, const double2* ref, double2* dev, size_t n) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    long long d = ref_to_dev(g, space, t);
    if (d >= 0) dev[d] = ref[t];
}
__global__ void to_ref_kernel(DevGrid g, int space, const double2* dev, double2* ref, size_t n) {
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    long long d = ref_to_dev(g, space, t);
    ref[t] = (d >= 0) ? dev[d] : make_double2(0.0, 0.0);
}
static size_t ref_elems(const DevGrid& g, int space) {
    size_t ndimr = g.NR + 3, ndimth = g.NTH + 1;
    if (space == MLEGS_FFF) return (size_t)g.NRCHOPDIM * g.NTCHOPDIM * g.NXCHOPDIM;
    if (space == MLEGS_PFF) return ndimr * g.NTCHOPDIM * g.NXCHOPDIM;
    return ndimr * ndimth * g.NX;
}
void k_from_ref(const DevGrid& g, int space, const double2* ref, double2* dev, cudaStream_t s) {
    size_t n = ref_elems(g, space);
    from_ref_kernel<<<nblk(n, 256), 256, 0, s>>>(g, space, ref, dev, n);
    count_launch();
}
void k_to_ref(const DevGrid& g, int space, const double2* dev, double2* ref, cudaStream_t s) {
    size_t n = ref_elems(g, space);
    to_ref_kernel<<<nblk(n, 256), 256, 0, s>>>(g, space, dev, ref, n);
    count_launch();
}


// ---------------------------------------------------------------- fused GRAD, PC2VEL, PC2VOR
// One thread per FFF element evaluates the whole operator chain as a stencil
// in n of the (m, k) column, with every intermediate truncated to rows
// n < NRCHOPS(m) exactly as the chained operators are, so no intermediate
// field is written:
//   GRAD   (mod_legops.f90:1727-1786): rr = XXDX(a), rp = i m a, gz = i k a
//   PC2VEL (1789-1853): rur = i m psi + i k XXDX(chi), rup = -XXDX(psi) - m k chi,
//                       uz = -XM XM DELSQH(chi)
//   PC2VOR (1856-1919): oz' = DEL2(chi), ror = -i m oz' + i k XXDX(psi),
//                       rop = XXDX(oz') - k m psi, oz = -XM XM DELSQH(psi)
// with the log-term rows of XXDX (742-745), DEL2 (813-817) and DELSQH
// (128-130) at (m, k) = (0, 0).
namespace {

struct Col {
    const double2* p;  // row 0 of the (m, k) column
    size_t st;         // row stride (NXCHOPDIM)
    int nn;            // rows kept, NRCHOPS(m)
    __device__ __forceinline__ double2 at(int j) const {
        return (j >= 0 && j < nn) ? p[(size_t)j * st] : make_double2(0.0, 0.0);
    }
};

// XXDX of column c at row n (zero outside [0, nn)); log rows when ln is given at (0, 0)
__device__ __forceinline__ double2 xxdx_row(const DevGrid& g, int m, int k, const Col& c, int n, double ln) {
    if (n < 0 || n >= c.nn) return make_double2(0.0, 0.0);
    const double* tb = g.xxdx + ((size_t)m * g.NB + n) * 2;
    double2 v = make_double2(0.0, 0.0);
    if (n >= 1) {
        const double2 am = c.p[(size_t)(n - 1) * c.st];
        v.x += tb[0] * am.x;
        v.y += tb[0] * am.y;
    }
    if (n + 1 < c.nn) {
        const double2 ap = c.p[(size_t)(n + 1) * c.st];
        v.x += tb[1] * ap.x;
        v.y += tb[1] * ap.y;
    }
    if (m == 0 && k == 0) {
        if (n == 0) v.x += ln / g.norm0[0];
        else if (n == 1) v.x += ln / g.norm0[1];
    }
    return v;
}

// DELSQH of column c at row n (zero outside [0, nn)), log entry at (0, 0, 0)
__device__ __forceinline__ double2 delsqh_row(const DevGrid& g, int m, int k, const Col& c, int n, double ln) {
    if (m == 0 && n == 0 && k == 0) return make_double2(ln / g.ELL2 / g.norm0[0], 0.0);
    if (n < 0 || n >= c.nn) return make_double2(0.0, 0.0);
    const int N = m + n;
    return cscale(c.p[(size_t)n * c.st], -(double)(N * (N + 1)) / g.ELL2);
}

// DEL2 of column c at row n (zero outside [0, nn)), log rows at (0, 0)
__device__ __forceinline__ double2 del2_row(const DevGrid& g, int m, int k, const Col& c, int n, double ln) {
    if (n < 0 || n >= c.nn) return make_double2(0.0, 0.0);
    const double* tb = g.del2h + ((size_t)m * g.NB + n) * 5;
    double2 v = make_double2(0.0, 0.0);
    for (int d = 0; d < 5; ++d) {
        const int j = n + d - 2;
        if (j < 0 || j >= c.nn) continue;
        const double2 aj = c.p[(size_t)j * c.st];
        v.x += tb[d] * aj.x;
        v.y += tb[d] * aj.y;
    }
    const double k2 = g.ak[k] * g.ak[k];
    const double2 an = c.p[(size_t)n * c.st];
    v.x -= k2 * an.x;
    v.y -= k2 * an.y;
    if (m == 0 && k == 0) {
        if (n == 0) v.x += 4.0 / 3 * ln / g.ELL2 / g.norm0[0];
        else if (n == 1) v.x -= 2.0 * ln / g.ELL2 / g.norm0[1];
        else if (n == 2) v.x += 2.0 / 3 * ln / g.ELL2 / g.norm0[2];
    }
    return v;
}

// -XM XM DELSQH(c) at row n
__device__ __forceinline__ double2 neg_xm2_delsqh(const DevGrid& g, int m, int k, const Col& c, int n, double ln) {
    const double* xm = g.xm + (size_t)m * g.NB * 2;
    double2 d[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) d[q] = delsqh_row(g, m, k, c, n - 2 + q, ln);
    double2 w[3];  // XM of d at rows n-1, n, n+1
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int j = n - 1 + q;
        w[q] = make_double2(0.0, 0.0);
        if (j < 0 || j >= c.nn) continue;
        double2 v = d[q + 1];
        if (j >= 1) {
            v.x += xm[j * 2] * d[q].x;
            v.y += xm[j * 2] * d[q].y;
        }
        if (j + 1 < c.nn) {
            v.x += xm[j * 2 + 1] * d[q + 2].x;
            v.y += xm[j * 2 + 1] * d[q + 2].y;
        }
        w[q] = v;
    }
    double2 v = w[1];
    if (n >= 1) {
        v.x += xm[n * 2] * w[0].x;
        v.y += xm[n * 2] * w[0].y;
    }
    if (n + 1 < c.nn) {
        v.x += xm[n * 2 + 1] * w[2].x;
        v.y += xm[n * 2 + 1] * w[2].y;
    }
    return make_double2(-v.x, -v.y);
}

__device__ __forceinline__ bool fff_index(const DevGrid& g, size_t t, int& m, int& n, int& k) {
    const size_t total = (size_t)g.NTCHOPDIM * g.NRCHOPDIM * g.NXCHOPDIM;
    if (t >= total) return false;
    k = (int)(t % g.NXCHOPDIM);
    n = (int)((t / g.NXCHOPDIM) % g.NRCHOPDIM);
    m = (int)(t / ((size_t)g.NXCHOPDIM * g.NRCHOPDIM));
    return true;
}

__device__ __forceinline__ Col column(const DevGrid& g, const double2* a, int m, int k, int pad) {
    Col c;
    c.p = a + (size_t)m * g.NRCHOPDIM * g.NXCHOPDIM + k;
    c.st = g.NXCHOPDIM;
    c.nn = nrchops(g, m, pad);
    return c;
}

}  // namespace

__global__ void grad_fused_kernel(DevGrid g, const double2* a, const double* ln, double2* rr, double2* rp,
                                  double2* gz, int pad) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int m, n, k;
    if (!fff_index(g, t, m, n, k)) return;
    const Col c = column(g, a, m, k, pad);
    double2 v0 = make_double2(0.0, 0.0), v1 = v0, v2 = v0;
    if (n < c.nn) {
        const double2 an = c.p[(size_t)n * c.st];
        v0 = xxdx_row(g, m, k, c, n, ln ? *ln : 0.0);
        v1 = cmuli(an, (double)m);
        v2 = cmuli(an, g.ak[k]);
    }
    rr[t] = v0;
    rp[t] = v1;
    gz[t] = v2;
}

// sub = 1: the outputs are decremented by the velocity instead of set to it
__global__ void pc2vel_fused_kernel(DevGrid g, const double2* psi, const double* psi_ln, const double2* chi,
                                    const double* chi_ln, double2* rur, double2* rup, double2* uz, int pad, int sub,
                                    double* zl0, double* zl1, double* zl2) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int m, n, k;
    if (!fff_index(g, t, m, n, k)) return;
    // the outputs' LN slots (PC2VEL results carry no log term); read by no thread here
    if (t < 3 && zl0) *(t == 0 ? zl0 : (t == 1 ? zl1 : zl2)) = 0.0;
    const Col cp = column(g, psi, m, k, pad), cc = column(g, chi, m, k, pad);
    double2 v0 = make_double2(0.0, 0.0), v1 = v0, v2 = v0;
    if (n < cp.nn) {
        const double lp = psi_ln ? *psi_ln : 0.0, lc = chi_ln ? *chi_ln : 0.0;
        const double mv = (double)m, kv = g.ak[k];
        const double2 ps = cp.p[(size_t)n * cp.st], ch = cc.p[(size_t)n * cc.st];
        const double2 xc = xxdx_row(g, m, k, cc, n, lc);
        const double2 xp = xxdx_row(g, m, k, cp, n, lp);
        v0 = cadd(cmuli(ps, mv), cmuli(xc, kv));
        v1 = make_double2(-xp.x - (mv * kv) * ch.x, -xp.y - (mv * kv) * ch.y);
        v2 = neg_xm2_delsqh(g, m, k, cc, n, lc);
    }
    if (sub) {
        v0 = csub(rur[t], v0);
        v1 = csub(rup[t], v1);
        v2 = csub(uz[t], v2);
    }
    rur[t] = v0;
    rup[t] = v1;
    uz[t] = v2;
}

__global__ void pc2vor_fused_kernel(DevGrid g, const double2* psi, const double* psi_ln, const double2* chi,
                                    const double* chi_ln, double2* ror, double2* rop, double2* oz, int pad) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int m, n, k;
    if (!fff_index(g, t, m, n, k)) return;
    const Col cp = column(g, psi, m, k, pad), cc = column(g, chi, m, k, pad);
    double2 v0 = make_double2(0.0, 0.0), v1 = v0, v2 = v0;
    if (n < cp.nn) {
        const double lp = psi_ln ? *psi_ln : 0.0, lc = chi_ln ? *chi_ln : 0.0;
        const double mv = (double)m, kv = g.ak[k];
        const double2 ps = cp.p[(size_t)n * cp.st];
        // oz' = DEL2(chi) at rows n-1, n, n+1; XXDX(oz') has no log rows (oz'%LN = 0)
        const double2 dm = del2_row(g, m, k, cc, n - 1, lc), d0 = del2_row(g, m, k, cc, n, lc),
                      dp = del2_row(g, m, k, cc, n + 1, lc);
        const double* tb = g.xxdx + ((size_t)m * g.NB + n) * 2;
        double2 xo = make_double2(0.0, 0.0);
        if (n >= 1) {
            xo.x += tb[0] * dm.x;
            xo.y += tb[0] * dm.y;
        }
        if (n + 1 < cp.nn) {
            xo.x += tb[1] * dp.x;
            xo.y += tb[1] * dp.y;
        }
        const double2 xp = xxdx_row(g, m, k, cp, n, lp);
        v0 = cadd(cmuli(d0, -mv), cmuli(xp, kv));
        v1 = make_double2(xo.x - (kv * mv) * ps.x, xo.y - (kv * mv) * ps.y);
        v2 = neg_xm2_delsqh(g, m, k, cp, n, lp);
    }
    ror[t] = v0;
    rop[t] = v1;
    oz[t] = v2;
}

// The coefficient update of STEP_BOUSSI_ETDAB_CN (mod_march.f90:811-901) from
// the projected nonlinear terms to the new state, in one pass per FFF entry:
//   HYPERV of the nonlinear terms (1352-1416, at TF = 1, chopped at pad 0;
//   given as ROR, ROP, OZ, or formed here as PC2VEL of the projected PSI_N,
//   CHI_N, the last step of CALC_BOUSSI_NONLIN),
//   PC2VEL(PSI, CHI) at pad 3 (mod_legops.f90:1789-1853),
//   CALC_BOUSSI_ETDAB_SUB (1050-1139), HYPERV of the updated (RUR, RUP, UZ, B),
//   and the history update N_* <- the filtered nonlinear terms, R_PI_* <- the
//   filtered velocity.  hyper = 0 (VISC%SW /= 3) skips both filters.
// PC2VEL (mod_legops.f90:1789-1853) of (psi, chi) at one FFF entry (m, n, k).
__device__ __forceinline__ void pc2vel_at(const DevGrid& g, int m, int n, int k, const double2* psi, double lp,
                                          const double2* chi, double lc, int pad, double2 (&u)[3]) {
    const Col cp = column(g, psi, m, k, pad), cc = column(g, chi, m, k, pad);
    u[0] = u[1] = u[2] = make_double2(0.0, 0.0);
    if (n < cp.nn) {
        const double mv = (double)m, kv = g.ak[k];
        const double2 ps = cp.p[(size_t)n * cp.st], ch = cc.p[(size_t)n * cc.st];
        const double2 xc = xxdx_row(g, m, k, cc, n, lc);
        const double2 xp = xxdx_row(g, m, k, cp, n, lp);
        u[0] = cadd(cmuli(ps, mv), cmuli(xc, kv));
        u[1] = make_double2(-xp.x - (mv * kv) * ch.x, -xp.y - (mv * kv) * ch.y);
        u[2] = neg_xm2_delsqh(g, m, k, cc, n, lc);
    }
}

// Three 256-thread blocks per SM (at most 80 registers; a few bytes spill):
// the kernel is bound by memory-level parallelism, and this beats the 98-register
// form at two blocks per SM.
__global__ void __launch_bounds__(256, 3) etd_ab_fused_kernel(DevGrid g, EtdAbArgs a) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int m, n, k;
    if (!fff_index(g, t, m, n, k)) return;
    if (t < 3) *a.out_ln[t] = 0.0;
    double fv = 1.0, fd = 1.0;
    if (a.hyper) {
        if (n < nrchops(g, m, 0)) {
            fv = a.hv[0][(size_t)m * g.NRCHOP + n] * a.hv[1][m] * a.hv[2][k];
            fd = a.hd[0][(size_t)m * g.NRCHOP + n] * a.hd[1][m] * a.hd[2][k];
        } else {
            fv = fd = 0.0;
        }
    }
    // PC2VEL(PSI, CHI) at pad 3
    double2 u[3];
    pc2vel_at(g, m, n, k, a.psi, *a.psi_ln, a.chi, *a.chi_ln, 3, u);
    const double2 u0 = u[0], u1 = u[1], u2 = u[2];
    // the projected nonlinear terms in velocity form: read, or PC2VEL of (PSI_N, CHI_N) here
    double2 w[3];
    if (a.npsi) {
        pc2vel_at(g, m, n, k, a.npsi, *a.npsi_ln, a.nchi, *a.nchi_ln, 3, w);
    } else {
        w[0] = a.ror[t];
        w[1] = a.rop[t];
        w[2] = a.oz[t];
    }
    const double2 rn[4] = {cscale(w[0], fv), cscale(w[1], fv), cscale(w[2], fv), cscale(a.bn[t], fd)};
    const double notm0 = (m == 0) ? 0.0 : 1.0, notk0 = (k == 0) ? 0.0 : 1.0;
    // history: 0 N_B, 1 R_N_R, 2 R_N_P, 3 N_Z, 4 R_PI_R, 5 R_PI_P, 6 PI_Z
    const double2 ev[4] = {csub(u0, a.hist[4][t]), csub(u1, cscale(a.hist[5][t], notm0)),
                           csub(u2, cscale(a.hist[6][t], notk0)), a.b[t]};
    const double2 on[4] = {a.hist[1][t], a.hist[2][t], a.hist[3][t], a.hist[0][t]};
    double2 av[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) av[j] = csub(cscale(rn[j], 1.5), cscale(on[j], 0.5));
    // E and N are read from the parameter bank in the sums (no register copies);
    // at k = 0 rows 0 and 1 are the identity and dt times it.
    double2 cv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double2 x = make_double2(0.0, 0.0), y = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            x.x += a.E[i * 4 + j] * ev[j].x;
            x.y += a.E[i * 4 + j] * ev[j].y;
            y.x += a.N[i * 4 + j] * av[j].x;
            y.y += a.N[i * 4 + j] * av[j].y;
        }
        if (i < 2 && k == 0) {
            x = ev[i];
            y = cscale(av[i], a.dt);
        }
        cv[i] = a.raw_out ? cadd(x, y) : cscale(cadd(x, y), i < 3 ? fv : fd);
    }
    a.rur[t] = cv[0];
    a.rup[t] = cv[1];
    a.uz[t] = cv[2];
    a.b[t] = cv[3];
    a.hist[0][t] = rn[3];
    a.hist[1][t] = rn[0];
    a.hist[2][t] = rn[1];
    a.hist[3][t] = rn[2];
    if (!a.raw_out) {
        a.hist[4][t] = cv[0];
        a.hist[5][t] = cv[1];
        a.hist[6][t] = cv[2];
    }
}

// The damping of CALC_BOUSSI_ETD_SPONGE (mod_march.f90:1455-1464) on a PFP
// field ([r][z][m]): every z-plane times damp[z], the m = 0 modes made real.
__global__ void sponge_kernel(DevGrid g, double2* a, const double* damp) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t md = g.NTCHOPDIM, total = (size_t)g.NR * g.NX * md;
    if (t >= total) return;
    const int m = (int)(t % md), z = (int)((t / md) % g.NX);
    double2 v = cscale(a[t], damp[z]);
    if (m == 0) v.y = 0.0;
    a[t] = v;
}
void k_sponge(const DevGrid& g, double2* a, const double* damp, cudaStream_t s) {
    const size_t n = (size_t)g.NR * g.NX * g.NTCHOPDIM;
    sponge_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, damp);
    count_launch();
}

// ABSVEC2(U, V, W, A) of CALCXY (mod_march.f90:2050-2099) on PPP [r][z][j]:
// A = ((RU^2 + RV^2)/R^2 + W^2) / (1-x)^2 per packed sample (re and im apart).
// A may alias W.
__global__ void absvec2_kernel(DevGrid g, const double2* u, const double2* v, const double2* w, double2* a) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t plane = (size_t)g.NX * g.NTH;
    if (t >= (size_t)g.NR * plane) return;
    const int i = (int)(t / plane);
    const double r = g.r[i], om = 1.0 - g.x[i], f = om * om, r2 = r * r;
    const double2 uu = u[t], vv = v[t], ww = w[t];
    a[t] = make_double2(((uu.x * uu.x + vv.x * vv.x) / r2 + ww.x * ww.x) / f,
                        ((uu.y * uu.y + vv.y * vv.y) / r2 + ww.y * ww.y) / f);
}
void k_absvec2(const DevGrid& g, const double2* u, const double2* v, const double2* w, double2* a, cudaStream_t s) {
    const size_t n = (size_t)g.NR * g.NX * g.NTH;
    absvec2_kernel<<<nblk(n, 256), 256, 0, s>>>(g, u, v, w, a);
    count_launch();
}

// LAY(A, GAUS, IP = 2) (mod_layout.f90:64-117) for a list of vortices at once:
// A += GAUS(R, THR/THI, Z) / (1-x)^2 per vortex, GAUS (640-672) a Gaussian of
// strength Q / R0^2 and decay B around a centre displaced by DX, DY sin(AK1 Z - DP)
// with core R0 = R + DR sin(RK Z - RP); Z = ZLEN (z) / NX.  PPP [r][z][j].
__global__ void lay_gaus_kernel(DevGrid g, double zlen, const mlegs_vortex* v, int nv, const double* q, const double* b,
                                double2* a) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t plane = (size_t)g.NX * g.NTH;
    if (t >= (size_t)g.NR * plane) return;
    const int i = (int)(t / plane), z = (int)((t / g.NTH) % g.NX), j = (int)(t % g.NTH);
    const double pi = 3.141592653589793238462643383279502884;
    const double r = g.r[i], om = 1.0 - g.x[i], f = om * om;
    const double zz = zlen * z / g.NX;
    const double th[2] = {2.0 * pi / g.NTH * j, 2.0 * pi / g.NTH * (j + 0.5)};
    double2 acc = a[t];
    for (int p = 0; p < nv; ++p) {
        const double ak1 = 2.0 * pi * v[p].k / zlen, rk = 2.0 * pi * v[p].rk / zlen;
        const double dp = pi / 180.0 * v[p].dp, rp = pi / 180.0 * v[p].rp;
        const double xc = v[p].x + v[p].dx * sin(ak1 * zz - dp);
        const double yc = v[p].y + v[p].dy * sin(ak1 * zz - dp);
        const double r0 = v[p].r + v[p].dr * sin(rk * zz - rp);
        double val[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const double x = r * cos(th[h]), y = r * sin(th[h]);
            const double r2 = ((x - xc) * (x - xc) + (y - yc) * (y - yc)) / (r0 * r0);
            val[h] = q[p] / (r0 * r0) * exp(-b[p] * r2);
        }
        acc.x += val[0] / f;
        acc.y += val[1] / f;
    }
    a[t] = acc;
}
void k_lay_gaus(const DevGrid& g, double zlen, const mlegs_vortex* v, int nv, const double* q, const double* b,
                double2* a, cudaStream_t s) {
    const size_t n = (size_t)g.NR * g.NX * g.NTH;
    lay_gaus_kernel<<<nblk(n, 256), 256, 0, s>>>(g, zlen, v, nv, q, b, a);
    count_launch();
}

// max over n values of |a| (mode 0) or |Re a| (mode 1) into *out (zeroed by the
// caller); non-negative doubles order like their bit patterns.
__global__ void maxabs_kernel(const double2* a, size_t n, int mode, unsigned long long* out) {
    double mx = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const double2 v = a[t];
        mx = fmax(mx, mode ? fabs(v.x) : hypot(v.x, v.y));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}
void k_maxabs(const double2* a, size_t n, int mode, double* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(double), s);
    int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    if (blocks < 1) blocks = 1;
    maxabs_kernel<<<blocks, 256, 0, s>>>(a, n, mode, (unsigned long long*)out);
    count_launch();
}

// NOISE(A, ALEVEL), mod_layout.f90:165-226, on the FFF layout [m][n][k]: for
// m < NTCHOP, n < NRCHOPS(m) (pad 0), all k, in the reference's loop order
// (m, n, k) the call pair (2j, 2j+1) of RAN0 (196-214) gives X and Y; RAN0's
// state is the Park-Miller sequence v_{j+1} = 16807 v_j mod (2^31 - 1) from
// v_0 = ISEED xor 123459876, output v_{j+1} / (2^31 - 1), so element j jumps
// ahead by modular powers.  FAC = 0.1 exp(-12 ((AK/AKMAX)^2 + (N/NRCHOP)^2)),
// and A += (X, Y) REFVAL with REFVAL = ALEVEL max|A| (refmax holds max|A|); the
// reference is built with default REAL of 8 bytes (-r8 / -fdefault-real-8), so
// the literals, FLOAT and CMPLX are all double precision.
__device__ __forceinline__ unsigned long long powmod_ia(unsigned long long e) {
    const unsigned long long IM = 2147483647ull;
    unsigned long long r = 1, b = 16807;
    while (e) {
        if (e & 1) r = r * b % IM;
        b = b * b % IM;
        e >>= 1;
    }
    return r;
}
__global__ void noise_kernel(DevGrid g, double2* a, const double* refmax, double alevel, double akmax, long long v0) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int m, n, k;
    if (!fff_index(g, t, m, n, k)) return;
    const int mlim = g.NTCHOP < g.NTCHOPDIM ? g.NTCHOP : g.NTCHOPDIM;
    if (m >= mlim || n >= nrchops(g, m, 0)) return;
    long long row = n;  // rows before (m, n) in the (m, n) loop order
    for (int mm = 0; mm < m; ++mm) row += nrchops(g, mm, 0);
    const unsigned long long j = 2ull * ((unsigned long long)row * g.NXCHOPDIM + k);
    const unsigned long long IM = 2147483647ull;
    const double AM = 1.0 / 2147483647.0;
    const unsigned long long vx = powmod_ia(j + 1) * (unsigned long long)v0 % IM;
    const unsigned long long vy = vx * 16807ull % IM;
    const double akr = g.ak[k] / akmax;
    const double q = (double)(m + n) / (double)g.NRCHOP;
    const double fac = 0.1 * exp(-12.0 * (akr * akr + q * q));
    const double x = fac * (AM * (double)vx), y = fac * (AM * (double)vy);
    const double refval = alevel * *refmax;
    double2 v = a[t];
    v.x += x * refval;
    v.y += y * refval;
    a[t] = v;
}
void k_noise(const DevGrid& g, double2* a, const double* refmax, double alevel, double akmax, long long v0,
             cudaStream_t s) {
    const size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    noise_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, refmax, alevel, akmax, v0);
    count_launch();
}

// FLATTEN(A, B), mod_layout.f90:228-278, on PPP: A = B + (A - B) tanh(20 B / REFVAL)^2
// per packed sample, REFVAL = max |Re A| (1 if zero; refmax holds it).
__global__ void flatten_kernel(DevGrid g, double2* a, const double2* b, const double* refmax) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)g.NR * g.NX * g.NTH) return;
    double refval = *refmax;
    if (refval == 0.0) refval = 1.0;
    const double2 rb = b[t], av = a[t];
    const double fr = tanh(rb.x / refval * 20.0), fi = tanh(rb.y / refval * 20.0);
    a[t] = make_double2(rb.x + (av.x - rb.x) * (fr * fr), rb.y + (av.y - rb.y) * (fi * fi));
}
void k_flatten(const DevGrid& g, double2* a, const double2* b, const double* refmax, cudaStream_t s) {
    const size_t n = (size_t)g.NR * g.NX * g.NTH;
    flatten_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, b, refmax);
    count_launch();
}

// dst = src * {1, R cos(th), R sin(th), R^2}[mode] on PPP [r][z][j], the re
// sample at THR(j) = 2 pi j / NTH and the im sample at THI(j) = 2 pi (j + 1/2) / NTH
// (MULRCOSTH / MULRSINTH / MULR2, mod_march.f90:2102-2225; TFM%THR/THI, mod_fft.f90:323-324).
__global__ void mulr_kernel(DevGrid g, const double2* src, double2* dst, int mode) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t plane = (size_t)g.NX * g.NTH;
    if (t >= (size_t)g.NR * plane) return;
    const int i = (int)(t / plane), j = (int)(t % g.NTH);
    const double r = g.r[i];
    const double pi = 3.141592653589793238462643383279502884;
    const double thr = 2.0 * pi / g.NTH * j, thi = 2.0 * pi / g.NTH * (j + 0.5);
    double fr = 1.0, fi = 1.0;
    if (mode == 1) {
        fr = r * cos(thr);
        fi = r * cos(thi);
    } else if (mode == 2) {
        fr = r * sin(thr);
        fi = r * sin(thi);
    } else if (mode == 3) {
        fr = fi = r * r;
    }
    const double2 a = src[t];
    dst[t] = make_double2(fr * a.x, fi * a.y);
}
void k_mulr(const DevGrid& g, const double2* src, double2* dst, int mode, cudaStream_t s) {
    const size_t n = (size_t)g.NR * g.NX * g.NTH;
    mulr_kernel<<<nblk(n, 256), 256, 0, s>>>(g, src, dst, mode);
    count_launch();
}

void k_etd_ab_fused(const DevGrid& g, const EtdAbArgs& a, cudaStream_t s) {
    const size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    etd_ab_fused_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a);
    count_launch();
}

void k_grad_fused(const DevGrid& g, const double2* a, const double* ln, double2* rr, double2* rp, double2* gz, int pad,
                  cudaStream_t s) {
    const size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    grad_fused_kernel<<<nblk(n, 256), 256, 0, s>>>(g, a, ln, rr, rp, gz, pad);
    count_launch();
}

void k_pc2vel_fused(const DevGrid& g, const double2* psi, const double* psi_ln, const double2* chi, const double* chi_ln,
                    double2* rur, double2* rup, double2* uz, int pad, cudaStream_t s, int sub, double* const* zero_ln) {
    const size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    pc2vel_fused_kernel<<<nblk(n, 256), 256, 0, s>>>(g, psi, psi_ln, chi, chi_ln, rur, rup, uz, pad, sub,
                                                     zero_ln ? zero_ln[0] : nullptr, zero_ln ? zero_ln[1] : nullptr,
                                                     zero_ln ? zero_ln[2] : nullptr);
    count_launch();
}

void k_pc2vor_fused(const DevGrid& g, const double2* psi, const double* psi_ln, const double2* chi, const double* chi_ln,
                    double2* ror, double2* rop, double2* oz, int pad, cudaStream_t s) {
    const size_t n = g.NTCHOPDIM * (size_t)g.NRCHOPDIM * g.NXCHOPDIM;
    pc2vor_fused_kernel<<<nblk(n, 256), 256, 0, s>>>(g, psi, psi_ln, chi, chi_ln, ror, rop, oz, pad);
    count_launch();
}

}  // namespace mlegs
