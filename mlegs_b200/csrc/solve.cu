// Batched banded solves of the Laplacian / Helmholtz operators, FP64.
//
// Restates the per-(m,k) systems of mod_legops.f90 IDEL2LN (1013-1176),
// IDEL2 (823-1010) and IHELM (1204-1354), factored without pivoting as
// LUDCMPB/LUBKSBB do (mod_bandmat.f90:65-155, 320-401).  One thread owns one
// (m, k) system: it builds each band row on the fly from the DEL2H/XM
// coefficient tables, eliminates its sub-diagonal entries against the
// previous pivot rows (kept in registers), writes the resulting U row to a
// scratch array laid out [row][entry][system] (coalesced across threads),
// and back-substitutes in place.  Band entries that reach past the system's
// size are dropped, which is BANDAUX's truncation of each leading block.
//
//  kind 0  IDEL2LN: m = 0 systems carry the log-term column (k = 0), 5-band
//  kind 1  IDEL2:   m = 0 uses the 7-band row-shifted system (k = 0: row 0 is
//                   the log-term boundary condition)
//  kind 2  IHELM:   m = 0 solves (H XM) y = rhs on NN-1 rows, A = XM y
#include "mlegs_internal.h"

namespace mlegs {

namespace {
constexpr int MAXW = 7;  // band width bound (7-band m = 0 systems)
constexpr int RB = 6;    // rows whose loads are issued together; a multiple of 3 so that
                         // the 3-row pivot window is indexed by compile-time constants
}

struct BandRowCtx {
    const double* del2h;  // [NB][5] for this m
    const double* xm;     // [NB][2] for this m (m = 0 only)
    double shift;         // k^2 + alpha
    int kind, m, k;
    double l0, l1, l2;    // log-term column entries (IDEL2LN / IDEL2 at m = k = 0)
};

// Entry (row, col) of the original DEL2H - shift operator (with the log column).
__device__ __forceinline__ double del2_entry(const BandRowCtx& c, int row, int col) {
    int d = col - row;
    if (d < -2 || d > 2 || row < 0 || col < 0) return 0.0;
    double v = c.del2h[(size_t)row * 5 + (d + 2)];
    if (d == 0) v -= c.shift;
    if (col == 0 && (c.kind == 0 || c.kind == 1) && c.m == 0 && c.k == 0) {
        if (row == 0) v += c.l0;
        else if (row == 1) v += c.l1;
        else if (row == 2) v += c.l2;
    }
    return v;
}

// Row `row` of the system matrix, as entries at columns row-3..row+3 (w[0..6]).
__device__ __forceinline__ void build_row(const BandRowCtx& c, int row, double* w) {
#pragma unroll
    for (int q = 0; q < MAXW; ++q) w[q] = 0.0;
    if (c.m != 0 || c.kind == 0) {
        for (int d = -2; d <= 2; ++d) w[d + 3] = del2_entry(c, row, row + d);
        return;
    }
    if (c.kind == 1) {
        if (c.k != 0) {
            for (int d = -2; d <= 2; ++d) w[d + 3] = del2_entry(c, row, row + d);
        } else if (row == 0) {
            w[3] = 1.0;
        } else {
            // new row r = original row r-1 over the same columns
            for (int col = row - 3; col <= row + 1; ++col)
                if (col >= 0) w[col - row + 3] = del2_entry(c, row - 1, col);
        }
        return;
    }
    // kind 2, m = 0: (H XM)(row, col) = sum_l H(row, l) XM(l, col)
    for (int l = row - 2; l <= row + 2; ++l) {
        if (l < 0) continue;
        double h = del2_entry(c, row, l);
        if (h == 0.0) continue;
        const double* x = c.xm + (size_t)l * 2;
        // XM(l, l-1) = sub(l), XM(l, l) = 1, XM(l, l+1) = super(l)
        if (l - 1 >= 0) w[(l - 1) - row + 3] += h * x[0];
        w[l - row + 3] += h;
        w[(l + 1) - row + 3] += h * x[1];
    }
}

__global__ void solve_kernel(DevGrid g, double2* A, double* ln_out, int kind, double alp, int has_ln,
                             double ln_in, const double* b_ln, double* scratch, int pad) {
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsys) return;
    const int k = t % g.NXCHOPDIM;
    const int m = t / g.NXCHOPDIM;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    BandRowCtx c;
    c.del2h = g.del2h + (size_t)m * g.NB * 5;
    c.xm = g.xm + (size_t)m * g.NB * 2;
    c.shift = g.ak[k] * g.ak[k] + ((kind == 2) ? alp : 0.0);
    c.kind = kind;
    c.m = m;
    c.k = k;
    c.l0 = 4.0 / 3 / g.ELL2;
    c.l1 = -2 * g.norm0[0] / g.norm0[1] / g.ELL2;
    c.l2 = 2.0 / 3 * g.norm0[0] / g.norm0[2] / g.ELL2;
    int lo = 2, up = 2;
    if (m == 0 && kind != 0) {
        lo = 3;
        up = 3;
    }
    int size = (m == 0 && kind == 2) ? nn - 1 : nn;
    double2* col = A + (size_t)m * g.NRCHOPDIM * g.NXCHOPDIM + k;
    const size_t st = g.NXCHOPDIM;
    if (size <= 0) return;
    // IDEL2 (m = 0, k = 0): shift the rhs down one row, row 0 <- LN BC (929-936)
    if (kind == 1 && m == 0 && k == 0) {
        for (int r = size - 1; r >= 1; --r) col[(size_t)r * st] = col[(size_t)(r - 1) * st];
        col[0] = make_double2(has_ln ? ln_in / g.norm0[0] : 0.0, 0.0);
    }
    // forward elimination; window of the last 3 pivot rows (U entries d = 0..up)
    double U[3][4];
    double2 R[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        R[a] = make_double2(0.0, 0.0);
#pragma unroll
        for (int b = 0; b < 4; ++b) U[a][b] = 0.0;
    }
    for (int r0 = 0; r0 < size; r0 += RB) {
        // each row reads only its own right-hand side, so the block's loads go first
        double2 rb[RB];
#pragma unroll
        for (int q = 0; q < RB; ++q) rb[q] = (r0 + q < size) ? col[(size_t)(r0 + q) * st] : make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int r = r0 + q;  // r0 is a multiple of 3: r % 3 == q % 3
            if (r >= size) break;
            double w[MAXW];
            build_row(c, r, w);
            double2 rhs = rb[q];
            // eliminate columns r-lo .. r-1 (left to right)
#pragma unroll
            for (int d = 3; d >= 1; --d) {
                if (d > lo || r - d < 0) continue;
                const int wi = (q - d + 3) % 3;  // (r - d) % 3
                const double f = w[3 - d] / U[wi][0];
                w[3 - d] = 0.0;
#pragma unroll
                for (int j = 1; j <= 3; ++j) {
                    if (j > up) continue;
                    const int qq = 3 - d + j;
                    if (qq < MAXW) w[qq] -= f * U[wi][j];
                }
                rhs.x -= f * R[wi].x;
                rhs.y -= f * R[wi].y;
            }
            const int wr = q % 3;
            U[wr][0] = w[3];
#pragma unroll
            for (int j = 1; j <= 3; ++j) U[wr][j] = (j <= up) ? w[3 + j] : 0.0;
            R[wr] = rhs;
#pragma unroll
            for (int j = 0; j <= 3; ++j) scratch[((size_t)r * 4 + j) * nsys + t] = U[wr][j];
            col[(size_t)r * st] = rhs;
        }
    }
    // back substitution
    double2 x1 = make_double2(0.0, 0.0), x2 = x1, x3 = x1;  // x[r+1], x[r+2], x[r+3]
    for (int r1 = size - 1; r1 >= 0; r1 -= RB) {
        double2 vb[RB];
        double ub[RB][4];
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int r = r1 - q;
            vb[q] = make_double2(0.0, 0.0);
            ub[q][0] = 1.0;
            ub[q][1] = ub[q][2] = ub[q][3] = 0.0;
            if (r >= 0) {
                vb[q] = col[(size_t)r * st];
#pragma unroll
                for (int j = 0; j < 4; ++j) ub[q][j] = scratch[((size_t)r * 4 + j) * nsys + t];
            }
        }
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            const int r = r1 - q;
            if (r < 0) break;
            double2 v = vb[q];
            const double u0 = ub[q][0], u1 = ub[q][1], u2 = ub[q][2], u3 = ub[q][3];
            if (r + 1 < size) { v.x -= u1 * x1.x; v.y -= u1 * x1.y; }
            if (r + 2 < size) { v.x -= u2 * x2.x; v.y -= u2 * x2.y; }
            if (r + 3 < size) { v.x -= u3 * x3.x; v.y -= u3 * x3.y; }
            v.x /= u0;
            v.y /= u0;
            col[(size_t)r * st] = v;
            x3 = x2;
            x2 = x1;
            x1 = v;
        }
    }
    if (m == 0 && kind == 2) {
        // A(NN) = 0; A(:NN) = XM(:NN) y  (1310-1316)
        col[(size_t)(nn - 1) * st] = make_double2(0.0, 0.0);
        double2 prev = make_double2(0.0, 0.0);
        for (int r = 0; r < nn; ++r) {
            double2 cur = col[(size_t)r * st];
            double2 nxt = (r + 1 < nn) ? col[(size_t)(r + 1) * st] : make_double2(0.0, 0.0);
            const double* x = c.xm + (size_t)r * 2;
            double2 v = cur;
            if (r >= 1) { v.x += x[0] * prev.x; v.y += x[0] * prev.y; }
            if (r + 1 < nn) { v.x += x[1] * nxt.x; v.y += x[1] * nxt.y; }
            col[(size_t)r * st] = v;
            prev = cur;
        }
    }
    if (m == 0 && k == 0) {
        if (kind == 0) {
            *ln_out = col[0].x * g.norm0[0];
            col[0] = make_double2(0.0, 0.0);
        } else if (kind == 1 && has_ln) {
            *ln_out = col[0].x * g.norm0[0];
        }
    }
}

// ---------------------------------------------------------------------------
// Factor once, solve many.  For a fixed (kind, pad, alp) the system matrices
// do not change from call to call, so their LU factors (the same unpivoted
// elimination as solve_kernel, LUDCMPB of mod_bandmat.f90:65-155) are stored
// once and every later solve is only the substitutions of LUBKSBB (320-401):
//   F5 [row][5][system]  f2 = L(r, r-2), f1 = L(r, r-1), U(r, r), U(r, r+1), U(r, r+2)
//                        for the 5-band systems;
//   F7 [row][7][k]       f3, f2, f1, U(r, r .. r+3) for the 7-band m = 0 systems
//                        of kinds 1 and 2.
// The multipliers and pivots are the ones solve_kernel forms, and the
// substitutions apply them in the same order.  The two kernels are compiled
// separately (solve_kernel's elimination is unrolled in register windows), so
// the compiler contracts different products into FMAs: the results agree to a
// few units in the last place (about 2e-16 relative to the field, 1e-15 at
// most, measured on B200), not bit for bit.
__global__ void factor_kernel(DevGrid g, int kind, double alp, int pad, double* F5, double* F7) {
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsys) return;
    const int k = t % g.NXCHOPDIM;
    const int m = t / g.NXCHOPDIM;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    BandRowCtx c;
    c.del2h = g.del2h + (size_t)m * g.NB * 5;
    c.xm = g.xm + (size_t)m * g.NB * 2;
    c.shift = g.ak[k] * g.ak[k] + ((kind == 2) ? alp : 0.0);
    c.kind = kind;
    c.m = m;
    c.k = k;
    c.l0 = 4.0 / 3 / g.ELL2;
    c.l1 = -2 * g.norm0[0] / g.norm0[1] / g.ELL2;
    c.l2 = 2.0 / 3 * g.norm0[0] / g.norm0[2] / g.ELL2;
    const bool wide = (m == 0 && kind != 0);
    const int lo = wide ? 3 : 2, up = wide ? 3 : 2;
    const int size = (m == 0 && kind == 2) ? nn - 1 : nn;
    double U[3][4] = {};
    for (int r = 0; r < size; ++r) {
        double w[MAXW];
        build_row(c, r, w);
        double f[4] = {0.0, 0.0, 0.0, 0.0};
        for (int d = 3; d >= 1; --d) {
            if (d > lo || r - d < 0) continue;
            const int wi = (r - d) % 3;
            f[d] = w[3 - d] / U[wi][0];
            w[3 - d] = 0.0;
            for (int j = 1; j <= 3; ++j) {
                if (j > up) continue;
                const int qq = 3 - d + j;
                if (qq < MAXW) w[qq] -= f[d] * U[wi][j];
            }
        }
        const int wr = r % 3;
        U[wr][0] = w[3];
        for (int j = 1; j <= 3; ++j) U[wr][j] = (j <= up) ? w[3 + j] : 0.0;
        if (wide) {
            double* o = F7 + (size_t)r * 7 * g.NXCHOPDIM + k;
            o[0] = f[3];
            o[(size_t)1 * g.NXCHOPDIM] = f[2];
            o[(size_t)2 * g.NXCHOPDIM] = f[1];
            for (int j = 0; j < 4; ++j) o[(size_t)(3 + j) * g.NXCHOPDIM] = U[wr][j];
        } else {
            double* o = F5 + (size_t)r * 5 * nsys + t;
            o[0] = f[2];
            o[(size_t)1 * nsys] = f[1];
            for (int j = 0; j < 3; ++j) o[(size_t)(2 + j) * nsys] = U[wr][j];
        }
    }
}

// One thread per (system, real or imaginary part).  Reads the right-hand side
// from src, writes the solution to dst (rows >= the system size are zeroed),
// then the per-kind tails of solve_kernel; farfield = 1 also applies the
// CALCAT1 row-0 correction over n < NRCHOP + pad to the m = 0 columns.
// One (system, real or imaginary part) u of the factored substitutions: the
// body of solve_factored_kernel, also run by the grouped ensemble kernel.
// WB: rows per load block of the 7-band systems (16 where registers allow)
template <int WB>
__device__ __forceinline__ void solve_factored_sys(const DevGrid& g, const double* __restrict__ F5,
                                                   const double* __restrict__ F7, const double2* src, double2* dst,
                                                   double* ln_out, int kind, int has_ln, double ln_in, int pad,
                                                   int farfield, int u) {
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int t = u >> 1, comp = u & 1;
    if (t >= nsys) return;
    const int k = t % g.NXCHOPDIM;
    const int m = t / g.NXCHOPDIM;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    const bool wide = (m == 0 && kind != 0);
    int size = (m == 0 && kind == 2) ? nn - 1 : nn;
    if (size < 0) size = 0;
    const size_t cofs = (size_t)m * g.NRCHOPDIM * g.NXCHOPDIM + k;
    const double* in = (const double*)(src + cofs) + comp;
    double* col = (double*)(dst + cofs) + comp;
    const size_t st = 2 * (size_t)g.NXCHOPDIM;
    // IDEL2 (m = 0, k = 0): right-hand side shifted down one row, row 0 <- the LN condition (929-936)
    const bool shift = (kind == 1 && m == 0 && k == 0);
    auto rhs = [&](int r) -> double {
        if (!shift) return in[(size_t)r * st];
        if (r == 0) return comp ? 0.0 : (has_ln ? ln_in / g.norm0[0] : 0.0);
        return in[(size_t)(r - 1) * st];
    };
    // out of place, the substitution reads the shifted rows directly; in place,
    // they are shifted first (each row read before it is overwritten)
    const bool direct = shift && (const void*)src != (const void*)dst;
    if (shift && !direct) {
        double prev = rhs(0);
        for (int r = 0; r < size; ++r) {
            const double cur = (r + 1 < size) ? rhs(r + 1) : 0.0;
            col[(size_t)r * st] = prev;
            prev = cur;
        }
        in = col;
    }
    constexpr int RBF = 16;
    if (!wide) {
        double y1 = 0.0, y2 = 0.0;
        for (int r0 = 0; r0 < size; r0 += RBF) {
            double rb[RBF], fa[RBF], fb[RBF];
#pragma unroll
            for (int q = 0; q < RBF; ++q) {
                const int r = r0 + q;
                const bool ok = r < size;
                rb[q] = ok ? in[(size_t)r * st] : 0.0;
                fa[q] = ok ? F5[(size_t)r * 5 * nsys + t] : 0.0;
                fb[q] = ok ? F5[((size_t)r * 5 + 1) * nsys + t] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < RBF; ++q) {
                if (r0 + q >= size) break;
                const double y = __fma_rn(-fb[q], y1, __fma_rn(-fa[q], y2, rb[q]));
                col[(size_t)(r0 + q) * st] = y;
                y2 = y1;
                y1 = y;
            }
        }
        double x1 = 0.0, x2 = 0.0;
        for (int r1 = size - 1; r1 >= 0; r1 -= RBF) {
            double vb[RBF], u0[RBF], u1[RBF], u2[RBF];
#pragma unroll
            for (int q = 0; q < RBF; ++q) {
                const int r = r1 - q;
                const bool ok = r >= 0;
                vb[q] = ok ? col[(size_t)r * st] : 0.0;
                u0[q] = ok ? F5[((size_t)r * 5 + 2) * nsys + t] : 1.0;
                u1[q] = ok ? F5[((size_t)r * 5 + 3) * nsys + t] : 0.0;
                u2[q] = ok ? F5[((size_t)r * 5 + 4) * nsys + t] : 0.0;
            }
            // the diagonal's reciprocal and the scaled row are formed off the
            // recurrence, which then costs one dependent FMA per row (a divide
            // on the recurrence made the substitution latency-bound)
#pragma unroll
            for (int q = 0; q < RBF; ++q) {
                const int r = r1 - q;
                const double ri = 1.0 / u0[q];
                vb[q] = __dmul_rn(vb[q], ri);
                u1[q] = (r + 1 < size) ? __dmul_rn(u1[q], ri) : 0.0;
                u2[q] = (r + 2 < size) ? __dmul_rn(u2[q], ri) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < RBF; ++q) {
                const int r = r1 - q;
                if (r < 0) break;
                const double v = __fma_rn(-u1[q], x1, __fma_rn(-u2[q], x2, vb[q]));
                col[(size_t)r * st] = v;
                x2 = x1;
                x1 = v;
            }
        }
    } else {
        const size_t NK = g.NXCHOPDIM;
        constexpr int RBW = WB;
        double y1 = 0.0, y2 = 0.0, y3 = 0.0;
        for (int r0 = 0; r0 < size; r0 += RBW) {
            double rb[RBW], f3[RBW], f2[RBW], f1[RBW];
#pragma unroll
            for (int q = 0; q < RBW; ++q) {
                const int r = r0 + q;
                const bool ok = r < size;
                const double* f = F7 + (size_t)r * 7 * NK + k;
                rb[q] = ok ? (direct ? rhs(r) : in[(size_t)r * st]) : 0.0;
                f3[q] = ok ? f[0] : 0.0;
                f2[q] = ok ? f[NK] : 0.0;
                f1[q] = ok ? f[2 * NK] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < RBW; ++q) {
                if (r0 + q >= size) break;
                const double y = __fma_rn(-f1[q], y1, __fma_rn(-f2[q], y2, __fma_rn(-f3[q], y3, rb[q])));
                col[(size_t)(r0 + q) * st] = y;
                y3 = y2;
                y2 = y1;
                y1 = y;
            }
        }
        double x1 = 0.0, x2 = 0.0, x3 = 0.0;
        for (int r1 = size - 1; r1 >= 0; r1 -= RBW) {
            double vb[RBW], u0[RBW], u1[RBW], u2[RBW], u3[RBW];
#pragma unroll
            for (int q = 0; q < RBW; ++q) {
                const int r = r1 - q;
                const bool ok = r >= 0;
                const double* f = F7 + (size_t)(ok ? r : 0) * 7 * NK + k;
                vb[q] = ok ? col[(size_t)r * st] : 0.0;
                u0[q] = ok ? f[3 * NK] : 1.0;
                u1[q] = ok ? f[4 * NK] : 0.0;
                u2[q] = ok ? f[5 * NK] : 0.0;
                u3[q] = ok ? f[6 * NK] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < RBW; ++q) {
                const int r = r1 - q;
                const double ri = 1.0 / u0[q];
                vb[q] = __dmul_rn(vb[q], ri);
                u1[q] = (r + 1 < size) ? __dmul_rn(u1[q], ri) : 0.0;
                u2[q] = (r + 2 < size) ? __dmul_rn(u2[q], ri) : 0.0;
                u3[q] = (r + 3 < size) ? __dmul_rn(u3[q], ri) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < RBW; ++q) {
                const int r = r1 - q;
                if (r < 0) break;
                const double v = __fma_rn(-u1[q], x1, __fma_rn(-u2[q], x2, __fma_rn(-u3[q], x3, vb[q])));
                col[(size_t)r * st] = v;
                x3 = x2;
                x2 = x1;
                x1 = v;
            }
        }
    }
    for (int r = size; r < g.NRCHOPDIM; ++r) col[(size_t)r * st] = 0.0;
    if (m == 0 && kind == 2 && nn > 0) {
        // A(NN) = 0; A(:NN) = XM(:NN) y  (1310-1316)
        const double* xm = g.xm;
        double prev = 0.0;
        for (int r = 0; r < nn; ++r) {
            const double cur = col[(size_t)r * st];
            const double nxt = (r + 1 < nn) ? col[(size_t)(r + 1) * st] : 0.0;
            // explicit roundings here and below: every kernel that runs this
            // body (single and grouped) gives the same bits
            double v = cur;
            if (r >= 1) v = __fma_rn(xm[(size_t)r * 2], prev, v);
            if (r + 1 < nn) v = __fma_rn(xm[(size_t)r * 2 + 1], nxt, v);
            col[(size_t)r * st] = v;
            prev = cur;
        }
    }
    if (m == 0 && k == 0 && size > 0) {
        if (kind == 0) {
            if (!comp) *ln_out = __dmul_rn(col[0], g.norm0[0]);
            col[0] = 0.0;
        } else if (kind == 1 && !comp && ln_out) {
            *ln_out = has_ln ? __dmul_rn(col[0], g.norm0[0]) : 0.0;
        }
    }
    if (farfield && m == 0) {
        // a(n=0, m=0, k) -= sum_{n < NRCHOP+pad} AT1(n) a(n, 0, k) / AT1(0)
        const int nr_sum = g.NRCHOP + pad;
        double sum = 0.0;
        for (int r = 0; r < nr_sum && r < g.NRCHOPDIM; ++r) sum = __fma_rn(g.at1[r], col[(size_t)r * st], sum);
        col[0] = __dsub_rn(col[0], __ddiv_rn(sum, g.at1[0]));
    }
}

void solve_factor_sizes(const DevGrid& g, size_t* f5, size_t* f7) {
    *f5 = (size_t)g.NRCHOPDIM * 5 * g.NTCHOPDIM * g.NXCHOPDIM;
    *f7 = (size_t)g.NRCHOPDIM * 7 * g.NXCHOPDIM;
}

void k_solve_factor(const DevGrid& g, int kind, double alp, int pad, double* F5, double* F7, cudaStream_t s) {
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    factor_kernel<<<(nsys + 63) / 64, 64, 0, s>>>(g, kind, alp, pad, F5, F7);
    count_launch();
}

__global__ void __launch_bounds__(128) solve_factored_kernel(DevGrid g, const double* __restrict__ F5,
                                                             const double* __restrict__ F7, const double2* src,
                                                             double2* dst, double* ln_out, int kind, int has_ln,
                                                             double ln_in, int pad, int farfield, int wpad) {
    // kinds 1 and 2: the 7-band m = 0 systems (u < 2 NXCHOPDIM) take whole
    // warps, the 5-band ones start after wpad idle threads, so that no warp
    // runs both substitutions one after the other
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int nw = 2 * g.NXCHOPDIM;
    if (wpad) {
        if (u >= nw && u < nw + wpad) return;
        if (u >= nw) u -= wpad;
    }
    solve_factored_sys<16>(g, F5, F7, src, dst, ln_out, kind, has_ln, ln_in, pad, farfield, u);
}

// Small systems (NRCHOP + pad <= SMALL_R rows): one warp takes 16 systems
// (lane = system x real/imaginary part), copies their factor rows and
// right-hand sides into shared memory in one burst of cp.async copies, and
// runs the substitutions and the tails of solve_factored_sys there, with the
// same operations in the same order.  Blocks [0, nb0) hold the t_begin
// 7-band m = 0 systems of kinds 1 and 2, the rest the 5-band ones, so no
// warp mixes the two.  Shared memory per block: R x 144 doubles (factor rows
// [r][7][16], values [r][16] complex), R = NRCHOP + pad.
constexpr int SMALL_R = 72;

__device__ __forceinline__ void cpa8(double* d, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(d)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa16(double2* d, const double2* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(d)), "l"(src)
                 : "memory");
}

__global__ void __launch_bounds__(32) solve_small_kernel(DevGrid g, const double* __restrict__ F5,
                                                         const double* __restrict__ F7, const double2* src,
                                                         double2* dst, double* ln_out, int kind, int has_ln,
                                                         double ln_in, int pad, int farfield, int t_begin, int nb0) {
    extern __shared__ __align__(16) double sms[];
    const int R = g.NRCHOP + pad;
    double* Fs = sms;                         // [R][7][16]
    double2* Xs = (double2*)(sms + R * 112);  // [R][16]
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int lane = threadIdx.x, sy = lane >> 1, comp = lane & 1;
    const bool wide_blk = (int)blockIdx.x < nb0;
    const int tb = wide_blk ? blockIdx.x * 16 : t_begin + (blockIdx.x - nb0) * 16;
    const int tend = wide_blk ? t_begin : nsys;
    const int nsb = min(16, tend - tb);
    const size_t NK = g.NXCHOPDIM;
    // the burst: factor rows, then the right-hand sides
    if (wide_blk) {
        for (int e = lane; e < R * 112; e += 32) {
            const int r = e / 112, j = (e / 16) % 7, q = e % 16;
            if (q < nsb) cpa8(Fs + e, F7 + ((size_t)r * 7 + j) * NK + tb + q);
        }
    } else {
        for (int e = lane; e < R * 80; e += 32) {
            const int r = e / 80, j = (e / 16) % 5, q = e % 16;
            if (q < nsb) cpa8(Fs + (r * 7 + j) * 16 + q, F5 + ((size_t)r * 5 + j) * nsys + tb + q);
        }
    }
    for (int e = lane; e < R * 16; e += 32) {
        const int r = e / 16, q = e % 16;
        if (q < nsb) {
            const int tq = tb + q, mq = tq / g.NXCHOPDIM, kq = tq - mq * g.NXCHOPDIM;
            cpa16(Xs + e, src + (size_t)mq * g.NRCHOPDIM * NK + (size_t)r * NK + kq);
        }
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    if (sy >= nsb) return;
    const int t = tb + sy, k = t % g.NXCHOPDIM, m = t / g.NXCHOPDIM;
    int nn = g.NRCHOP + pad - m;
    if (nn < 0) nn = 0;
    const bool wide = wide_blk;
    int size = (m == 0 && kind == 2) ? nn - 1 : nn;
    if (size < 0) size = 0;
    double* X = (double*)Xs + sy * 2 + comp;  // row r at X[r * 32]
    auto F = [&](int r, int j) { return Fs[(r * 7 + j) * 16 + sy]; };
    // IDEL2 (m = 0, k = 0): right-hand side shifted down one row, row 0 <- the LN condition
    if (kind == 1 && m == 0 && k == 0) {
        for (int r = size - 1; r >= 1; --r) X[r * 32] = X[(r - 1) * 32];
        if (size > 0) X[0] = comp ? 0.0 : (has_ln ? ln_in / g.norm0[0] : 0.0);
    }
    if (!wide) {
        double y1 = 0.0, y2 = 0.0;
        for (int r = 0; r < size; ++r) {
            const double y = __fma_rn(-F(r, 1), y1, __fma_rn(-F(r, 0), y2, X[r * 32]));
            X[r * 32] = y;
            y2 = y1;
            y1 = y;
        }
        double x1 = 0.0, x2 = 0.0;
        for (int r = size - 1; r >= 0; --r) {
            const double ri = 1.0 / F(r, 2);
            const double a1 = (r + 1 < size) ? __dmul_rn(F(r, 3), ri) : 0.0;
            const double a2 = (r + 2 < size) ? __dmul_rn(F(r, 4), ri) : 0.0;
            const double v = __fma_rn(-a1, x1, __fma_rn(-a2, x2, __dmul_rn(X[r * 32], ri)));
            X[r * 32] = v;
            x2 = x1;
            x1 = v;
        }
    } else {
        double y1 = 0.0, y2 = 0.0, y3 = 0.0;
        for (int r = 0; r < size; ++r) {
            const double y = __fma_rn(-F(r, 2), y1, __fma_rn(-F(r, 1), y2, __fma_rn(-F(r, 0), y3, X[r * 32])));
            X[r * 32] = y;
            y3 = y2;
            y2 = y1;
            y1 = y;
        }
        double x1 = 0.0, x2 = 0.0, x3 = 0.0;
        for (int r = size - 1; r >= 0; --r) {
            const double ri = 1.0 / F(r, 3);
            const double a1 = (r + 1 < size) ? __dmul_rn(F(r, 4), ri) : 0.0;
            const double a2 = (r + 2 < size) ? __dmul_rn(F(r, 5), ri) : 0.0;
            const double a3 = (r + 3 < size) ? __dmul_rn(F(r, 6), ri) : 0.0;
            const double v =
                __fma_rn(-a1, x1, __fma_rn(-a2, x2, __fma_rn(-a3, x3, __dmul_rn(X[r * 32], ri))));
            X[r * 32] = v;
            x3 = x2;
            x2 = x1;
            x1 = v;
        }
    }
    // the tails of solve_factored_sys, on the staged column
    for (int r = size; r < R; ++r) X[r * 32] = 0.0;
    if (m == 0 && kind == 2 && nn > 0) {
        const double* xm = g.xm;
        double prev = 0.0;
        for (int r = 0; r < nn; ++r) {
            const double cur = X[r * 32];
            const double nxt = (r + 1 < nn) ? X[(r + 1) * 32] : 0.0;
            double v = cur;
            if (r >= 1) v = __fma_rn(xm[(size_t)r * 2], prev, v);
            if (r + 1 < nn) v = __fma_rn(xm[(size_t)r * 2 + 1], nxt, v);
            X[r * 32] = v;
            prev = cur;
        }
    }
    if (m == 0 && k == 0 && size > 0) {
        if (kind == 0) {
            if (!comp) *ln_out = __dmul_rn(X[0], g.norm0[0]);
            X[0] = 0.0;
        } else if (kind == 1 && !comp && ln_out) {
            *ln_out = has_ln ? __dmul_rn(X[0], g.norm0[0]) : 0.0;
        }
    }
    if (farfield && m == 0) {
        double sum = 0.0;
        for (int r = 0; r < R && r < g.NRCHOPDIM; ++r) sum = __fma_rn(g.at1[r], X[r * 32], sum);
        X[0] = __dsub_rn(X[0], __ddiv_rn(sum, g.at1[0]));
    }
    double* col = (double*)(dst + (size_t)m * g.NRCHOPDIM * NK + k) + comp;
    const size_t st = 2 * NK;
    for (int r = 0; r < g.NRCHOPDIM; ++r) col[(size_t)r * st] = r < R ? X[r * 32] : 0.0;
}

bool solve_small_ok(const DevGrid& g, int pad) { return g.NRCHOP + pad <= SMALL_R; }

void k_solve_small(const DevGrid& g, const double* F5, const double* F7, const double2* src, double2* dst,
                   double* ln_out, int kind, int has_ln, double ln_in, int pad, int farfield, cudaStream_t s) {
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int t_begin = kind == 0 ? 0 : g.NXCHOPDIM;
    const int nb0 = (t_begin + 15) / 16, nb1 = (nsys - t_begin + 15) / 16;
    const int R = g.NRCHOP + pad;
    const size_t smem = (size_t)R * 144 * sizeof(double);
    static size_t attr = 0;
    if (smem > attr && smem > 48 * 1024) {
        cudaFuncSetAttribute(solve_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = smem;
    }
    solve_small_kernel<<<nb0 + nb1, 32, smem, s>>>(g, F5, F7, src, dst, ln_out, kind, has_ln, ln_in, pad, farfield,
                                                   t_begin, nb0);
    count_launch();
}

void k_solve_factored(const DevGrid& g, const double* F5, const double* F7, const double2* src, double2* dst,
                      double* ln_out, int kind, int has_ln, double ln_in, int pad, int farfield, cudaStream_t s) {
    if (solve_small_ok(g, pad)) {  // the whole system fits in shared memory
        k_solve_small(g, F5, F7, src, dst, ln_out, kind, has_ln, ln_in, pad, farfield, s);
        return;
    }
    const int wpad = kind == 0 ? 0 : (32 - (2 * g.NXCHOPDIM) % 32) % 32;
    const int n = 2 * g.NTCHOPDIM * g.NXCHOPDIM + wpad;
    solve_factored_kernel<<<(n + 127) / 128, 128, 0, s>>>(g, F5, F7, src, dst, ln_out, kind, has_ln, ln_in, pad,
                                                          farfield, wpad);
    count_launch();
}

void k_solve_del2(const DevGrid& g, double2* a, double* ln_out, int kind, double alp, int has_ln, double ln_in,
                  const double* b_ln, double* scratch, int pad, cudaStream_t s) {
    int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    solve_kernel<<<(nsys + 63) / 64, 64, 0, s>>>(g, a, ln_out, kind, alp, has_ln, ln_in, b_ln, scratch, pad);
    count_launch();
}

// ---------------------------------------------------------------------------
// IHELMP (mod_legops.f90:1409-1592), the implicit hyperviscosity solve of
// HYPERV (VISC%SW = 2, mod_march.f90:1639-1686): per (m, k) the system
//   H = (DEL2H - k^2)^(P/2) + NU (DEL2H - k^2) - ALP
// of half-bandwidth P on the leading NN = NRCHOP + pad - m rows.  H's rows are
// formed from the powers D^q of the DEL2H band (table dq, built on the host
// with BANBANMUL's summation order), combined binomially as the reference
// writes them out for each P (D^(P/2) - C(P/2,1) k^2 D^(P/2-1) + ... ), then
// eliminated without pivoting, one thread per (m, k), the U rows in scratch
// [row][P+1][system], the right-hand side in place.  The (m, k) = (0, 0)
// thread first moves the log term's contribution to the right-hand side:
// rows -= AL + NU AL2, AL2 the DEL2 image of LN (-log(1-x)) and AL = D^(P/2-1) AL2.
// dq layout: [m][q = 1..HP][row < rows][4q + 1], q's block at rows (q - 1)(2q + 1)
// within the m block of rows HP (2 HP + 3) doubles.
template <int HP>
__global__ void ihelmp_kernel(DevGrid g, const double* dq, int rows, double2* A, const double* ln, double alp,
                              double nu, double* scratch, int pad) {
    constexpr int P = 2 * HP, W = 2 * P + 1;
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsys) return;
    const int k = t % g.NXCHOPDIM;
    const int m = t / g.NXCHOPDIM;
    int nn = g.NRCHOP + pad - m;
    if (nn > rows) nn = rows;
    if (nn <= 0) return;
    const double K2 = g.ak[k] * g.ak[k];
    const size_t mstride = (size_t)rows * HP * (2 * HP + 3);  // rows * sum_{q <= HP} (4q + 1)
    const double* dm = dq + (size_t)m * mstride;
    // q's block starts after rows * sum_{q' < q} (4q' + 1) = rows (q - 1)(2q + 1)
    auto dq_row = [&](int q, int r) { return dm + (size_t)rows * (q - 1) * (2 * q + 1) + (size_t)r * (4 * q + 1); };
    double2* col = A + (size_t)m * g.NRCHOPDIM * g.NXCHOPDIM + k;
    const size_t st = g.NXCHOPDIM;
    if (m == 0 && k == 0) {
        // log term (1444-1466): A%LN was set to -B%LN/ALP by the caller
        const int nr = g.NRCHOP + pad;
        const double L = *ln;
        double al2[P + 3], al[P + 3], y[P + 3];
        for (int i = 0; i < P + 3; ++i) al2[i] = 0.0;
        al2[0] = L * (4.0 / 3 / g.ELL2) / g.norm0[0];
        al2[1] = L * (-2 / g.norm0[1] / g.ELL2);
        al2[2] = L * (+2.0 / 3 / g.norm0[2] / g.ELL2);
        for (int i = 0; i < P + 3; ++i) al[i] = al2[i];
        const double* d2 = g.del2h;  // m = 0 rows, [row][5]
        for (int rep = 1; rep < HP; ++rep) {  // BANMUL(DEL2H, 3, AL), band index ascending
            for (int r = 0; r < P + 3; ++r) {
                double v = 0.0;
                for (int e = 0; e < 5; ++e) {
                    const int c = r + e - 2;
                    if (r < nr && c >= 0 && c < nr && c < P + 3) v += d2[(size_t)r * 5 + e] * al[c];
                }
                y[r] = v;
            }
            for (int r = 0; r < P + 3; ++r) al[r] = y[r];
        }
        for (int r = 0; r < P + 3 && r < nr; ++r) {
            double2 v = col[(size_t)r * st];
            v.x -= al[r] + nu * al2[r];
            col[(size_t)r * st] = v;
        }
    }
    // forward elimination, left-looking per row (the pivot rows come from scratch)
    for (int r = 0; r < nn; ++r) {
        double w[W];
        const double* top = dq_row(HP, r);
#pragma unroll
        for (int e = 0; e < W; ++e) w[e] = top[e];
        double c = 1.0;
#pragma unroll
        for (int j = 1; j <= HP; ++j) {
            c *= -K2;
            // binomial coefficient C(HP, j)
            double bin = 1.0;
            for (int q = 1; q <= j; ++q) bin = bin * (HP - q + 1) / q;
            const int q = HP - j;
            if (q == 0) {
                w[P] += c;
            } else {
                const double* dr = dq_row(q, r);
                const double f = bin * c;
                for (int e = 0; e <= 4 * q; ++e) w[P - 2 * q + e] += f * dr[e];
            }
        }
        {
            const double* d1 = dq_row(1, r);
            for (int e = 0; e < 5; ++e) w[P - 2 + e] += nu * (e == 2 ? d1[e] - K2 : d1[e]);
        }
        w[P] -= alp;
        double2 rhs = col[(size_t)r * st];
        for (int d = P; d >= 1; --d) {
            if (r - d < 0) continue;
            const double* u = scratch + (size_t)(r - d) * (P + 1) * nsys + t;
            const double f = w[P - d] / u[0];
            w[P - d] = 0.0;
            for (int j = 1; j <= P; ++j) {
                const int qq = P - d + j;
                if (qq < W) w[qq] -= f * u[(size_t)j * nsys];
            }
            const double2 pr = col[(size_t)(r - d) * st];
            rhs.x -= f * pr.x;
            rhs.y -= f * pr.y;
        }
        double* ur = scratch + (size_t)r * (P + 1) * nsys + t;
        for (int j = 0; j <= P; ++j) ur[(size_t)j * nsys] = w[P + j];
        col[(size_t)r * st] = rhs;
    }
    // back substitution
    for (int r = nn - 1; r >= 0; --r) {
        const double* ur = scratch + (size_t)r * (P + 1) * nsys + t;
        double2 v = col[(size_t)r * st];
        for (int j = 1; j <= P && r + j < nn; ++j) {
            const double u = ur[(size_t)j * nsys];
            const double2 x = col[(size_t)(r + j) * st];
            v.x -= u * x.x;
            v.y -= u * x.y;
        }
        v.x /= ur[0];
        v.y /= ur[0];
        col[(size_t)r * st] = v;
    }
}

size_t ihelmp_scratch_doubles(const DevGrid& g, int P) {
    return (size_t)g.NRCHOPDIM * (P + 1) * g.NTCHOPDIM * g.NXCHOPDIM;
}

void k_ihelmp(const DevGrid& g, int P, const double* dq, int rows, double2* a, const double* ln, double alp,
              double nu, double* scratch, int pad, cudaStream_t s) {
    const int nsys = g.NTCHOPDIM * g.NXCHOPDIM;
    const int bs = 128, nb = (nsys + bs - 1) / bs;
    switch (P) {
        case 4: ihelmp_kernel<2><<<nb, bs, 0, s>>>(g, dq, rows, a, ln, alp, nu, scratch, pad); break;
        case 6: ihelmp_kernel<3><<<nb, bs, 0, s>>>(g, dq, rows, a, ln, alp, nu, scratch, pad); break;
        case 8: ihelmp_kernel<4><<<nb, bs, 0, s>>>(g, dq, rows, a, ln, alp, nu, scratch, pad); break;
        case 10: ihelmp_kernel<5><<<nb, bs, 0, s>>>(g, dq, rows, a, ln, alp, nu, scratch, pad); break;
        case 12: ihelmp_kernel<6><<<nb, bs, 0, s>>>(g, dq, rows, a, ln, alp, nu, scratch, pad); break;
        default: ihelmp_kernel<7><<<nb, bs, 0, s>>>(g, dq, rows, a, ln, alp, nu, scratch, pad); break;
    }
    count_launch();
}

// Grouped factored substitutions over the instances of an ensemble: each
// block belongs to one problem (found by binary search over `first`), 64
// systems per block.
__global__ void __launch_bounds__(128) grouped_solve_kernel(const GroupSolve* __restrict__ pr,
                                                            const int* __restrict__ first, int np) {
    const int b = blockIdx.x;
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const GroupSolve P = pr[lo];
    // the 7-band m = 0 systems in whole warps, as in solve_factored_kernel
    int u = (b - P.first) * 128 + threadIdx.x;
    const int nw = 2 * P.g.NXCHOPDIM, wpad = P.kind == 0 ? 0 : (32 - nw % 32) % 32;
    if (u >= nw && u < nw + wpad) return;
    if (u >= nw) u -= wpad;
    solve_factored_sys<8>(P.g, P.F5, P.F7, P.src, P.dst, P.ln_out, P.kind, P.has_ln, P.ln_in, P.pad, P.farfield, u);
}

int group_solve_blocks(const GroupSolve& p) {
    const int nw = 2 * p.g.NXCHOPDIM, wpad = p.kind == 0 ? 0 : (32 - nw % 32) % 32;
    return (2 * p.g.NTCHOPDIM * p.g.NXCHOPDIM + wpad + 127) / 128;
}

void k_grouped_solve(const GroupSolve* d, const int* first, int np, int total_blocks, cudaStream_t s) {
    grouped_solve_kernel<<<total_blocks, 128, 0, s>>>(d, first, np);
    count_launch();
}

}  // namespace mlegs
