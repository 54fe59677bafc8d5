// Internal declarations of the B200 MLegS library (not part of the C ABI).
//
// Device layouts (0-based, all complex values are double2 = (re, im)):
//   FFF  [m][n][k]  (NTCHOPDIM, NRCHOPDIM, NXCHOPDIM)   k fastest
//   PFF  [m][r][k]  (NTCHOPDIM, NR,        NXCHOPDIM)
//   PFP  [r][z][m]  (NR,        NX,        NTCHOPDIM)
//   PPP  [r][z][j]  (NR,        NX,        NTH)  packed samples: re -> theta_{2j},
//                                                 im -> theta_{2j+1} (mod_fft.f90:844-848)
// The reference's zero padding (rows NR+1..NR+3, theta column NTH+1, chopped
// m/k) is not stored; upload/download map to and from the Fortran layout.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mlegs_b200.h"

namespace mlegs {

struct Dims {
    int NR, NRH, NTH, NX, NRCHOP, NTCHOP, NXCHOP;
    int NDIMR, NDIMTH, NRCHOPDIM, NTCHOPDIM, NXCHOPDIM, NXCHOPH, NLN;
    double ELL, ELL2, ZLEN;
    size_t fff() const { return (size_t)NTCHOPDIM * NRCHOPDIM * NXCHOPDIM; }
    size_t pff() const { return (size_t)NTCHOPDIM * NR * NXCHOPDIM; }
    size_t pfp() const { return (size_t)NR * NX * NTCHOPDIM; }
    size_t ppp() const { return (size_t)NR * NX * NTH; }
    size_t elems(int space) const {
        switch (space) {
            case MLEGS_FFF: return fff();
            case MLEGS_PFF: return pff();
            case MLEGS_PFP: return pfp();
            default: return ppp();
        }
    }
    size_t cap() const {
        size_t c = fff();
        if (pff() > c) c = pff();
        if (pfp() > c) c = pfp();
        if (ppp() > c) c = ppp();
        return c;
    }
};

// Device-side copy of the grid constants passed to kernels by value.
struct DevGrid {
    int NR, NRH, NTH, NX, NRCHOP, NTCHOP, NXCHOP;
    int NRCHOPDIM, NTCHOPDIM, NXCHOPDIM, NLN;
    double ELL2;
    const double* x;        // [NR] Gauss-Legendre nodes (ascending)
    const double* w;        // [NR] weights
    const double* r;        // [NR] mapped radii
    const double* lnx;      // [NR] -log(1-x)
    const double* pf;       // [NTCHOPDIM][NRCHOPDIM+1][NRH]
    const double* ak;       // [NXCHOPDIM] axial wavenumbers (AK(m,k) is m-independent)
    const double* norm0;    // [NLN] NORM(:, m=0)
    const double* at1;      // [NRCHOPDIM] Pbar_n(+1)
    // band tables per (m, n), n < NRCHOPDIM+1 (row index of the band):
    const double* xxdx;     // [NTCHOPDIM][NB][2]  (sub, super)
    const double* xm;       // [NTCHOPDIM][NB][2]  (sub, super)     diag = 1
    const double* del2h;    // [NTCHOPDIM][NB][5]
    int NB;                 // NRCHOPDIM + 2
};

struct Field {
    double2* data = nullptr;   // current buffer (capacity Dims::cap())
    double2* home = nullptr;   // buffer owned at allocation time
    double* ln = nullptr;      // device scalar LN (mod_scalar3.f90:43)
    int space = MLEGS_FFF;
    int slot = -1;
    bool persistent = false;
};

// Kernel launch helpers (kernels.cu, fft.cu, gemm.cu, solve.cu, tables.cu).
void k_tables_gauss(double* x, double* w, int n, cudaStream_t s);
void k_tables_pf(const double* x, double* pf, int nrh, int ne, int ntchopdim, cudaStream_t s);
void k_tables_project(const DevGrid& g, double* V, double* D, double* T, int pad, cudaStream_t s);

void fft_set_attributes();
void k_fill(double2* p, size_t n, cudaStream_t s);
void k_copy(double2* dst, const double2* src, size_t n, cudaStream_t s);
void k_chopdo_fff(const DevGrid& g, double2* a, int pad, cudaStream_t s);
void k_copy_ln(double2* dst, const double2* src, size_t n, double* dln, const double* sln, cudaStream_t s);
void k_axpby_ln(double2* y, double a, const double2* x1, double b, const double2* x2, double c, size_t n, double* yl,
                double la, const double* l1, double lb, const double* l2, double lc, cudaStream_t s);
void k_copy_chop_fff(const DevGrid& g, double2* dst, const double2* src, double* dln, const double* sln, int pad,
                     cudaStream_t s);

// Legendre transforms (FP64 and split-BF16 tensor-core forms).
// Split-BF16 tensor-core forms (split_gemm.cu).  mode 0: RTRAN(+1) images from
// PF; mode 1: fold images from a weight table Wt[m][n][i] with wt_rows rows.
bool split_supported(const DevGrid& g, int S, int wt_rows);
size_t split_image_bytes(const DevGrid& g, int S, int mode, int wt_rows);
void k_split_prepare(const DevGrid& g, int S, int mode, const double* W, int wt_rows, uint8_t* img, int* eA,
                     cudaStream_t s);
void k_split_b2p(const DevGrid& g, int S, const uint8_t* img, const int* eA, const double2* a, double2* b,
                 const double* ln, int pad, int* err, uint64_t wait_cycles, cudaStream_t s);
// Same contract as k_fold_gemm (mode bit 0 = EO/OE, use_w separate).  wait_cycles:
// limit of the kernel's pipeline waits in SM cycles (0: the default, about a second);
// a wait that runs out sets *err and the kernel returns early.
void k_split_fold(const DevGrid& g, int S, const uint8_t* img, const int* eA, int wt_rows, const double2* in,
                  double2* out, int mode, int scale, int accumulate, int pad, int use_w, int* err,
                  uint64_t wait_cycles, cudaStream_t s);
void k_rtran_b2p(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s);
// Fold GEMM arguments (gemm_dmma.cu): RTRAN(-1) and PROJECT's five EOMUL/OEMUL
// products as K-concatenated segments.
struct FoldArgs {
    const double* w[5];  // weights per segment, [m][wt_rows][NRH]
    const double* x[5];  // inputs per segment, PFF [m][NR][2 NXCHOPDIM]
    int mode[5];         // 0: EO fold, 1: OE fold
    int scale[5];        // 0 none, 1 -v, 2 -i m v, 3 i k v, 4 m k v
    int nseg, split;     // segments [0, split) -> out0, [split, nseg) -> out1
    double* out0;
    double* out1;
    int wt_rows, pad, use_w, accumulate;
};
// Grouped persistent GEMMs over the instances of an ensemble (gemm_dmma.cu):
// one problem per (instance, transform); `first` = its first tile number;
// nj = 2 or 4 (column tiles of 8 nj columns).  *_prepare fills SA/RTmax and
// ntx and returns the problem's tile count; *_smem its shared memory.
struct GroupB2P {
    DevGrid g;
    const double* in;
    double* out;
    const double* ln;
    int pad, SA, nj, ntx, first;
};
struct GroupFold {
    DevGrid g;
    FoldArgs fa;
    int RTmax, nj, ntx, first;
};
bool group_supported(const DevGrid& g);
int group_b2p_prepare(GroupB2P& p);
size_t group_b2p_smem(const GroupB2P& p);
int group_fold_prepare(GroupFold& p);
size_t group_fold_smem(const GroupFold& p);
void k_grouped_b2p(const GroupB2P* d, const int* first, int np, int total, size_t smem, int ctas, int* next,
                   cudaStream_t s);
void k_grouped_fold(const GroupFold* d, const int* first, int np, int total, size_t smem, int ctas, int* next,
                    cudaStream_t s);
// Grouped banded substitutions (solve.cu): one problem per (instance, solve);
// 64 systems (128 threads: real and imaginary parts) per block, `first` =
// the problem's first block.
struct GroupSolve {
    DevGrid g;
    const double* F5;
    const double* F7;
    const double2* src;
    double2* dst;
    double* ln_out;
    int kind, has_ln;
    double ln_in;
    int pad, farfield, first;
};
int group_solve_blocks(const GroupSolve& p);
void k_grouped_solve(const GroupSolve* d, const int* first, int np, int total_blocks, cudaStream_t s);
// RTRAN(+1) with bulk-copy staging and a warp-specialised mbarrier pipeline
// (gemm_bulk.cu), the form k_rtran_b2p takes when supported; a timed-out
// wait raises the module's error word, read (and cleared) by bulk_gemm_error.
bool b2p_bulk_supported(const DevGrid& g);
// FP64 tensor-path ceiling microbenchmark (register-only MMAs); FLOPs per launch
double k_dmma_peak(double* out, cudaStream_t s);
double dmma_peak_flops();
void k_rtran_b2p_bulk(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s);
int bulk_gemm_error(bool reset);
// Fold GEMMs (RTRAN(-1), PROJECT's products) on the same pipeline: weight
// tables re-laid per (m, parity, 16-row chunk) by k_fold_table (times w_i when
// use_w), then k_fold_bulk over nseg segments (mode / scale as in FoldArgs;
// segments [0, split) -> out0, the rest -> out1).
int fold_table_rows(const DevGrid& g, int wt_rows);
size_t fold_table_doubles(const DevGrid& g, int wt_rows);
void k_fold_table(const DevGrid& g, const double* W, int wt_rows, int use_w, double* Wc, cudaStream_t s);
bool fold_bulk_supported(const DevGrid& g, int wt_rows);
void k_fold_bulk(const DevGrid& g, const double* const* wc, const double2* const* x, const int* mode,
                 const int* scale, int nseg, int split, double2* out0, double2* out1, int wt_rows, int pad,
                 int accumulate, cudaStream_t s);
// FP64 tensor-path (mma.sync m8n8k4.f64) forms used by k_rtran_b2p / k_fold_gemm when supported.
bool dmma_supported(const DevGrid& g);
void k_rtran_b2p_dmma(const DevGrid& g, const double2* a, double2* b, const double* ln, int pad, cudaStream_t s);
void k_fold_gemm_dmma(const DevGrid& g, const double* Wt, int wt_rows, const double2* in, double2* out, int mode,
                      int scale, int accumulate, int pad, cudaStream_t s);
// PROJECT's five fold products in one launch (FP64 tensor path): PSI and CHI from
// RUR, RUP, UZ in PFF with the weights V, D, T ([m][n][i], NRCHOPDIM x NRH).
void k_project_dmma(const DevGrid& g, const double* V, const double* D, const double* T, const double2* rur,
                    const double2* rup, const double2* uz, double2* psi, double2* chi, cudaStream_t s);
// PROJECT of FFF velocity fields through per-m composite matrices
// Comp_W = 2 W . PF^T restricted to one input-row parity (gemm_dmma.cu):
// k_proj_comp forms one ([m][pr][r][t], proj_comp_doubles entries; p_flip 0
// for the EO weights V, T, 1 for the OE weight D); k_project_fff_dmma runs
// VEL2PLN on RUP's (0, 0) column (in place, PSI%LN <- PLN) and then the
// products.  Input LN terms must be zero.
size_t proj_comp_doubles(const DevGrid& g);
void k_proj_comp(const DevGrid& g, const double* W, int p_flip, double* Cm, cudaStream_t s);
void k_project_fff_dmma(const DevGrid& g, const double* CV, const double* CD, const double* CT, double2* rur,
                        double2* rup, double2* uz, double2* psi, double2* chi, double* psi_ln, const double* Lfff,
                        cudaStream_t s, double* chi_ln = nullptr);
// out[m][n][k] (+)= scale(m,k) * sum_i Wt[m][n][i] * fold(in)(i,k); fold parity per row given by mode
//   mode 0 (EO): row n even -> even fold, odd -> odd fold;  mode 1 (OE): swapped
//   scale: 0 -> 1, 1 -> -1, 2 -> -i m, 3 -> i k, 4 -> m k
void k_fold_gemm(const DevGrid& g, const double* Wt, int wt_rows, const double2* in, double2* out,
                 int mode, int scale, int accumulate, int pad, cudaStream_t s);

// FFTs.
struct FFTPlan {
    double2* tw_x = nullptr;     // exp(-2 pi i q / NX), q < NX
    double2* tw_t = nullptr;     // exp(-2 pi i q / NTH), q < NTH
    double2* tw_h = nullptr;     // exp(-i pi q / NTH),  q <= NTH (real-FFT post-processing)
    int lx = 0, lt = 0;          // log2 NX, log2 NTH
};
void k_verfft_b(const DevGrid& g, const FFTPlan& p, const double2* pff, double2* pfp, cudaStream_t s);
void k_verfft_f(const DevGrid& g, const FFTPlan& p, const double2* pfp, double2* pff, cudaStream_t s);
void k_horfft_b(const DevGrid& g, const FFTPlan& p, const double2* pfp, double2* ppp, cudaStream_t s);
void k_horfft_f(const DevGrid& g, const FFTPlan& p, const double2* ppp, double2* pfp, cudaStream_t s);

// Fused physical stage (phys.cu): 9 (10 with linear terms) PFP inputs -> 4 PFP outputs.
void phys_set_attributes();
void k_theta_fused(const DevGrid& g, const FFTPlan& p, const double2* const in[10], double2* const out[4],
                   double omega, double bv0, int linear, cudaStream_t s);
void k_horfft_warp(const DevGrid& g, const FFTPlan& p, const double2* src, double2* dst, int dir, cudaStream_t s);
// Four-step VERFFT (dir +1: PFF -> PFP, -1: PFP -> PFF); false if NX has no specialisation.
bool k_verfft4(const DevGrid& g, const FFTPlan& p, const double2* src, double2* dst, int dir, cudaStream_t s);

// Spectral operators on FFF.
void k_delsqh(const DevGrid& g, const double2* a, const double* ln_a, double2* b, int pad, cudaStream_t s);
void k_idelsqh(const DevGrid& g, const double2* b, double2* a, int pad, cudaStream_t s);
void k_band3(const DevGrid& g, const double2* a, double2* b, int which /*0 xxdx, 1 xm*/, int pad, cudaStream_t s);
void k_del2(const DevGrid& g, const double2* a, double2* b, int pad, cudaStream_t s);
void k_logterm_rows(const DevGrid& g, double2* b, const double* ln, int which, double coef, cudaStream_t s);
void k_mk_combine(const DevGrid& g, int op, const double2* x, const double2* y, double2* out, int pad, cudaStream_t s);
// GRAD, PC2VEL, PC2VOR each in one pass (kernels.cu); outputs FFF, log terms read from *ln.
void k_grad_fused(const DevGrid& g, const double2* a, const double* ln, double2* rr, double2* rp, double2* gz, int pad,
                  cudaStream_t s);
void k_pc2vel_fused(const DevGrid& g, const double2* psi, const double* psi_ln, const double2* chi, const double* chi_ln,
                    double2* rur, double2* rup, double2* uz, int pad, cudaStream_t s, int sub = 0,
                    double* const* zero_ln = nullptr);
void k_pc2vor_fused(const DevGrid& g, const double2* psi, const double* psi_ln, const double2* chi, const double* chi_ln,
                    double2* ror, double2* rop, double2* oz, int pad, cudaStream_t s);
void k_farfield_fix(const DevGrid& g, double2* a, int nr_sum, cudaStream_t s, int by_pf = 0);
// IHELMP (solve.cu): dq = DEL2H power tables [m][q][rows][4q+1], scratch of
// ihelmp_scratch_doubles(g, P) doubles; a is solved in place, ln = A%LN.
size_t ihelmp_scratch_doubles(const DevGrid& g, int P);
void k_ihelmp(const DevGrid& g, int P, const double* dq, int rows, double2* a, const double* ln, double alp,
              double nu, double* scratch, int pad, cudaStream_t s);
// VEL2PLN through its coefficient vectors (k_vel2pln_coef, once per context):
// on the PFF line of RUP (Lpff, NR entries), or on RUP's FFF (0, 0) column
// (Lfff, NRCHOP entries; mode 0, applied to that column).
void k_vel2pln_coef(const DevGrid& g, const double* explog0, int nn, double* Lpff, double* Lfff, cudaStream_t s);
// zero_ln (optional): one more LN slot set to 0 by the same launch.
void launch_vel2pln(const DevGrid& g, double2* rup_pff, double* psi_ln, int mode, double ln, const double* Lpff,
                    cudaStream_t s, double* zero_ln = nullptr);
void launch_vel2pln_fff(const DevGrid& g, double2* rup_fff, double* psi_ln, const double* Lfff, cudaStream_t s,
                        double* zero_ln = nullptr);

// Banded solves (IDEL2LN, IDEL2, IHELM) with per-system elimination scratch.
void k_solve_del2(const DevGrid& g, double2* a, double* ln_out, int kind, double alp, int has_ln,
                  double ln_in, const double* b_ln, double* scratch, int pad, cudaStream_t s);
// Factor-once form of the same solves (solve.cu): LU factors of every (m, k)
// system for one (kind, pad, alp), then substitutions only; src -> dst with
// rows past the system size zeroed, farfield = 1 adds the CALCAT1 row-0 fix.
void solve_factor_sizes(const DevGrid& g, size_t* f5, size_t* f7);
void k_solve_factor(const DevGrid& g, int kind, double alp, int pad, double* F5, double* F7, cudaStream_t s);
void k_solve_factored(const DevGrid& g, const double* F5, const double* F7, const double2* src, double2* dst,
                      double* ln_out, int kind, int has_ln, double ln_in, int pad, int farfield, cudaStream_t s);
// Fixed __device__ solve scratch (solve_static.cu) for the allocation-free
// IDEL2LN entry point: returns 0 and its address on `device` (the current
// device), 1 if need_doubles exceeds kStaticSolveBytes, 2 on a CUDA error;
// `msg` receives the reason.
extern const size_t kStaticSolveBytes;
int static_solve_scratch(int device, size_t need_doubles, double** out, char* msg, size_t msg_len);

// Pointwise physics in PPP.
void k_force_pointwise(const DevGrid& g, double2* rur, double2* rup, double2* uz, double2* ror,
                       double2* rop, double2* oz, const double2* rbr, const double2* rbp,
                       const double2* bz, double2* bn, const double2* bphys, double omega,
                       double bv0, int linear, cudaStream_t s);

// Per-(m, k) quadratures of PFF fields (kernels.cu): mode 0 the PRODCT_MK_ALLK
// sum of Re(A conj B) w, mode 1 the L2NORM_MK_ALLK sum of |A|^2 w / (1 - x)^2,
// times scale, into out[m][k] (NTCHOPDIM x NXCHOPDIM, m = 0 not yet halved).
void k_prodct_mk(const DevGrid& g, const double2* A, const double2* B, int mode, double scale, double* out,
                 cudaStream_t s);

// FFF-space updates.
void k_axpby(double2* y, double a, const double2* x1, double b, const double2* x2, double c,
             size_t n, cudaStream_t s);
void k_ln_axpby(double* y, double a, const double* x1, double b, const double* x2, double c, cudaStream_t s);
void k_ln_set(double* y, double v, cudaStream_t s);
void k_ln_copy(double* y, const double* x, double scale, cudaStream_t s);
void k_etd(const DevGrid& g, const double* E, const double* NL, double dt, int ab2,
           double2* rur, double2* rup, double2* uz, double2* b,
           const double2* rnr, const double2* rnp, const double2* nz, const double2* nb,
           const double2* hr, const double2* hp, const double2* hz,
           const double2* onr, const double2* onp, const double2* onz, const double2* onb,
           cudaStream_t s);
// One-pass ETD2AB coefficient update of the steady step (kernels.cu).
struct EtdAbArgs {
    const double* E;  // 4 x 4 real ETD matrices, row-major
    const double* N;
    double dt;
    int hyper;              // apply the VISC%SW = 3 filters (hv: velocity, hd: buoyancy)
    const double* hv[3];    // [m][n] (NRCHOP per m), [m], [k]
    const double* hd[3];
    const double2* psi;     // state read for PC2VEL
    const double2* chi;
    const double* psi_ln;
    const double* chi_ln;
    double2* rur;           // out: updated velocity terms
    double2* rup;
    double2* uz;
    double2* b;             // in/out
    const double2* ror;     // projected nonlinear terms of this step (used when npsi is null)
    const double2* rop;
    const double2* oz;
    const double2* npsi;    // or: their PSI_N, CHI_N (FFF), PC2VEL formed in the kernel
    const double2* nchi;
    const double* npsi_ln;
    const double* nchi_ln;
    const double2* bn;
    double2* hist[7];       // in/out: 0 N_B, 1 R_N_R, 2 R_N_P, 3 N_Z, 4 R_PI_R, 5 R_PI_P, 6 PI_Z
    double* out_ln[3];      // LN slots of rur, rup, uz: set to 0 (PC2VEL outputs carry no log term)
    int raw_out;            // 1: outputs unfiltered and R_PI_* not written (the sponge comes between)
};
// CALC_BOUSSI_ETD_SPONGE's damping of one PFP field by damp[z] (NX entries).
void k_sponge(const DevGrid& g, double2* a, const double* damp, cudaStream_t s);
// Adaptive hyperviscosity state of VISC (mod_march.f90:74-76) and its host code (hyperadj.cu).
struct Hyp3State {
    double nupb = -1.0, kappapb = -1.0;
    double hist[4] = {0, 0, 0, 0};    // CURVMO CURVKO SLOPMO SLOPKO
    double phist[4] = {0, 0, 0, 0};   // PCURVMO PCURVKO PSLOPMO PSLOPKO
};
double specurv(const double* e, int size, double use_ratio);
double speslop(const double* e, int size, double ratio);
double pdajust(double coeff, double current, double previous, double baseline, const double params[4],
               bool has_threshold, double threshold);
void hyp3adj_update(Hyp3State& st, const double* em, int nm, const double* ek, int nk, double nup[3],
                    const double* pm, int npm, const double* pk, int npk, double kap[3]);
void k_lay_gaus(const DevGrid& g, double zlen, const mlegs_vortex* v, int nv, const double* q, const double* b,
                double2* a, cudaStream_t s);
void k_maxabs(const double2* a, size_t n, int mode, double* out, cudaStream_t s);
void k_noise(const DevGrid& g, double2* a, const double* refmax, double alevel, double akmax, long long v0,
             cudaStream_t s);
void k_flatten(const DevGrid& g, double2* a, const double2* b, const double* refmax, cudaStream_t s);
void k_absvec2(const DevGrid& g, const double2* u, const double2* v, const double2* w, double2* a, cudaStream_t s);
void k_mulr(const DevGrid& g, const double2* src, double2* dst, int mode, cudaStream_t s);
void k_etd_ab_fused(const DevGrid& g, const EtdAbArgs& a, cudaStream_t s);
void k_hyperv(const DevGrid& g, double2* a, const double* hr, const double* ht, const double* hx,
              double tf, int pad, cudaStream_t s);
void k_finite(const double2* a, size_t n, int* flag, cudaStream_t s);

// Layout conversion between the reference's Fortran arrays and device layouts.
void k_from_ref(const DevGrid& g, int space, const double2* ref, double2* dev, cudaStream_t s);
void k_to_ref(const DevGrid& g, int space, const double2* dev, double2* ref, cudaStream_t s);

extern thread_local int64_t* g_launch_counter;
inline void count_launch() {
    if (g_launch_counter) ++(*g_launch_counter);
}

}  // namespace mlegs
