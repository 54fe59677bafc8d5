// Host-side internals of the library shared by the C ABI translation units
// (ctx.cu: contexts and fields; ensemble.cu: grouped ensembles): the error
// types, the device allocator that records every allocation of a context,
// the context and field structures and the ABI guard.
#pragma once

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <algorithm>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlegs_internal.h"

using namespace mlegs;

namespace mlegs_host {

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
struct ApiError : std::runtime_error {
    int code;
    ApiError(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            throw mlegs_host::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Every device allocation of a context is recorded here and released in one
// place, whatever field or scratch slot currently points at it.
extern thread_local std::vector<void*>* g_allocs;

template <class T>
T* dalloc(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) throw ApiError(MLEGS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    if (g_allocs) g_allocs->push_back(p);
    return (T*)p;
}

}  // namespace mlegs_host

using namespace mlegs_host;

struct mlegs_field {
    Field f;
    mlegs_ctx* owner;
};

struct mlegs_ctx {
    mlegs_params p{};
    Dims d{};
    DevGrid g{};
    cudaStream_t s = nullptr;
    cudaStream_t s2 = nullptr;         // second stream of the RTRAN(+1) -> VERFFT(+1) pipeline
    cudaEvent_t evs[64] = {};          // fork/join events, used in rotation
    int ev_next = 0;
    double2* pbuf[3] = {};             // PFF images in flight between the two stages
    int dev = 0;
    std::string err;
    int64_t launches = 0;
    int64_t graph_launches = 0;   // kernels in one captured step
    std::vector<void*> allocs;

    // device tables
    double *x = nullptr, *w = nullptr, *r = nullptr, *lnx = nullptr, *pf = nullptr, *ak = nullptr;
    double *norm0 = nullptr, *explog0 = nullptr, *at1 = nullptr, *tb_xxdx = nullptr, *tb_xm = nullptr,
           *tb_del2h = nullptr;
    double *V = nullptr, *D = nullptr, *T = nullptr;
    double *hv[3] = {nullptr, nullptr, nullptr}, *hd[3] = {nullptr, nullptr, nullptr};
    // HYP3SET masks (VISC%MASK_R/T/X) and the adaptive state of VISC
    // (mod_march.f90:70-86): NUP_R/T/X, KAPPAP_R/T/X, the controllers' history.
    std::vector<double> h3_mr, h3_mt, h3_mx, h3_ak;
    double nup3[3] = {0, 0, 0}, kap3[3] = {0, 0, 0};
    Hyp3State adj;
    double *compV = nullptr, *compD = nullptr, *compT = nullptr;  // PROJECT composites (FP64 contexts)
    // chunked weight tables of the bulk fold GEMMs (FP64 contexts): PF times w_i
    // (RTRAN(-1)) and V, D, T (PROJECT of PFF inputs)
    double *fc_pf = nullptr, *fc_V = nullptr, *fc_D = nullptr, *fc_T = nullptr;
    double *v2p_pff = nullptr, *v2p_fff = nullptr;                 // VEL2PLN coefficient vectors
    double* diag = nullptr;                                         // 4 x [m][k] quadratures (energy)
    double *sp_damp = nullptr, *sp_damp_h = nullptr;                // sponge factors for DT and DT/2 (RMV%SW = 2)
    double *etdE = nullptr, *etdN = nullptr, *hetdE = nullptr, *hetdN = nullptr;
    FFTPlan fft;
    std::vector<double> h_x, h_w, h_lognorm;

    // memory
    double* lnslots = nullptr;
    int nslots = 0, used_slots = 0;
    double2* scratch = nullptr;
    double* solve_scr = nullptr;
    // split-BF16 tensor-core GEMMs (MLEGS_PREC_SPLIT)
    int split_S = 0;                 // slices per operand; 0 = FP64 GEMMs
    uint8_t* split_img = nullptr;    // PF slice images for RTRAN(+1)
    int* split_eA = nullptr;         // PF row scale exponents
    int* split_err = nullptr;        // raised by a timed-out wait in a tensor-core kernel
    uint64_t split_wait = 0;         // limit of those waits in SM cycles (0: the kernel's default)
    uint8_t* fimg[4] = {};           // weight slice images: 0 PF (RTRAN -1), 1 V, 2 D, 3 T (PROJECT)
    int* feA[4] = {};
    // out (+)= s Wt . fold(in): FP64 kernel, or the split tensor-core kernel when enabled
    void fold(int w, const double* Wt, int wt_rows, const double2* in, double2* out, int mode, int scale,
              int accumulate, int pad, cudaStream_t st = nullptr) {
        if (!st) st = s;
        if (split_S) {
            k_split_fold(g, split_S, fimg[w], feA[w], wt_rows, in, out, mode & 1, scale, accumulate, pad,
                         (mode & 2) ? 1 : 0, split_err, split_wait, st);
            return;
        }
        // RTRAN(-1) (PF with the Gauss weights) on the bulk-copy pipeline when its table exists
        if (w == 0 && (mode & 2) && Wt == pf && fc_pf) {
            const double* wc[1] = {fc_pf};
            const double2* x[1] = {in};
            const int md[1] = {mode & 1}, sc[1] = {scale};
            k_fold_bulk(g, wc, x, md, sc, 1, 1, out, nullptr, wt_rows, pad, accumulate, st);
            return;
        }
        k_fold_gemm(g, Wt, wt_rows, in, out, mode, scale, accumulate, pad, st);
    }
    double2* staging = nullptr;
    // mlegs_run_host, set up on its first call: copy streams each way, staging
    // per state field and direction, page-locked LN slots, and the events per
    // field i "uploaded" [i], "converted for download" [3 + i] and, per chunk j
    // of its download, "downloaded" [6 + IO_CHUNKS i + j]
    static constexpr int IO_CHUNKS = 4;
    cudaStream_t s_up = nullptr, s_down = nullptr;
    double2* io_in[3] = {};
    double2* io_out[3] = {};
    double* io_ln = nullptr;
    cudaEvent_t io_ev[6 + 3 * IO_CHUNKS] = {};
    int* dflag = nullptr;
    std::vector<std::unique_ptr<mlegs_field>> owned;  // every field, incl. user ones
    std::vector<Field*> pool;                         // free temporaries (stack)
    std::vector<Field*> temps;                        // all temporaries
    Field* hist[7] = {};

    // adjoint (adjoint.cu), formed on first use: the grid with transposed band
    // tables, PROJECT's weights in PF's row stride, a reduction slot, NORM(1:3, m = 0)
    // on the host and the scratch state of the step and start-up maps
    bool adj_ready = false;
    DevGrid gT{};
    double* adj_w[3] = {};
    double* adj_dot = nullptr;
    double adj_n0[3] = {};
    Field* adj_state[6] = {};
    // CUDA graphs of the step map (0) and the step VJP (1), keyed by their fields:
    // the first call with a key runs eagerly (set-up), the second captures, later
    // ones replay
    struct AdjGraph {
        std::vector<const void*> key;
        cudaGraphExec_t exec = nullptr;
        bool warm = false;
        int64_t launches = 0;
    };
    AdjGraph adj_g[2];

    // solver state
    Field *psi = nullptr, *chi = nullptr, *b = nullptr;
    bool solver_ready = false;
    double t = 0.0;
    int n = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;

    // ------------------------------------------------------------------
    mlegs_field* new_field_h(int space, bool persistent) {
        auto mf = std::make_unique<mlegs_field>();
        mf->owner = this;
        Field& f = mf->f;
        f.data = dalloc<double2>(d.cap());
        f.home = f.data;
        if (used_slots >= nslots) throw ApiError(MLEGS_ERR_NOMEM, "out of LN slots");
        f.slot = used_slots++;
        f.ln = lnslots + f.slot;
        f.space = space;
        f.persistent = persistent;
        CK(cudaMemsetAsync(f.data, 0, d.cap() * sizeof(double2), s));
        mlegs_field* out = mf.get();
        owned.push_back(std::move(mf));
        return out;
    }
    Field* new_field(int space, bool persistent) { return &new_field_h(space, persistent)->f; }
    Field* tmp(int space = MLEGS_FFF) {
        if (pool.empty()) throw ApiError(MLEGS_ERR_NOMEM, "temporary field pool exhausted");
        Field* f = pool.back();
        pool.pop_back();
        f->space = space;
        return f;
    }
    void rel(Field* f) { pool.push_back(f); }

    void set_error(const std::string& e) { err = e; }

    // ------------------------------------------------------------------ set-up
    void init(const mlegs_params& prm);
    void destroy();

    // ------------------------------------------------------------------ basic
    size_t fff() const { return d.fff(); }
    void zero_fff(Field* f) { k_fill(f->data, fff(), s); }
    void ln_zero(Field* f) { CK(cudaMemsetAsync(f->ln, 0, sizeof(double), s)); }
    void chopdo(Field* f, int pad) {
        if (f->space == MLEGS_FFF) k_chopdo_fff(g, f->data, pad, s);
        // PFF/PFP/PPP: the device layouts do not store the padded rows/columns.
    }
    void require(const Field* f, int space, const char* who) {
        if (f->space != space)
            throw ApiError(MLEGS_ERR_TRANSFORM, std::string(who) + ": input not in the expected space");
    }
    // COPY0 (mod_fft.f90:705-769): dst = src, CHOPDO for FFF, LN copied.
    void copy0(Field* dst, const Field* src, int pad) {
        if (dst == src) return;
        dst->space = src->space;
        if (src->space == MLEGS_FFF) {  // copy, LN and CHOPDO in one pass
            k_copy_chop_fff(g, dst->data, src->data, dst->ln, src->ln, pad, s);
            return;
        }
        k_copy_ln(dst->data, src->data, d.elems(src->space), dst->ln, src->ln, s);
    }
    void swap_scratch(Field* f) {
        if (f->persistent) throw ApiError(MLEGS_ERR_STATE, "in-place transform of a persistent field");
        std::swap(f->data, scratch);
    }
    void swap_scratch_any(Field* f) { std::swap(f->data, scratch); }

    // ------------------------------------------------------------------ transforms
    // RTRAN(A, IS), mod_fft.f90:1150-1340.  Both directions zero A%LN.
    void rtran(Field* f, int is, int pad) {
        if (is == -1) {
            require(f, MLEGS_PFF, "RTRAN");
            fold(0, pf, d.NRCHOPDIM + 1, f->data, scratch, 0 | 2, 0, 0, pad);
            swap_scratch_any(f);
            f->space = MLEGS_FFF;
        } else {
            require(f, MLEGS_FFF, "RTRAN");
            if (split_S)
                k_split_b2p(g, split_S, split_img, split_eA, f->data, scratch, f->ln, pad, split_err, split_wait, s);
            else
                k_rtran_b2p(g, f->data, scratch, f->ln, pad, s);
            swap_scratch_any(f);
            f->space = MLEGS_PFF;
        }
        ln_zero(f);
    }
    // VERFFT(A, IS), mod_fft.f90:928-1113 (LN preserved).
    void verfft(Field* f, int is) {
        if (is == -1) {
            require(f, MLEGS_PFP, "VERFFT");
            if (!k_verfft4(g, fft, f->data, scratch, -1, s)) k_verfft_f(g, fft, f->data, scratch, s);
            swap_scratch_any(f);
            f->space = MLEGS_PFF;
        } else {
            require(f, MLEGS_PFF, "VERFFT");
            if (!k_verfft4(g, fft, f->data, scratch, +1, s)) k_verfft_b(g, fft, f->data, scratch, s);
            swap_scratch_any(f);
            f->space = MLEGS_PFP;
        }
    }
    // HORFFT(A, IS), mod_fft.f90:771-926.
    void horfft(Field* f, int is) {
        if (is == -1) {
            require(f, MLEGS_PPP, "HORFFT");
            k_horfft_warp(g, fft, f->data, scratch, -1, s);
            swap_scratch_any(f);
            f->space = MLEGS_PFP;
        } else {
            require(f, MLEGS_PFP, "HORFFT");
            k_horfft_warp(g, fft, f->data, scratch, +1, s);
            swap_scratch_any(f);
            f->space = MLEGS_PPP;
        }
    }
    void plnfft(Field* f, int is) {
        if (is == -1) {
            horfft(f, -1);
            verfft(f, -1);
        } else {
            verfft(f, 1);
            horfft(f, 1);
        }
    }
    void toff(Field* f, int pad) {
        if (f->space == MLEGS_PPP) horfft(f, -1);
        if (f->space == MLEGS_PFP) verfft(f, -1);
        if (f->space == MLEGS_PFF) rtran(f, -1, pad);
    }
    void tofp(Field* f, int pad) {
        if (f->space == MLEGS_FFF) rtran(f, 1, pad);
        if (f->space == MLEGS_PFF) verfft(f, 1);
        if (f->space == MLEGS_PFP) horfft(f, 1);
    }

    // TOFP of FFF fields up to PFP (RTRAN(+1) then VERFFT(+1), the reference's
    // order per field) as a two-stream pipeline: the RTRAN(+1) GEMM of field
    // i + 1 on s runs beside the VERFFT(+1) of field i on s2, through three
    // rotating PFF buffers.  Each field ends in its own buffer, in PFP, LN 0.
    cudaEvent_t next_event() {
        cudaEvent_t e = evs[ev_next];
        ev_next = (ev_next + 1) % 64;
        return e;
    }
    void tofp_pipe(Field* const* fs, const int* pads, int n, const cudaEvent_t* ready = nullptr) {
        for (int i = 0; i < n; ++i) require(fs[i], MLEGS_FFF, "RTRAN");
        cudaEvent_t e0 = next_event();
        CK(cudaEventRecord(e0, s));
        CK(cudaStreamWaitEvent(s2, e0, 0));
        cudaEvent_t done[3] = {nullptr, nullptr, nullptr};  // last VERFFT reading pbuf[j]
        for (int i = 0; i < n; ++i) {
            Field* f = fs[i];
            double2* buf = pbuf[i % 3];
            if (done[i % 3]) CK(cudaStreamWaitEvent(s, done[i % 3], 0));
            if (ready && ready[i]) CK(cudaStreamWaitEvent(s, ready[i], 0));  // field made on s2
            if (split_S)
                k_split_b2p(g, split_S, split_img, split_eA, f->data, buf, f->ln, pads[i], split_err, split_wait, s);
            else
                k_rtran_b2p(g, f->data, buf, f->ln, pads[i], s);
            cudaEvent_t eb = next_event();
            CK(cudaEventRecord(eb, s));
            CK(cudaStreamWaitEvent(s2, eb, 0));
            if (!k_verfft4(g, fft, buf, f->data, +1, s2)) k_verfft_b(g, fft, buf, f->data, s2);
            CK(cudaMemsetAsync(f->ln, 0, sizeof(double), s2));  // RTRAN zeroes LN (off the GEMM stream)
            cudaEvent_t ev = next_event();
            CK(cudaEventRecord(ev, s2));
            done[i % 3] = ev;
            f->space = MLEGS_PFP;
        }
        cudaEvent_t ej = next_event();
        CK(cudaEventRecord(ej, s2));
        CK(cudaStreamWaitEvent(s, ej, 0));
    }

    // ------------------------------------------------------------------ operators
    void delsqh(const Field* a, Field* b, int pad) {  // mod_legops.f90:76-133
        require(a, MLEGS_FFF, "DELSQH");
        k_delsqh(g, a->data, a->ln, b->data, pad, s);
        b->space = MLEGS_FFF;
        ln_zero(b);
    }
    void idelsqh(const Field* bb, Field* a, int pad) {  // mod_legops.f90:136-241
        require(bb, MLEGS_FFF, "IDELSQH");
        // A%LN = B(1,1,1) NORM(1,1) ELL2
        k_idelsqh(g, bb->data, a->data, pad, s);
        a->space = MLEGS_FFF;
        ln_from_coef(a->ln, bb->data, d.ELL2);
        k_farfield_fix(g, a->data, d.NRCHOP + pad, s);
    }
    void ln_from_coef(double* ln, const double2* data, double scale);
    void mulxm(const Field* a, Field* b, int pad) {  // 371-428
        require(a, MLEGS_FFF, "MULXM");
        k_band3(g, a->data, b->data, 1, pad, s);
        b->space = MLEGS_FFF;
        ln_zero(b);
    }
    void xxdx(const Field* a, Field* b, int pad) {  // 680-748
        require(a, MLEGS_FFF, "XXDX");
        k_band3(g, a->data, b->data, 0, pad, s);
        k_logterm_rows(g, b->data, a->ln, 0, 1.0, s);
        b->space = MLEGS_FFF;
        ln_zero(b);
    }
    void del2(const Field* a, Field* b, int pad) {  // 751-820
        require(a, MLEGS_FFF, "DEL2");
        k_del2(g, a->data, b->data, pad, s);
        k_logterm_rows(g, b->data, a->ln, 1, 1.0, s);
        b->space = MLEGS_FFF;
        ln_zero(b);
    }
    // IDEL2 (823-1010): has_ln = 0 -> LN absent.
    // LU factors per (kind, pad, alp), formed on first use outside graph capture
    struct SolveFactors {
        int kind, pad;
        double alp;
        double *F5, *F7;
    };
    std::deque<SolveFactors> sfac;  // a deque: entries stay put as the cache grows
    const SolveFactors* factors(int kind, int pad, double alp) {
        for (const SolveFactors& f : sfac)
            if (f.kind == kind && f.pad == pad && f.alp == alp) return &f;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(s, &cs));
        if (cs != cudaStreamCaptureStatusNone || sfac.size() >= 16 || pad < 0 || d.NRCHOP + pad > d.NRCHOPDIM)
            return nullptr;
        size_t n5, n7;
        solve_factor_sizes(g, &n5, &n7);
        SolveFactors f{kind, pad, alp, dalloc<double>(n5), dalloc<double>(n7)};
        k_solve_factor(g, kind, alp, pad, f.F5, f.F7, s);
        sfac.push_back(f);
        return &sfac.back();
    }
    void idel2(const Field* bb, Field* a, int has_ln, double ln, int pad) {
        require(bb, MLEGS_FFF, "IDEL2");
        if (const SolveFactors* f = factors(1, pad, 0.0)) {
            k_solve_factored(g, f->F5, f->F7, bb->data, a->data, a->ln, 1, has_ln, ln, pad, 1, s);
            a->space = MLEGS_FFF;
            return;
        }
        copy0(a, bb, pad);
        ln_zero(a);
        k_solve_del2(g, a->data, a->ln, 1, 0.0, has_ln, ln, nullptr, solve_scr, pad, s);
        chopdo(a, pad);
        k_farfield_fix(g, a->data, d.NRCHOP + pad, s);
    }
    void idel2ln(const Field* bb, Field* a, int pad) {  // 1013-1176
        require(bb, MLEGS_FFF, "IDEL2LN");
        if (const SolveFactors* f = factors(0, pad, 0.0)) {
            k_solve_factored(g, f->F5, f->F7, bb->data, a->data, a->ln, 0, 0, 0.0, pad, 1, s);
            a->space = MLEGS_FFF;
            return;
        }
        copy0(a, bb, pad);
        ln_zero(a);
        k_solve_del2(g, a->data, a->ln, 0, 0.0, 0, 0.0, nullptr, solve_scr, pad, s);
        chopdo(a, pad);
        k_farfield_fix(g, a->data, d.NRCHOP + pad, s);
    }
    void ihelm(const Field* bb, Field* a, double alp, int pad) {  // 1204-1354
        require(bb, MLEGS_FFF, "IHELM");
        if (alp == 0.0) throw ApiError(MLEGS_ERR_LEGOPERATOR, "IHELM: ALP CAN'T BE ZERO");
        copy0(a, bb, pad);
        k_ln_copy(a->ln, bb->ln, -1.0 / alp, s);      // A%LN = -B%LN/ALP
        k_logterm_rows(g, a->data, a->ln, 2, 1.0, s);  // rhs -= LN * DEL2(log)
        if (const SolveFactors* f = factors(2, pad, alp))
            k_solve_factored(g, f->F5, f->F7, a->data, a->data, nullptr, 2, 0, 0.0, pad, 0, s);
        else
            k_solve_del2(g, a->data, nullptr, 2, alp, 0, 0.0, nullptr, solve_scr, pad, s);
        chopdo(a, pad);
    }
    // IHELMP (mod_legops.f90:1409-1592): DEL2H power tables per P (built on the
    // host, uploaded once) and the elimination scratch, both allocated outside
    // graph capture (at set-up for the configured VISC%P when VISC%SW = 2)
    std::vector<std::pair<int, double*>> helmp_tab;
    double* helmp_scr = nullptr;
    int helmp_scr_p = 0;
    int helmp_rows() const { return d.NRCHOPDIM; }
    void no_capture(const char* who) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(s, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            throw ApiError(MLEGS_ERR_STATE, std::string(who) + ": set-up needed outside graph capture");
    }
    const double* helmp_tables(int P);
    double* helmp_scratch(int P) {
        if (helmp_scr && helmp_scr_p >= P) return helmp_scr;
        no_capture("IHELMP");
        helmp_scr = dalloc<double>(ihelmp_scratch_doubles(g, P));
        helmp_scr_p = P;
        return helmp_scr;
    }
    void ihelmp(const Field* bb, Field* a, int P, double alp, double nu, int pad) {  // 1409-1592
        require(bb, MLEGS_FFF, "IHELMP");
        if (P < 4 || P > 14 || P % 2) throw ApiError(MLEGS_ERR_ARG, "IHELMP: P OUT OF RANGE (EVEN, 4..14)");
        if (alp == 0.0) throw ApiError(MLEGS_ERR_LEGOPERATOR, "IHELMP: ALP CANNOT BE ZERO.");
        const double* tab = helmp_tables(P);
        double* scr = helmp_scratch(P);
        copy0(a, bb, pad);                        // A = B
        k_ln_copy(a->ln, bb->ln, -1.0 / alp, s);  // A%LN = -B%LN/ALP
        k_ihelmp(g, P, tab, helmp_rows(), a->data, a->ln, alp, nu, scr, pad, s);
        k_farfield_fix(g, a->data, d.NRCHOP + pad, s, 1);  // CALCAT1(A)/TFM%PF(1,1,1)
        chopdo(a, pad);
        a->space = MLEGS_FFF;
    }
    // HYPERV(A, NU, NUP, P, DT, WK) (mod_march.f90:1639-1686), in place on A.
    void hyperv2(Field* a, double nu, double nup, int P, double dt) {
        if (nup == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "HYPERV: NUP CAN'T BE ZERO");
        if (a->space != MLEGS_FFF) throw ApiError(MLEGS_ERR_SOLVER, "HYPERV: INPUT IS NOT IN FFF_SPACE");
        const int ph = P / 2;
        const double sg = (ph % 2) ? -1.0 : 1.0;  // (-1)**PH
        const double alp = 1 / dt / nup * sg;
        const double bet = -sg * nu / nup;
        Field* wk = tmp();
        k_axpby_ln(wk->data, alp, a->data, 0.0, nullptr, 0.0, fff(), wk->ln, alp, a->ln, 0.0, nullptr, 0.0, s);
        wk->space = MLEGS_FFF;
        ihelmp(wk, a, P, -alp, bet, 0);
        rel(wk);
    }
    // The fused derivative kernels read row neighbours of their inputs while
    // writing the outputs, so an output may not share a buffer with an input.
    static void distinct(std::initializer_list<const Field*> in, std::initializer_list<const Field*> out,
                         const char* who) {
        for (const Field* o : out)
            for (const Field* i : in)
                if (o->data == i->data)
                    throw ApiError(MLEGS_ERR_ARG, std::string(who) + ": outputs must be distinct from the inputs");
    }
    void grad(const Field* a, Field* rr, Field* rp, Field* gz, int pad, cudaStream_t st = nullptr) {  // 1727-1786
        require(a, MLEGS_FFF, "GRAD");
        distinct({a}, {rr, rp, gz}, "GRAD");
        if (!st) st = s;
        k_grad_fused(g, a->data, a->ln, rr->data, rp->data, gz->data, pad, st);
        rr->space = rp->space = gz->space = MLEGS_FFF;
        for (Field* f : {rr, rp, gz}) CK(cudaMemsetAsync(f->ln, 0, sizeof(double), st));
    }
    void pc2vel(const Field* psi_, const Field* chi_, Field* rur, Field* rup, Field* uz, int pad) {  // 1789-1853
        require(psi_, MLEGS_FFF, "PC2VEL");
        require(chi_, MLEGS_FFF, "PC2VEL");
        distinct({psi_, chi_}, {rur, rup, uz}, "PC2VEL");
        double* zl[3] = {rur->ln, rup->ln, uz->ln};  // set to 0 by the kernel
        k_pc2vel_fused(g, psi_->data, psi_->ln, chi_->data, chi_->ln, rur->data, rup->data, uz->data, pad, s, 0, zl);
        rur->space = rup->space = uz->space = MLEGS_FFF;
    }
    void pc2vor(const Field* psi_, const Field* chi_, Field* ror, Field* rop, Field* oz, int pad,
                cudaStream_t st = nullptr) {  // 1856-1919
        require(psi_, MLEGS_FFF, "PC2VOR");
        require(chi_, MLEGS_FFF, "PC2VOR");
        distinct({psi_, chi_}, {ror, rop, oz}, "PC2VOR");
        if (!st) st = s;
        k_pc2vor_fused(g, psi_->data, psi_->ln, chi_->data, chi_->ln, ror->data, rop->data, oz->data, pad, st);
        ror->space = rop->space = oz->space = MLEGS_FFF;
        for (Field* f : {ror, rop, oz}) CK(cudaMemsetAsync(f->ln, 0, sizeof(double), st));
    }
    // PROJECT (mod_legops.f90:2397-2545).  ln_mode: 0 none, 1 value, 2 PSI%LN by reference.
    void project(Field* rur, Field* rup, Field* uz, Field* psi_, Field* chi_, int ln_mode, double ln) {
        if (!(rur->space == rup->space && rup->space == uz->space))
            throw ApiError(MLEGS_ERR_TRANSFORM, "PROJECT: RUR, RUP, UZ MUST BE IN THE SAME SPACE.");
        if (rur->space == MLEGS_PPP) {
            plnfft(rur, -1);
            plnfft(rup, -1);
            plnfft(uz, -1);
        } else if (rur->space == MLEGS_PFP) {  // PPP already taken through HORFFT(-1)
            verfft(rur, -1);
            verfft(rup, -1);
            verfft(uz, -1);
        } else if (rur->space == MLEGS_FFF) {
            rtran(rur, 1, 0);
            rtran(rup, 1, 0);
            rtran(uz, 1, 0);
        } else if (rur->space != MLEGS_PFF) {
            throw ApiError(MLEGS_ERR_TRANSFORM, "PROJECT: bad input space");
        }
        psi_->space = chi_->space = MLEGS_FFF;
        if (ln_mode == 1) launch_vel2pln(g, rup->data, psi_->ln, 1, ln, v2p_pff, s, chi_->ln);
        else if (ln_mode == 2) launch_vel2pln(g, rup->data, psi_->ln, 0, 0.0, v2p_pff, s, chi_->ln);
        else {
            ln_zero(psi_);
            ln_zero(chi_);
        }
        if (!split_S && fc_V) {
            project_bulk(rur->data, rup->data, uz->data, psi_->data, chi_->data, s);
            k_farfield_fix(g, psi_->data, d.NRCHOP, s);
            return;
        }
        if (!split_S && dmma_supported(g)) {
            k_project_dmma(g, V, D, T, rur->data, rup->data, uz->data, psi_->data, chi_->data, s);
            k_farfield_fix(g, psi_->data, d.NRCHOP, s);
            return;
        }
        const int wr = d.NRCHOPDIM;
        // PSI = -(i m) EO(V, RUR) - OE(D, RUP)
        fold(1, V, wr, rur->data, psi_->data, 0, 2, 0, 0);
        fold(2, D, wr, rup->data, psi_->data, 1, 1, 1, 0);
        // CHI = (i k) OE(D, RUR) + m k EO(V, RUP) - EO(T, UZ)
        fold(2, D, wr, rur->data, chi_->data, 1, 3, 0, 0);
        fold(1, V, wr, rup->data, chi_->data, 0, 4, 1, 0);
        fold(3, T, wr, uz->data, chi_->data, 0, 1, 1, 0);
        k_farfield_fix(g, psi_->data, d.NRCHOP, s);
    }

    // PROJECT's five fold products of PFF inputs (mod_legops.f90:2497-2535) on
    // the bulk-copy pipeline: PSI = -(i m) EO(V, RUR) - OE(D, RUP),
    // CHI = (i k) OE(D, RUR) + m k EO(V, RUP) - EO(T, UZ).
    void project_bulk(const double2* rur, const double2* rup, const double2* uz, double2* psi_, double2* chi_,
                      cudaStream_t st) {
        const double* wc[5] = {fc_V, fc_D, fc_D, fc_V, fc_T};
        const double2* x[5] = {rur, rup, rur, rup, uz};
        const int md[5] = {0, 1, 1, 0, 0}, sc[5] = {2, 1, 3, 4, 1};
        k_fold_bulk(g, wc, x, md, sc, 5, 2, psi_, chi_, d.NRCHOPDIM, 0, 0, st);
    }
    // PROJECT(RUR, RUP, UZ, PSI, CHI) with PSI%LN by reference (ln_mode 2) for
    // FFF inputs whose LN terms are zero: one composite FFF -> FFF product per m
    // in FP64 contexts (RUP's (0, 0) column is changed in place by VEL2PLN).
    void project_fff_ln2(Field* rur, Field* rup, Field* uz, Field* psi_, Field* chi_) {
        if (!compV || rur->space != MLEGS_FFF || rup->space != MLEGS_FFF || uz->space != MLEGS_FFF) {
            project(rur, rup, uz, psi_, chi_, 2, 0.0);
            return;
        }
        psi_->space = chi_->space = MLEGS_FFF;
        k_project_fff_dmma(g, compV, compD, compT, rur->data, rup->data, uz->data, psi_->data, chi_->data, psi_->ln,
                           v2p_fff, s, chi_->ln);
        k_farfield_fix(g, psi_->data, d.NRCHOP, s);
    }

    // ------------------------------------------------------------------ physics
    void force(const Field* PSI, const Field* CHI, const Field* B, Field* PSIN, Field* CHIN, Field* BN);
    void energy(const Field* PSI, const Field* CHI, const Field* B, double* ke, double* pe, double* dke);
    void diagnost(const Field* PSI, const Field* CHI, double out[11]);
    void boussi_pe(const Field* B, double* pe);
    void enemon(const Field* PSI, const Field* CHI, int pad, double* em, double* ek);
    void hyp3set(const double nu[3], double** tables);
    void qvortex(const mlegs_vortex* v, int n, const int32_t* seeds, Field* PSI, Field* CHI);
    void hyp3adj(const Field* PSI, const Field* CHI, const Field* B);
    void halfk(const double* all, double sign, double* out, bool accumulate) const;
    void nonlin(const Field* B, Field* RUR, Field* RUP, Field* UZ, Field* ROR, Field* ROP, Field* OZ,
                Field* BN, cudaEvent_t vor_ready = nullptr, Field* PSIN = nullptr, Field* CHIN = nullptr);
    void visc1(Field* A, double nu, double dt);
    void visc2(Field* A, const Field* AO, double nu, double dt);
    void visc_be(Field* P, Field* C, Field* B, double dt);
    void visc_cn(Field* P, Field* C, Field* B, const Field* PO, const Field* CO, const Field* BO);
    void hyperv3(Field* P, Field* C, Field* B, double tf);
    void etd_hyperv(Field* R, Field* Pp, Field* Z, Field* B, double tf);
    void sponge(Field* UZ, Field* B, double dt);
    void rich_fe_be();
    void step_ab_cn();
    void etdfe_be(Field* P, Field* C, Field* B, const double* E, const double* NL, double dt, bool store);
    void rich_etdfe_be();
    void step_etdab_cn();
    void step_once() { p.adams ? step_ab_cn() : step_etdab_cn(); }

    // snapshot of the temporaries' buffers so every step reuses the same pointers
    std::vector<double2*> snap;
    double2* snap_scratch = nullptr;
    void mark() {
        snap.clear();
        for (Field* f : temps) snap.push_back(f->data);
        snap_scratch = scratch;
    }
    void restore() {
        for (size_t i = 0; i < temps.size(); ++i) temps[i]->data = snap[i];
        scratch = snap_scratch;
    }
};

// C ABI helpers
template <class F>
inline int guard(mlegs_ctx* ctx, F&& fn) {
    if (!ctx) return MLEGS_ERR_ARG;
    int64_t* prev = g_launch_counter;
    std::vector<void*>* prev_allocs = g_allocs;
    g_launch_counter = &ctx->launches;
    g_allocs = &ctx->allocs;
    int rc = MLEGS_OK;
    try {
        cudaSetDevice(ctx->dev);
        fn();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw CudaError(std::string("kernel launch: ") + cudaGetErrorString(e));
    } catch (const ApiError& e) {
        ctx->set_error(e.what());
        rc = e.code;
    } catch (const CudaError& e) {
        ctx->set_error(e.what());
        rc = MLEGS_ERR_CUDA;
    } catch (const std::exception& e) {
        ctx->set_error(e.what());
        rc = MLEGS_ERR_STATE;
    }
    g_launch_counter = prev;
    g_allocs = prev_allocs;
    return rc;
}
inline Field* F(mlegs_field* f) {
    if (!f) throw ApiError(MLEGS_ERR_ARG, "null field");
    return &f->f;
}
inline const Field* F(const mlegs_field* f) {
    if (!f) throw ApiError(MLEGS_ERR_ARG, "null field");
    return &f->f;
}
inline void check_pad(const mlegs_ctx* c, int pad) {
    if (c->d.NRCHOP + pad > c->d.NRCHOPDIM || c->d.NRCHOP + pad < 0)
        throw ApiError(MLEGS_ERR_SCALAR3, "CHOPSET: NRCHOP TOO LARGE");
}
