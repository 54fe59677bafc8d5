// Ensembles: independent AB2-CN runs of different grids on one GPU, advanced in
// lock-step with grouped persistent launches (the batched-run configuration).
//
// The reference runs one Boussinesq instance per MPI job; STEP_BOUSSI_AB_CN
// (mod_march.f90:609-661) with CALC_BOUSSI_FORCE (mod_boussinesq.f90:317-410)
// calls, per instance and step, ten RTRAN(+1), PROJECT's five EOMUL/OEMUL
// products, one RTRAN(-1) (per-m GEMMs of uneven size NN_m = NRCHOP + pad - m,
// mod_fft.f90:1189-1336, mod_legops.f90:2497-2535) and the banded solves of
// IDEL2LN and IHELM (mod_legops.f90:1013-1354).  Here every instance is an
// ordinary context (its own fields, tables and streams), and a step is cut at
// those calls into five phases:
//   0  GRAD / PC2VEL / PC2VOR at CHOPSET(3), W = B            | grouped RTRAN(+1) x 10
//   1  VERFFT(+1), theta stage, VERFFT(-1), VEL2PLN             | grouped PROJECT folds + RTRAN(-1)
//   2  far-field fix, B_N                                       | grouped IDEL2LN solves
//   3  AB2 update, history, VISC2 right-hand sides (DEL2)       | grouped IHELM solves
//   4  CHOPDO, CALC_BOUSSI_HYPERV
// The per-instance work of a phase runs on each instance's stream; each
// grouped launch runs on the ensemble's stream after all instances reach it,
// over every instance's problems at once: persistent CTAs take (problem, m,
// column tile) work items from a global counter (gemm_dmma.cu), the solves one
// block per 64 systems (solve.cu).  The arithmetic is the single-grid path's,
// tile for tile.  A step is captured once as a CUDA graph over all streams.
//
// Autotuner: the column-tile width of each class of GEMM problems -- key
// (transform, NRH, NRCHOP), which fixes the GEMM's rows and its K extents
// NN_m -- is 16 or 32 columns, chosen by timing the class's grouped launch
// with each width (best of three), and the number of persistent CTAs per SM
// (2, 3 or 4) by timing the full launch.  Choices are cached for the process
// and reused by ensembles with the same classes.
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>

#include "ctx_internal.h"

namespace {

struct EnsInst {
    mlegs_ctx* c = nullptr;
    std::vector<Field*> pool0;  // the temporary pool's order at the start of a step
    Field *PN = nullptr, *CN = nullptr, *BN = nullptr;
    Field* f[10] = {};  // RUR, RUP, UZ, ROR, ROP, OZ, RBR, RBP, BZ, W
    Field* T[10] = {};  // their RTRAN(+1) images
    Field *NR = nullptr, *NP = nullptr, *NZ = nullptr, *BNp = nullptr, *Wf = nullptr;
    Field *P0 = nullptr, *C0 = nullptr, *B0 = nullptr;
    Field* WK[3] = {};
    Field* VA[3] = {};  // fields solved by IHELM in phase 3
    int nvisc = 0;
    cudaEvent_t ev = nullptr;
};

using ClassKey = std::tuple<int, int, int>;  // (0 RTRAN(+1) | 1 fold, NRH, NRCHOP)
std::mutex g_tune_mu;
std::map<ClassKey, int> g_tuned_nj;     // column tiles of 8 nj columns
std::map<int, int> g_tuned_ctas;        // kind -> persistent CTAs per SM

template <class D>
struct Group {
    std::vector<D> h;            // this step's problems
    std::vector<D> up;           // what the device holds
    std::vector<int> first;      // first tile / block per problem
    D* d = nullptr;
    int* d_first = nullptr;
    size_t cap = 0;
    int total = 0;
    size_t smem = 0;
};

}  // namespace

struct mlegs_ensemble {
    int dev = 0;
    std::vector<mlegs_ctx*> inst;
    std::vector<EnsInst> st;
    cudaStream_t gs = nullptr;
    cudaEvent_t gev = nullptr;
    std::string err;
    std::vector<void*> allocs;
    int64_t launches = 0, graph_launches = 0;
    int* d_next = nullptr;  // tile counters of the two GEMM groups
    int sms = 148;
    int ctas[2] = {3, 3};
    bool prepared = false, tuned = false;
    Group<GroupB2P> gb2p;
    Group<GroupFold> gfold;
    Group<GroupSolve> gs1, gs2;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool capturing = false;

    void destroy() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (EnsInst& I : st)
            if (I.ev) cudaEventDestroy(I.ev);
        if (gev) cudaEventDestroy(gev);
        for (mlegs_ctx* c : inst) mlegs_destroy(c);
        for (void* p : allocs) cudaFree(p);
        if (gs) cudaStreamDestroy(gs);
    }

    int nj_for(int kind, const DevGrid& g) const {
        auto it = g_tuned_nj.find(ClassKey(kind, g.NRH, g.NRCHOP));
        return it == g_tuned_nj.end() ? 4 : it->second;
    }

    // all instance streams -> the ensemble stream
    void join_to_group() {
        for (EnsInst& I : st) {
            CK(cudaEventRecord(I.ev, I.c->s));
            CK(cudaStreamWaitEvent(gs, I.ev, 0));
        }
    }
    void group_to_all() {
        CK(cudaEventRecord(gev, gs));
        for (EnsInst& I : st) CK(cudaStreamWaitEvent(I.c->s, gev, 0));
    }

    template <class D>
    void upload(Group<D>& G, const std::function<int(D&)>& count) {
        G.first.resize(G.h.size());
        G.total = 0;
        for (size_t i = 0; i < G.h.size(); ++i) {
            G.h[i].first = G.total;
            G.first[i] = G.total;
            G.total += count(G.h[i]);
        }
        const bool same = G.up.size() == G.h.size() &&
                          std::memcmp(G.up.data(), G.h.data(), G.h.size() * sizeof(D)) == 0;
        if (same) return;
        if (capturing) throw ApiError(MLEGS_ERR_STATE, "ensemble: the problems changed during graph capture");
        CK(cudaStreamSynchronize(gs));
        if (G.h.size() > G.cap) {
            G.cap = G.h.size();
            G.d = dalloc<D>(G.cap);
            G.d_first = dalloc<int>(G.cap);
        }
        CK(cudaMemcpy(G.d, G.h.data(), G.h.size() * sizeof(D), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(G.d_first, G.first.data(), G.first.size() * sizeof(int), cudaMemcpyHostToDevice));
        G.up = G.h;
    }

    void launch_b2p() {
        upload<GroupB2P>(gb2p, [](GroupB2P& p) { return group_b2p_prepare(p); });
        gb2p.smem = 0;
        for (const GroupB2P& p : gb2p.up) gb2p.smem = std::max(gb2p.smem, group_b2p_smem(p));
        k_grouped_b2p(gb2p.d, gb2p.d_first, (int)gb2p.up.size(), gb2p.total, gb2p.smem,
                      std::min(gb2p.total, sms * ctas[0]), d_next, gs);
    }
    void launch_fold() {
        upload<GroupFold>(gfold, [](GroupFold& p) { return group_fold_prepare(p); });
        gfold.smem = 0;
        for (const GroupFold& p : gfold.up) gfold.smem = std::max(gfold.smem, group_fold_smem(p));
        k_grouped_fold(gfold.d, gfold.d_first, (int)gfold.up.size(), gfold.total, gfold.smem,
                       std::min(gfold.total, sms * ctas[1]), d_next + 1, gs);
    }
    void launch_solve(Group<GroupSolve>& G) {
        upload<GroupSolve>(G, [](GroupSolve& p) { return group_solve_blocks(p); });
        if (G.total) k_grouped_solve(G.d, G.d_first, (int)G.up.size(), G.total, gs);
    }

    void prepare();
    void step();
    void tune();
};

namespace {

constexpr int P3 = 3;  // CHOPSET(3) of CALC_BOUSSI_FORCE

// Phase 0: the derivative fields of CALC_BOUSSI_FORCE (GRAD, PC2VEL, PC2VOR at
// CHOPSET(3); W = B at CHOPSET(0)) and their RTRAN(+1) problems.
void phase0(mlegs_ensemble& E, EnsInst& I) {
    mlegs_ctx* c = I.c;
    I.pool0 = c->pool;
    c->mark();
    c->t += c->p.dt;
    c->n += 1;
    I.PN = c->tmp();
    I.CN = c->tmp();
    I.BN = c->tmp();
    for (Field*& f : I.f) f = c->tmp();
    Field **f = I.f;
    c->grad(c->b, f[6], f[7], f[8], P3);
    c->pc2vel(c->psi, c->chi, f[0], f[1], f[2], P3);
    c->pc2vor(c->psi, c->chi, f[3], f[4], f[5], P3);
    c->copy0(f[9], c->b, 0);
    for (int q = 0; q < 10; ++q) {
        I.T[q] = c->tmp(MLEGS_PFF);
        GroupB2P p{};
        p.g = c->g;
        p.in = (const double*)f[q]->data;
        p.out = (double*)I.T[q]->data;
        p.ln = f[q]->ln;
        p.pad = q < 9 ? P3 : 0;
        p.nj = E.nj_for(0, c->g);
        E.gb2p.h.push_back(p);
    }
}

// Phase 1: VERFFT(+1) of the ten images, the theta stage with the linear terms,
// PROJECT's VERFFT(-1) and VEL2PLN, TOFF(B_N) up to PFF; fold problems.
void phase1(mlegs_ensemble& E, EnsInst& I) {
    mlegs_ctx* c = I.c;
    const DevGrid& g = c->g;
    for (int q = 0; q < 10; ++q) {
        if (!k_verfft4(g, c->fft, I.T[q]->data, I.f[q]->data, +1, c->s)) k_verfft_b(g, c->fft, I.T[q]->data, I.f[q]->data, c->s);
        c->ln_zero(I.f[q]);
        I.f[q]->space = MLEGS_PFP;
        c->rel(I.T[q]);
    }
    I.NR = c->tmp();
    I.NP = c->tmp();
    I.NZ = c->tmp();
    I.BNp = c->tmp();
    const double2* in[10];
    for (int q = 0; q < 10; ++q) in[q] = I.f[q]->data;
    double2* out[4] = {I.NR->data, I.NP->data, I.NZ->data, I.BNp->data};
    k_theta_fused(g, c->fft, in, out, c->p.omega, c->p.bv0, 1, c->s);
    for (Field* x : {I.NR, I.NP, I.NZ, I.BNp}) {
        x->space = MLEGS_PFP;
        c->ln_zero(x);
    }
    for (Field* x : I.f) c->rel(x);
    I.Wf = c->tmp();
    // PROJECT(NR, NP, NZ, PSI_N, W, 0) of PFP input (mod_legops.f90:2397-2545)
    c->verfft(I.NR, -1);
    c->verfft(I.NP, -1);
    c->verfft(I.NZ, -1);
    I.PN->space = I.Wf->space = MLEGS_FFF;
    launch_vel2pln(g, I.NP->data, I.PN->ln, 1, 0.0, c->v2p_pff, c->s, I.Wf->ln);
    GroupFold pj{};
    pj.g = g;
    const double* w[5] = {c->V, c->D, c->D, c->V, c->T};
    const double2* x[5] = {I.NR->data, I.NP->data, I.NR->data, I.NP->data, I.NZ->data};
    const int mode[5] = {0, 1, 1, 0, 0}, scale[5] = {2, 1, 3, 4, 1};
    for (int q = 0; q < 5; ++q) {
        pj.fa.w[q] = w[q];
        pj.fa.x[q] = (const double*)x[q];
        pj.fa.mode[q] = mode[q];
        pj.fa.scale[q] = scale[q];
    }
    pj.fa.nseg = 5;
    pj.fa.split = 2;
    pj.fa.out0 = (double*)I.PN->data;
    pj.fa.out1 = (double*)I.Wf->data;
    pj.fa.wt_rows = g.NRCHOPDIM;
    pj.nj = E.nj_for(1, g);
    E.gfold.h.push_back(pj);
    // TOFF(B_N): VERFFT(-1), then RTRAN(-1) into the context's scratch buffer
    c->verfft(I.BNp, -1);
    GroupFold rt{};
    rt.g = g;
    rt.fa.w[0] = c->pf;
    rt.fa.x[0] = (const double*)I.BNp->data;
    rt.fa.nseg = rt.fa.split = 1;
    rt.fa.out0 = rt.fa.out1 = (double*)c->scratch;
    rt.fa.wt_rows = g.NRCHOPDIM + 1;
    rt.fa.use_w = 1;
    rt.nj = E.nj_for(1, g);
    E.gfold.h.push_back(rt);
}

// Phase 2: PROJECT's far-field fix, B_N = TOFF(...), IDEL2LN(W -> CHI_N) problem.
void phase2(mlegs_ensemble& E, EnsInst& I) {
    mlegs_ctx* c = I.c;
    k_farfield_fix(c->g, I.PN->data, c->d.NRCHOP, c->s);
    c->swap_scratch_any(I.BNp);
    I.BNp->space = MLEGS_FFF;
    c->ln_zero(I.BNp);
    c->copy0(I.BN, I.BNp, 0);
    for (Field* x : {I.BNp, I.NR, I.NP, I.NZ}) c->rel(x);
    const auto* fc = c->factors(0, 0, 0.0);
    if (!fc) throw ApiError(MLEGS_ERR_STATE, "ensemble: IDEL2LN factors missing");
    GroupSolve p{};
    p.g = c->g;
    p.F5 = fc->F5;
    p.F7 = fc->F7;
    p.src = I.Wf->data;
    p.dst = I.CN->data;
    p.ln_out = I.CN->ln;
    p.kind = 0;
    p.farfield = 1;
    I.CN->space = MLEGS_FFF;
    E.gs1.h.push_back(p);
}

// Phase 3: the AB2 update and history (mod_march.f90:639-647), VISC2's
// right-hand sides and IHELM problems (CALC_BOUSSI_VISC_CN, 1233-1265).
void phase3(mlegs_ensemble& E, EnsInst& I) {
    mlegs_ctx* c = I.c;
    const DevGrid& g = c->g;
    const double dt = c->p.dt;
    c->rel(I.Wf);
    I.P0 = c->tmp();
    I.C0 = c->tmp();
    I.B0 = c->tmp();
    c->copy0(I.P0, c->psi, 0);
    c->copy0(I.C0, c->chi, 0);
    c->copy0(I.B0, c->b, 0);
    const size_t N = c->fff();
    Field **H = c->hist;
    k_axpby_ln(c->psi->data, 1.5 * dt, I.PN->data, -0.5 * dt, H[0]->data, 1.0, N,
               c->psi->ln, 1.5 * dt, I.PN->ln, -0.5 * dt, H[0]->ln, 1.0, c->s);
    k_axpby_ln(c->chi->data, 1.5 * dt, I.CN->data, -0.5 * dt, H[1]->data, 1.0, N,
               c->chi->ln, 1.5 * dt, I.CN->ln, -0.5 * dt, H[1]->ln, 1.0, c->s);
    k_axpby(c->b->data, 1.5 * dt, I.BN->data, -0.5 * dt, H[2]->data, 1.0, N, c->s);
    c->copy0(H[0], I.PN, 0);
    c->copy0(H[1], I.CN, 0);
    c->copy0(H[2], I.BN, 0);
    c->rel(I.PN);
    c->rel(I.CN);
    c->rel(I.BN);
    I.nvisc = 0;
    if (c->p.visc_sw != 1) return;
    Field* A[3] = {c->psi, c->chi, c->b};
    Field* AO[3] = {I.P0, I.C0, I.B0};
    const double nu[3] = {c->p.nu, c->p.nu, c->p.kappa};
    for (int q = 0; q < 3; ++q) {
        if (q == 2 && c->p.kappa == 0.0) break;
        if (nu[q] == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "VISC2: NU CAN'T BE ZERO");
        const double alp = 2 / nu[q] / dt;
        Field* WK = c->tmp();
        c->del2(AO[q], WK, 2);
        c->chopdo(WK, 0);
        k_axpby_ln(WK->data, -alp, A[q]->data, 0.0, nullptr, -1.0, N,
                   WK->ln, -alp, A[q]->ln, 0.0, nullptr, 0.0, c->s);
        // IHELM(WK, A, ALP) up to its substitutions (mod_legops.f90:1204-1354)
        c->copy0(A[q], WK, 0);
        k_ln_copy(A[q]->ln, WK->ln, -1.0 / alp, c->s);
        k_logterm_rows(g, A[q]->data, A[q]->ln, 2, 1.0, c->s);
        const auto* fh = c->factors(2, 0, alp);
        if (!fh) throw ApiError(MLEGS_ERR_STATE, "ensemble: IHELM factors missing");
        GroupSolve p{};
        p.g = g;
        p.F5 = fh->F5;
        p.F7 = fh->F7;
        p.src = A[q]->data;
        p.dst = A[q]->data;
        p.kind = 2;
        E.gs2.h.push_back(p);
        I.WK[q] = WK;
        I.VA[q] = A[q];
        ++I.nvisc;
    }
}

// Phase 4: IHELM's CHOPDO, CALC_BOUSSI_HYPERV, and the step's temporaries back.
void phase4(mlegs_ensemble&, EnsInst& I) {
    mlegs_ctx* c = I.c;
    for (int q = 0; q < I.nvisc; ++q) {
        c->chopdo(I.VA[q], 0);
        c->rel(I.WK[q]);
    }
    c->rel(I.P0);
    c->rel(I.C0);
    c->rel(I.B0);
    c->hyperv3(c->psi, c->chi, c->b, 1.0);
    c->restore();
    c->pool = I.pool0;
}

}  // namespace

// Factors and checks before the first step (outside any capture).
void mlegs_ensemble::prepare() {
    if (prepared) return;
    for (mlegs_ctx* c : inst) {
        if (!c->solver_ready) throw ApiError(MLEGS_ERR_STATE, "ensemble: mlegs_solver_init has not run on every instance");
        if (!c->p.adams) throw ApiError(MLEGS_ERR_ARG, "ensemble: AB2-CN instances only (BOUSSINESQ ABSW = 1)");
        if (c->split_S) throw ApiError(MLEGS_ERR_ARG, "ensemble: FP64 instances only");
        if (!group_supported(c->g)) throw ApiError(MLEGS_ERR_ARG, "ensemble: grid outside the grouped GEMM limits");
        if (!c->factors(0, 0, 0.0)) throw ApiError(MLEGS_ERR_STATE, "ensemble: IDEL2LN factors");
        if (c->p.visc_sw == 1) {
            const double dt = c->p.dt;
            if (c->p.nu == 0.0) throw ApiError(MLEGS_ERR_SOLVER, "VISC2: NU CAN'T BE ZERO");
            c->factors(2, 0, 2 / c->p.nu / dt);
            if (c->p.kappa != 0.0) c->factors(2, 0, 2 / c->p.kappa / dt);
        }
    }
    CK(cudaDeviceSynchronize());
    prepared = true;
}

// Launch errors are attributed to the stage that raised them (outside capture).
static void stage_check(bool capturing, const char* stage) {
    if (capturing) return;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError(std::string("ensemble ") + stage + ": " + cudaGetErrorString(e));
}

void mlegs_ensemble::step() {
    gb2p.h.clear();
    gfold.h.clear();
    gs1.h.clear();
    gs2.h.clear();
    for (EnsInst& I : st) phase0(*this, I);
    stage_check(capturing, "phase 0");
    join_to_group();
    launch_b2p();
    stage_check(capturing, "grouped RTRAN(+1)");
    group_to_all();
    for (EnsInst& I : st) phase1(*this, I);
    stage_check(capturing, "phase 1");
    join_to_group();
    launch_fold();
    stage_check(capturing, "grouped folds");
    group_to_all();
    for (EnsInst& I : st) phase2(*this, I);
    stage_check(capturing, "phase 2");
    join_to_group();
    launch_solve(gs1);
    stage_check(capturing, "grouped IDEL2LN");
    group_to_all();
    for (EnsInst& I : st) phase3(*this, I);
    stage_check(capturing, "phase 3");
    join_to_group();
    launch_solve(gs2);
    stage_check(capturing, "grouped IHELM");
    group_to_all();
    for (EnsInst& I : st) phase4(*this, I);
    stage_check(capturing, "phase 4");
    join_to_group();
}

// Autotuning on the problems of the last step (between steps: the grouped
// kernels only rewrite temporaries, which the next step recomputes).
void mlegs_ensemble::tune() {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto timed = [&](const std::function<void()>& fn) {
        float best = 1e30f;
        for (int r = 0; r < 3; ++r) {
            CK(cudaEventRecord(e0, gs));
            fn();
            CK(cudaEventRecord(e1, gs));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        return best;
    };
    // per class: column-tile width
    auto tune_kind = [&](auto& G, int kind, auto prepare, auto smem_of, auto launcher) {
        using D = typename std::decay<decltype(G.up)>::type::value_type;
        std::map<ClassKey, std::vector<D>> classes;
        for (const D& p : G.up) classes[ClassKey(kind, p.g.NRH, p.g.NRCHOP)].push_back(p);
        for (auto& kv : classes) {
            if (g_tuned_nj.count(kv.first)) continue;
            float best = 1e30f;
            int pick = 4;
            for (int nj : {2, 4}) {
                std::vector<D> sub = kv.second;
                std::vector<int> first(sub.size());
                int total = 0;
                size_t smem = 0;
                for (size_t i = 0; i < sub.size(); ++i) {
                    sub[i].nj = nj;
                    sub[i].first = total;
                    first[i] = total;
                    total += prepare(sub[i]);
                    smem = std::max(smem, smem_of(sub[i]));
                }
                D* d = dalloc<D>(sub.size());
                int* df = dalloc<int>(sub.size());
                CK(cudaMemcpy(d, sub.data(), sub.size() * sizeof(D), cudaMemcpyHostToDevice));
                CK(cudaMemcpy(df, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice));
                const float ms = timed([&] { launcher(d, df, (int)sub.size(), total, smem, std::min(total, sms * ctas[kind])); });
                if (ms < best) {
                    best = ms;
                    pick = nj;
                }
            }
            g_tuned_nj[kv.first] = pick;
        }
    };
    tune_kind(gb2p, 0, [](GroupB2P& p) { return group_b2p_prepare(p); },
              [](const GroupB2P& p) { return group_b2p_smem(p); },
              [&](GroupB2P* d, int* df, int n, int total, size_t smem, int c) {
                  k_grouped_b2p(d, df, n, total, smem, c, d_next, gs);
              });
    tune_kind(gfold, 1, [](GroupFold& p) { return group_fold_prepare(p); },
              [](const GroupFold& p) { return group_fold_smem(p); },
              [&](GroupFold* d, int* df, int n, int total, size_t smem, int c) {
                  k_grouped_fold(d, df, n, total, smem, c, d_next + 1, gs);
              });
    // the chosen widths into the step's problems, then CTAs per SM per kind
    for (GroupB2P& p : gb2p.h) p.nj = nj_for(0, p.g);
    for (GroupFold& p : gfold.h) p.nj = nj_for(1, p.g);
    for (int kind = 0; kind < 2; ++kind) {
        if (g_tuned_ctas.count(kind)) {
            ctas[kind] = g_tuned_ctas[kind];
            continue;
        }
        float best = 1e30f;
        int pick = 3;
        for (int c : {2, 3, 4}) {
            ctas[kind] = c;
            const float ms = timed([&] { kind == 0 ? launch_b2p() : launch_fold(); });
            if (ms < best) {
                best = ms;
                pick = c;
            }
        }
        ctas[kind] = pick;
        g_tuned_ctas[kind] = pick;
    }
    CK(cudaStreamSynchronize(gs));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tuned = true;
}

// ====================================================================== C ABI
namespace {
template <class Fn>
int eguard(mlegs_ensemble* e, Fn&& fn) {
    if (!e) return MLEGS_ERR_ARG;
    int64_t* prev = g_launch_counter;
    std::vector<void*>* prev_allocs = g_allocs;
    g_launch_counter = &e->launches;
    g_allocs = &e->allocs;
    int rc = MLEGS_OK;
    try {
        cudaSetDevice(e->dev);
        fn();
        cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) throw CudaError(std::string("kernel launch: ") + cudaGetErrorString(ce));
    } catch (const ApiError& x) {
        e->err = x.what();
        rc = x.code;
    } catch (const CudaError& x) {
        e->err = x.what();
        rc = MLEGS_ERR_CUDA;
    } catch (const std::exception& x) {
        e->err = x.what();
        rc = MLEGS_ERR_STATE;
    }
    g_launch_counter = prev;
    g_allocs = prev_allocs;
    return rc;
}
}  // namespace

extern "C" {

int mlegs_ensemble_create(const mlegs_params* p, int n, mlegs_ensemble** out) {
    if (!p || !out || n < 1) return MLEGS_ERR_ARG;
    *out = nullptr;
    mlegs_ensemble* e = new (std::nothrow) mlegs_ensemble();
    if (!e) return MLEGS_ERR_NOMEM;
    e->dev = p[0].device;
    for (int i = 0; i < n; ++i) {
        if (p[i].device != e->dev) {
            e->destroy();
            delete e;
            return MLEGS_ERR_ARG;
        }
        mlegs_ctx* c = nullptr;
        const int rc = mlegs_create(&p[i], &c);
        if (rc) {
            e->destroy();
            delete e;
            return rc;
        }
        e->inst.push_back(c);
    }
    const int rc = eguard(e, [&] {
        CK(cudaStreamCreateWithFlags(&e->gs, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&e->gev, cudaEventDisableTiming));
        CK(cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->dev));
        e->d_next = dalloc<int>(2);
        e->st.resize(e->inst.size());
        for (size_t i = 0; i < e->inst.size(); ++i) {
            e->st[i].c = e->inst[i];
            CK(cudaEventCreateWithFlags(&e->st[i].ev, cudaEventDisableTiming));
        }
    });
    if (rc) {
        e->destroy();
        delete e;
        return rc;
    }
    *out = e;
    return MLEGS_OK;
}

int mlegs_ensemble_destroy(mlegs_ensemble* e) {
    if (!e) return MLEGS_ERR_ARG;
    cudaSetDevice(e->dev);
    cudaDeviceSynchronize();
    e->destroy();
    delete e;
    return MLEGS_OK;
}

const char* mlegs_ensemble_last_error(const mlegs_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

int mlegs_ensemble_size(const mlegs_ensemble* e) { return e ? (int)e->inst.size() : -1; }

mlegs_ctx* mlegs_ensemble_context(mlegs_ensemble* e, int i) {
    if (!e || i < 0 || i >= (int)e->inst.size()) return nullptr;
    return e->inst[i];
}

int mlegs_ensemble_step(mlegs_ensemble* e, int nsteps, int graph) {
    return eguard(e, [&] {
        if (nsteps < 0) throw ApiError(MLEGS_ERR_ARG, "ensemble: nsteps < 0");
        e->prepare();
        int done = 0;
        if (!graph) {
            for (; done < nsteps; ++done) e->step();
            return;
        }
        if (!e->gexec) {
            if (nsteps == 0) return;
            e->step();  // eager: problems uploaded, every buffer in place
            ++done;
            if (!e->tuned) {
                CK(cudaDeviceSynchronize());
                e->tune();
            }
            if (done == nsteps) return;
            std::vector<double> t0;
            std::vector<int> n0;
            for (mlegs_ctx* c : e->inst) {
                t0.push_back(c->t);
                n0.push_back(c->n);
            }
            const int64_t before = e->launches;
            CK(cudaStreamBeginCapture(e->gs, cudaStreamCaptureModeThreadLocal));
            e->capturing = true;
            try {
                e->group_to_all();  // every instance stream joins the capture
                e->step();
            } catch (...) {
                cudaGraph_t gtmp = nullptr;
                cudaStreamEndCapture(e->gs, &gtmp);
                if (gtmp) cudaGraphDestroy(gtmp);
                e->capturing = false;
                throw;
            }
            e->capturing = false;
            CK(cudaStreamEndCapture(e->gs, &e->graph));
            e->graph_launches = e->launches - before;
            e->launches = before;
            for (size_t i = 0; i < e->inst.size(); ++i) {
                e->inst[i]->t = t0[i];
                e->inst[i]->n = n0[i];
            }
            CK(cudaGraphInstantiate(&e->gexec, e->graph, 0));
        }
        for (; done < nsteps; ++done) {
            CK(cudaGraphLaunch(e->gexec, e->gs));
            e->launches += e->graph_launches;
            for (mlegs_ctx* c : e->inst) {
                c->t += c->p.dt;
                c->n += 1;
            }
        }
    });
}

int mlegs_ensemble_tune(mlegs_ensemble* e) {
    return eguard(e, [&] {
        if (e->gb2p.up.empty()) throw ApiError(MLEGS_ERR_STATE, "ensemble: tune after a first step");
        CK(cudaDeviceSynchronize());
        e->tune();
    });
}

int mlegs_ensemble_tuning(const mlegs_ensemble* e, int32_t* out, int cap) {
    if (!e || !out || cap < 0) return -1;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    int n = 0;
    for (const auto& kv : g_tuned_nj) {
        if (n + 1 > cap) break;
        out[4 * n + 0] = std::get<0>(kv.first);
        out[4 * n + 1] = std::get<1>(kv.first);
        out[4 * n + 2] = std::get<2>(kv.first);
        out[4 * n + 3] = 8 * kv.second;
        ++n;
    }
    return n;
}

int mlegs_ensemble_ctas(const mlegs_ensemble* e, int32_t* out) {
    if (!e || !out) return MLEGS_ERR_ARG;
    out[0] = e->ctas[0];
    out[1] = e->ctas[1];
    return MLEGS_OK;
}

int mlegs_ensemble_sync(mlegs_ensemble* e) {
    return eguard(e, [&] { CK(cudaDeviceSynchronize()); });
}

int64_t mlegs_ensemble_launch_count(const mlegs_ensemble* e) { return e ? e->launches : 0; }

void* mlegs_ensemble_stream(mlegs_ensemble* e) { return e ? (void*)e->gs : nullptr; }

}  // extern "C"
