/*
 * mlegs_b200.h -- C ABI of the B200-native MLegS transform-and-step library.
 *
 * Each entry point replaces one Fortran module procedure of the reference
 * (paths relative to the MLegS project root).  Fields live on the device,
 * owned by the context; hosts move data with upload/download in the
 * reference's own array layout (Fortran column-major COMPLEX(P8) E(:,:,:)
 * with the per-space shapes of SALLOC, mod_fft.f90:603-670):
 *   FFF  E(NRCHOPDIM, NTCHOPDIM, NXCHOPDIM)
 *   PFF  E(NDIMR,     NTCHOPDIM, NXCHOPDIM)
 *   PFP  E(NDIMR,     NDIMTH,    NX)
 *   PPP  E(NDIMR,     NDIMTH,    NX)
 * with NDIMR = NR+3, NDIMTH = NTH+1, NRCHOPDIM = min(NRCHOP+6, NR),
 * NTCHOPDIM = min(NTCHOP, NTH), NXCHOPDIM = 2*NXCHOP-1 (mod_fft.f90:225-235).
 *
 * Truncation: the reference's global CHOPSET(+p)/CHOPSET(-p) state
 * (mod_scalar3.f90:165-211) becomes the explicit `pad` argument: every
 * operator uses NRCHOPS(m) = max(NRCHOP + pad - m, 0).
 *
 * Errors: every function returns 0 on success, otherwise one of the
 * reference's ERR_FLAGS codes (mod_scalar3.f90:88-106) or an MLEGS_ERR_*
 * code below; nothing aborts the process.  Calls on one context are
 * stream-ordered on that context's CUDA stream and must not be issued
 * concurrently from several host threads; distinct contexts are independent
 * (except for mlegs_idel2ln_static, whose calls share one array per device).
 */
#ifndef MLEGS_B200_H
#define MLEGS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ERR_FLAGS values of the reference (mod_scalar3.f90:88-106). */
#define MLEGS_OK                 0
#define MLEGS_ERR_SCALAR3        1
#define MLEGS_ERR_SCALAR3_ISNAN 10
#define MLEGS_ERR_DEALIASING    11
#define MLEGS_ERR_DIVERGENCE    12
#define MLEGS_ERR_LOGTERM       13
#define MLEGS_ERR_TRANSFORM      2
#define MLEGS_ERR_LEGOPERATOR    3
#define MLEGS_ERR_CALCULATION   31
#define MLEGS_ERR_DIMMISMATCH   32
#define MLEGS_ERR_SOLVER         5
/* Codes with no counterpart in the reference. */
#define MLEGS_ERR_CUDA         100
#define MLEGS_ERR_ARG          101
#define MLEGS_ERR_NOMEM        102
#define MLEGS_ERR_NONFINITE    103
#define MLEGS_ERR_STATE        104
#define MLEGS_ERR_TIMEOUT      105   /* a bounded device-side wait ran out */

/* Space tags, mod_scalar3.f90:82-85. */
#define MLEGS_PPP 0
#define MLEGS_FFF 1
#define MLEGS_PFP 2
#define MLEGS_PFF 3

/* Arithmetic of the mapped-Legendre GEMMs (RTRAN, PROJECT). */
#define MLEGS_PREC_FP64   0   /* FP64 FMA                                          */
#define MLEGS_PREC_SPLIT  1   /* split-BF16 (Ozaki) slices on tcgen05, FP64 combine */

/* Run parameters: the read.input keys the hot path reads (mod_init.f90:401-705,
 * with VISCOSITY NU/NUP >= 1 already inverted as READIN0 does, 539-551). */
typedef struct mlegs_params {
    int32_t nr, nth, nx;              /* DIMENSION                                 */
    int32_t nrchop, ntchop, nxchop;   /* CHOPS                                     */
    double  ell, zlen;                /* ELL, ZLEN (MINC = 1, MKLINK = 0)          */
    double  dt;                       /* DT                                        */
    int32_t adams;                    /* BOUSSINESQ ABSW: 1 AB2-CN, 0 ETD2AB-CN    */
    double  omega, bv0, kappa, kappap;/* BOUSSINESQ OMEGA, BV0, KAPPA, KAPPAP      */
    int32_t visc_sw, visc_p;          /* VISCOSITY SW, P                           */
    double  nu, nup;                  /* VISCOSITY NU, NUP                         */
    int32_t precision;                /* MLEGS_PREC_*                              */
    int32_t split_slices;             /* slices per operand for MLEGS_PREC_SPLIT   */
    int32_t device;                   /* CUDA device ordinal                        */
    int32_t rmv_sw;                   /* REMOVE SW: 2 turns on the axial sponge of the
                                         ETD steps (CALC_BOUSSI_ETD_SPONGE); 0 or 1
                                         leave the step as it is                      */
} mlegs_params;

typedef struct mlegs_ctx mlegs_ctx;
typedef struct mlegs_field mlegs_field;

/* Context: LEGINIT + SETUP_GRID (mod_fft.f90:165-367) for one grid; builds the
 * Gauss-Legendre nodes and the orthonormal P^m_n table in FP64 on the device. */
int mlegs_create(const mlegs_params* p, mlegs_ctx** out);
int mlegs_destroy(mlegs_ctx* ctx);
const char* mlegs_last_error(const mlegs_ctx* ctx);
/* Waits for the context's stream; returns MLEGS_ERR_TIMEOUT (once) when a
 * bounded wait inside a tensor-core kernel ran out since the last sync (the
 * results of that launch are invalid; the context stays usable). */
int mlegs_sync(mlegs_ctx* ctx);
/* Limit of the pipeline waits inside the tensor-core kernels, in SM cycles
 * (0 restores the default, about one second).  No counterpart in the
 * reference.  A short limit makes a wait run out: the kernel then drains what
 * it has in flight, frees its tensor memory and returns, and the next
 * mlegs_sync reports MLEGS_ERR_TIMEOUT; used to test that error path. */
int mlegs_set_wait_limit(mlegs_ctx* ctx, int64_t cycles);
/* Sizes (NDIMR, NDIMTH, NX, NRCHOPDIM, NTCHOPDIM, NXCHOPDIM, NRH, NR, NTH). */
int mlegs_dims(const mlegs_ctx* ctx, int32_t out[9]);

/* Fields: TYPE(SCALAR) (mod_scalar3.f90:41-47) with device storage;
 * SALLOC/SFREE (mod_fft.f90:603-703). */
int mlegs_field_alloc(mlegs_ctx* ctx, int space, mlegs_field** out);
int mlegs_field_free(mlegs_ctx* ctx, mlegs_field* f);
int mlegs_field_space(const mlegs_field* f);
/* host: interleaved (re, im) doubles in the reference layout of `space`. */
int mlegs_field_upload(mlegs_ctx* ctx, mlegs_field* f, int space, const double* host, double ln);
int mlegs_field_download(mlegs_ctx* ctx, const mlegs_field* f, double* host, double* ln);
/* Collocation grid built by mlegs_create: x (Gauss-Legendre nodes, ascending),
 * w (weights), r = ELL sqrt((1+x)/(1-x)); arrays of NR doubles (TFM%X/W/R,
 * mod_scalar3.f90:53-56).  Any pointer may be NULL. */
int mlegs_grid(const mlegs_ctx* ctx, double* x, double* w, double* r);
/* y = c*y + a*x1 + b*x2 on FFF fields, applied to E and LN alike (x2 may be
 * NULL); the array arithmetic the steppers write inline (mod_march.f90:639-643). */
int mlegs_field_axpby(mlegs_ctx* ctx, mlegs_field* y, double a, const mlegs_field* x1, double b,
                      const mlegs_field* x2, double c);
int mlegs_field_set_ln(mlegs_ctx* ctx, mlegs_field* f, double ln);
/* COPY0 (mod_fft.f90:705-769): dst = src (with CHOPDO at pad for FFF). */
int mlegs_field_copy(mlegs_ctx* ctx, mlegs_field* dst, const mlegs_field* src, int pad);
/* CHOPDO (mod_scalar3.f90:213-257). */
int mlegs_chopdo(mlegs_ctx* ctx, mlegs_field* f, int pad);

/* Space transitions, mod_fft.f90:771-1398. is = +1: towards physical, -1: towards spectral. */
int mlegs_rtran(mlegs_ctx* ctx, mlegs_field* f, int is, int pad);   /* RTRAN  1150 */
int mlegs_horfft(mlegs_ctx* ctx, mlegs_field* f, int is);           /* HORFFT  771 */
int mlegs_verfft(mlegs_ctx* ctx, mlegs_field* f, int is);           /* VERFFT  928 */
int mlegs_plnfft(mlegs_ctx* ctx, mlegs_field* f, int is);           /* PLNFFT 1115 */
int mlegs_toff(mlegs_ctx* ctx, mlegs_field* f, int pad);            /* TOFF   1342 */
int mlegs_tofp(mlegs_ctx* ctx, mlegs_field* f, int pad);            /* TOFP   1371 */

/* Spectral operators, mod_legops.f90 (b = op(a) unless noted). */
int mlegs_delsqh(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad);   /* DELSQH   76 */
int mlegs_idelsqh(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int pad);  /* IDELSQH 136 */
int mlegs_mulxm(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad);    /* MULXM   371 */
int mlegs_xxdx(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad);     /* XXDX    680 */
int mlegs_del2(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* b, int pad);     /* DEL2    751 */
/* IDEL2 (823): has_ln = 0 means the LN argument is absent. */
int mlegs_idel2(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int has_ln, double ln, int pad);
int mlegs_idel2ln(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int pad);  /* IDEL2LN 1013 */
/* IDEL2LN that allocates nothing; no counterpart in the reference.  For
 * callers that cannot call cudaMalloc where they solve (their own pool
 * allocator holds the memory they may use, or the implicit device-wide
 * synchronisation of cudaMalloc is unaffordable in their time loop).  The
 * elimination scratch is a fixed 64 MiB __device__ array inside this library,
 * held on a device from the first call there (from library load when CUDA's
 * lazy module loading is off) until the process exits; grids needing more
 * (NRCHOPDIM*4*NTCHOPDIM*NXCHOPDIM doubles > 8,388,608) get MLEGS_ERR_ARG.
 * The first call on a device looks the array up (cudaGetSymbolAddress), so
 * make it before any stream capture.  That address is cached for the life of
 * the process: a host that resets the device (cudaDeviceReset) must not call
 * this entry point afterwards.  All calls on a device share the array:
 * calls whose kernels overlap on the GPU race and must be ordered by the
 * caller.  Results equal mlegs_idel2ln's. */
int mlegs_idel2ln_static(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int pad);
int mlegs_ihelm(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, double alp, int pad); /* IHELM 1204 */
/* IHELMP(P, B, A, ALP, NUIN) (1409-1592): A = (DEL^P + nu DEL^2 - alp)^-1 B for
 * even p in 4..14 and alp /= 0 (the log term moved to the right-hand side,
 * A%LN = -B%LN/alp, the far-field fix, CHOPDO). */
int mlegs_ihelmp(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* a, int p, double alp, double nu, int pad);
/* HYPERV(A, NU, NUP, P, DT, WK) (mod_march.f90:1639-1686): one implicit
 * hyperviscosity step of A in place, IHELMP(P, alp A, A, -alp, bet) with
 * alp = (-1)^(P/2) / (dt nup), bet = -(-1)^(P/2) nu / nup.  The steppers apply
 * it to PSI, CHI (and B when KAPPAP /= 0) when VISC%SW = 2 (AB2-CN only). */
int mlegs_hyperv(mlegs_ctx* ctx, mlegs_field* a, double nu, double nup, int p, double dt);
int mlegs_grad(mlegs_ctx* ctx, const mlegs_field* a, mlegs_field* rgr, mlegs_field* rgp,
               mlegs_field* gz, int pad);                                            /* GRAD   1727 */
int mlegs_pc2vel(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi,
                 mlegs_field* rur, mlegs_field* rup, mlegs_field* uz, int pad);      /* PC2VEL 1789 */
int mlegs_pc2vor(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi,
                 mlegs_field* ror, mlegs_field* rop, mlegs_field* oz, int pad);      /* PC2VOR 1856 */
/* PROJECT (2397): ln_mode 0 = LN absent, 1 = LN given (ln), 2 = PSI%LN passed
 * by reference (the steppers' call form: PSI%LN then ends as the far-field
 * value VEL2PLN extracts). rur/rup/uz are consumed. */
int mlegs_project(mlegs_ctx* ctx, mlegs_field* rur, mlegs_field* rup, mlegs_field* uz,
                  mlegs_field* psi, mlegs_field* chi, int ln_mode, double ln);

/* Boussinesq right-hand side, mod_boussinesq.f90:317-410 (CALC_BOUSSI_FORCE). */
int mlegs_boussi_force(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi,
                       const mlegs_field* b, mlegs_field* psin, mlegs_field* chin,
                       mlegs_field* bn);

/* CALC_BOUSSI_NONLIN(B, RUR, RUP, UZ, BN, ROR, ROP, OZ), mod_boussinesq.f90:235-314:
 * GRAD(B) at CHOPSET(1), nine TOFP, VPRODSUB / VDOTPSUB, PROJECT (LN = 0),
 * IDEL2, PC2VEL at CHOPSET(3), TOFF(BN).  b, rur..oz in FFF.  On return ror,
 * rop, oz hold the velocity form of the projected u x omega (FFF), bn the
 * FFF -(u.grad)b; rur, rup, uz are consumed (the reference deallocates them):
 * they are left holding the physical velocity in PFP.  All fields distinct. */
int mlegs_boussi_nonlin(mlegs_ctx* ctx, const mlegs_field* b, mlegs_field* rur, mlegs_field* rup, mlegs_field* uz,
                        mlegs_field* bn, mlegs_field* ror, mlegs_field* rop, mlegs_field* oz);

/* TFM%PF (LEGINIT, mod_fft.f90:297): the orthonormal associated Legendre
 * table the device built, in the reference layout PF(NRH, NRCHOPDIM+1,
 * NTCHOPDIM) (column-major), NRH*(NRCHOPDIM+1)*NTCHOPDIM doubles.
 * Synchronises the context's stream. */
int mlegs_legendre_table(mlegs_ctx* ctx, double* pf);

/* Snapshots in the reference's files (mod_fft.f90:2224-2642), written and
 * read by one process: global = 1 is MSAVEX / MLOADX (one Fortran unformatted
 * file: sizes, chops, SPACE, LN, ZLEN, ELL, MINC, MKLINK, E); global = 0 is
 * MPISAVEX / MPILOADX (path.info with the header records, path with E as raw
 * COMPLEX(P8)).  E is the field in its space's reference layout.  Loading sets
 * the field's space and LN from the file; array sizes that differ from this
 * context's are MLEGS_ERR_DIMMISMATCH (the reference warns on ZLEN, ELL, MINC,
 * MKLINK and chop mismatches and loads anyway; so does this).  Records over
 * 2 GiB are not supported. */
int mlegs_msave(mlegs_ctx* ctx, const mlegs_field* f, const char* path, int global);
int mlegs_mload(mlegs_ctx* ctx, const char* path, mlegs_field* f, int global);

/* Energy diagnostics.  CALC_BOUSSI_ENERGY(PSI, CHI, B) (mod_boussinesq.f90:139-232)
 * without its file output: ke, pe, dke (any may be NULL) receive KE, PE and DKE
 * per (m >= 0, k >= 0), NTCHOP x NXCHOP doubles each in Fortran order; the
 * driver's especData_M / especData_K lines are their row / column sums.
 * MLEGS_ERR_LOGTERM when B%LN is not 0 (the reference aborts there).
 * CALC_BOUSSI_PE(B) (112-136): pe likewise, at the current chop.  Both
 * synchronise the context's stream. */
int mlegs_boussi_energy(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                        double* ke, double* pe, double* dke);
int mlegs_boussi_pe(mlegs_ctx* ctx, const mlegs_field* b, double* pe);
/* DIAGNOST(PSI, CHI) (mod_march.f90:1689-1966) without its printing and
 * stored initial values: out[11] = VALVOR, VALZMO, VALANG, VALENE, VALHEL,
 * the spread over k of |CALCAT1(PSI)| and |CALCAT1(CHI)|, the norm check's
 * |Im PSI(2,1,1) + Im CHI(2,1,1)|, and CALCXY's (1967-2047) <X>, <Y>, <R>.  The dealiasing and divergence checks
 * return MLEGS_ERR_DEALIASING / MLEGS_ERR_DIVERGENCE where the reference
 * aborts.  VALANG integrates the RTRAN(+1) image that INTEG_P forms (the
 * reference reads past its FFF argument there).  Synchronises the stream. */
int mlegs_diagnost(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, double* out);

/* One vortex of QPAIR (read.input's vortex list, mod_init.f90): centre X, Y;
 * strengths Q (toroidal) and H, decay B (poloidal); the z-waviness DX, DY
 * with axial wavenumber K and phase DP (degrees); core R with its modulation
 * DR, wavenumber RK and phase RP (degrees).  K and RK count periods per ZLEN. */
typedef struct mlegs_vortex {
    double x, y, q, h, b, dx, dy, k, dp, r, dr, rk, rp;
} mlegs_vortex;

/* QVORTEX(PSI, CHI) (mod_layout.f90:449-609) on the device: LAY(A, GAUS, 2)
 * of every vortex (Q -> 2Q, B -> 1 for PSI; Q -> H, B for CHI), TOFF, A = -A
 * with LN 0, IDELSQH.  psi and chi end in FFF.  n >= 1.
 * noise_seeds: NULL for QPAIR%NOISE = 0; else NOISE = 1 with the two RAN0
 * seeds ISEED (>= 0) for PSI and CHI, which the reference draws from
 * RANDOM_NUMBER (mod_layout.f90:175-177) and which are explicit here. */
int mlegs_qvortex(mlegs_ctx* ctx, const mlegs_vortex* vortices, int n, const int32_t* noise_seeds,
                  mlegs_field* psi, mlegs_field* chi);

/* Adaptive hyperviscosity (VISC%ADJSW /= 0 with VISC%SW = 3).
 * ENEMON(PSI, CHI, EM, EK) (mod_march.f90:2585-2617) at CHOPSET(pad):
 * em[NTCHOP] and ek[NXCHOP] (either may be NULL).  Synchronises the stream. */
int mlegs_enemon(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, int pad, double* em,
                 double* ek);
/* HYP3ADJ(PSI, CHI, B) (mod_march.f90:3000-3182) followed by the stepper's two
 * HYP3SET calls (283-288): updates NUP_R/T/X (and KAPPAP_R/T/X when b is not
 * NULL) and rewrites the HYPERV / HYPERD tables that the steps (and captured
 * step graphs) read.  The controller history persists in the context. */
int mlegs_hyp3adj(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b);
/* out[6] = NUP_R, NUP_T, NUP_X, KAPPAP_R, KAPPAP_T, KAPPAP_X. */
int mlegs_hyp3_coeffs(mlegs_ctx* ctx, double* out);
/* The host-side pieces of HYP3ADJ (no context, no device):
 * SPECURV(ESPEC(1:n), USE_RATIO) (2619-2698), SPESLOP(ESPEC(1:n), RATIO)
 * (2700-2774) and PDAJUST(COEFF, CURRENT, PREVIOUS, BASELINE, PARAMS[4]
 * [, OVERDAMP_THRESHOLD]) (2776-2812; has_threshold = PRESENT(...)). */
int mlegs_specurv(const double* espec, int n, double use_ratio, double* curv);
int mlegs_speslop(const double* espec, int n, double ratio, double* slope);
int mlegs_pdajust(double* coeff, double current, double previous, double baseline, const double* params,
                  int has_threshold, double threshold);
/* One field's HYP3ADJ controller (mod_march.f90:3025-3101) on given spectra,
 * no context: em[nm] (EM without its last two entries), ek[nk]; state[5] =
 * NUPB (negative before the first call), CURVMO, CURVKO, SLOPMO, SLOPKO, updated
 * in place; coef[3] = NUP_R, NUP_T, NUP_X, updated in place. */
int mlegs_hyp3_controller(const double* em, int nm, const double* ek, int nk, double* state, double* coef);

/* Solver: SOLVER_T%INITIALIZE (mod_march.f90:171-240, Richardson start-up) and
 * TIME_STEPPING's state update (243-307: STEP_BOUSSI_AB_CN 609 or
 * STEP_BOUSSI_ETDAB_CN 811).  The state fields stay owned by the caller. */
int mlegs_solver_init(mlegs_ctx* ctx, mlegs_field* psi, mlegs_field* chi, mlegs_field* b);
int mlegs_step(mlegs_ctx* ctx, int nsteps);
/* Capture one steady-state step as a CUDA graph and replay it nsteps times. */
int mlegs_step_graph(mlegs_ctx* ctx, int nsteps);
/* nsteps graph-replayed steps with the state streamed through host memory:
 * per step the same as mlegs_field_upload(psi, chi, b in FFF from host[0..2],
 * LN ln[0..2]), mlegs_step_graph(ctx, 1) and mlegs_field_download into the
 * same buffers (host-driven time stepping, TIME_STEPPING mod_march.f90:243-307,
 * with the state on the host between steps).  host[i] is a FFF array in the
 * reference layout (NRCHOPDIM x NTCHOPDIM x NXCHOPDIM complex, Fortran order),
 * page-locked for the copies to overlap; ln is read at the start and holds the
 * last step's LN values on return.  The copies run on their own streams, each
 * direction on its own: the upload of field i for the next step waits only for
 * field i's download, so it overlaps the downloads of the fields after it.
 * Returns after the last download; nsteps = 0 only sets up the streams and
 * buffers (3 + 3 FFF staging arrays on the device). */
int mlegs_run_host(mlegs_ctx* ctx, int nsteps, double* const* host, double* ln);
/* Simulation time and step counter (TIM%T, TIM%N). */
int mlegs_time(const mlegs_ctx* ctx, double* t, int32_t* n);
/* Non-finite check of the state (ANYNAN, mod_scalar3.f90:998-1045):
 * returns MLEGS_ERR_NONFINITE if any state coefficient is NaN/Inf. */
int mlegs_check_finite(mlegs_ctx* ctx);

/* Ensembles: n independent AB2-CN runs of different grids (the batched-run
 * configuration) on one device, advanced in lock-step.  No counterpart in the
 * reference, which runs one instance per MPI job.  Each instance is a context
 * as mlegs_create makes it (fields, uploads, mlegs_solver_init and downloads
 * go through mlegs_ensemble_context(e, i); the ensemble owns and destroys
 * them).  mlegs_ensemble_step advances every instance by nsteps AB2-CN steps
 * (STEP_BOUSSI_AB_CN, mod_march.f90:609-661): per step, the Legendre GEMMs of
 * all instances (10 RTRAN(+1); PROJECT's five products and one RTRAN(-1)) and
 * their banded solves (IDEL2LN; IHELM) run as four grouped launches, the GEMMs
 * persistent with a global work counter, everything else per instance on its
 * own stream.  graph = 1 runs the first step eagerly, autotunes the grouped
 * GEMMs (mlegs_ensemble_tune) and captures one step as a CUDA graph over all
 * streams for the rest.  Requirements: every instance FP64, BOUSSINESQ ABSW =
 * 1, mlegs_solver_init done, NRH <= 96 and NRCHOPDIM <= 190. */
typedef struct mlegs_ensemble mlegs_ensemble;
int mlegs_ensemble_create(const mlegs_params* p, int n, mlegs_ensemble** out);
int mlegs_ensemble_destroy(mlegs_ensemble* e);
const char* mlegs_ensemble_last_error(const mlegs_ensemble* e);
int mlegs_ensemble_size(const mlegs_ensemble* e);
mlegs_ctx* mlegs_ensemble_context(mlegs_ensemble* e, int i);
int mlegs_ensemble_step(mlegs_ensemble* e, int nsteps, int graph);
/* Autotuner: per class of GEMM problems (transform, NRH, NRCHOP) the column
 * tile (16 or 32 columns) with the shortest grouped launch (best of 3), then
 * persistent CTAs per SM (2, 3, 4) per transform; cached for the process.
 * Needs one step first.  mlegs_ensemble_tuning writes up to cap rows
 * (transform 0 RTRAN(+1) / 1 fold, NRH, NRCHOP, tile columns) and returns the
 * row count; mlegs_ensemble_ctas writes the two CTA-per-SM choices. */
int mlegs_ensemble_tune(mlegs_ensemble* e);
int mlegs_ensemble_tuning(const mlegs_ensemble* e, int32_t* out, int cap);
int mlegs_ensemble_ctas(const mlegs_ensemble* e, int32_t* out);
int mlegs_ensemble_sync(mlegs_ensemble* e);
int64_t mlegs_ensemble_launch_count(const mlegs_ensemble* e);
void* mlegs_ensemble_stream(mlegs_ensemble* e);

/* ---- Adjoint (vector-Jacobian products) of the AB2-CN path.  No counterpart in
 * the reference (it has no adjoint); these replace nothing and bind only from
 * the Python gradient path.  Transposes are for the real inner product
 * <a, b> = sum(Re a Re b + Im a Im b) over the stored entries, plus LN_a LN_b
 * where a field's log term enters the map.  FP64 contexts only; the step maps
 * and VJPs need AB2-CN with VISC%SW = 1.  Synchronise with mlegs_sync before
 * the host reads results. */

/* One transpose (op: MLEGS_T_* below) at CHOPSET(pad): y[] the cotangents of
 * the operator's outputs, x[] receives those of its inputs.  p1: ALP for
 * MLEGS_T_IHELM, NU for MLEGS_T_VISC2 (DT from the context). */
#define MLEGS_T_RTRAN_P      0   /* RTRAN(+1)^T:  y PFF -> x FFF (with LN)            */
#define MLEGS_T_RTRAN_M      1   /* RTRAN(-1)^T:  y FFF -> x PFF                      */
#define MLEGS_T_VERFFT_P     2   /* VERFFT(+1)^T: y PFP -> x PFF                      */
#define MLEGS_T_VERFFT_M     3   /* VERFFT(-1)^T: y PFF -> x PFP                      */
#define MLEGS_T_HORFFT_P     4   /* HORFFT(+1)^T: y PPP -> x PFP                      */
#define MLEGS_T_HORFFT_M     5   /* HORFFT(-1)^T: y PFP -> x PPP                      */
#define MLEGS_T_TOFP         6   /* TOFP^T:  y PPP -> x FFF (with LN)                 */
#define MLEGS_T_TOFF         7   /* TOFF^T:  y FFF -> x PPP                           */
#define MLEGS_T_XXDX         8   /* XXDX^T   (with LN)                                */
#define MLEGS_T_MULXM        9   /* MULXM^T                                           */
#define MLEGS_T_DELSQH      10   /* DELSQH^T (with LN)                                */
#define MLEGS_T_DEL2        11   /* DEL2^T   (with LN)                                */
#define MLEGS_T_GRAD        12   /* GRAD^T:   y[3] -> x[0]                            */
#define MLEGS_T_PC2VEL      13   /* PC2VEL^T: y[3] -> x[0] psi, x[1] chi              */
#define MLEGS_T_PC2VOR      14   /* PC2VOR^T: y[3] -> x[0] psi, x[1] chi              */
#define MLEGS_T_IDEL2LN     15   /* IDEL2LN^T at CHOPSET(0): y (with LN) -> x         */
#define MLEGS_T_IHELM       16   /* IHELM^T at CHOPSET(0): y (with LN) -> x (with LN) */
#define MLEGS_T_PROJECT_PPP 17   /* PROJECT(.., PSI, W, 0.0) of PPP inputs: y[0] PSI, y[1] W -> x[3] PPP */
#define MLEGS_T_VISC2       18   /* VISC2^T: y -> x[0] A, x[1] AO                     */
#define MLEGS_T_IDELSQH     19   /* IDELSQH^T (y with LN)                             */
#define MLEGS_T_FARFIELD    20   /* the far-field fix (CALCAT1) transposed            */
int mlegs_transpose(mlegs_ctx* ctx, int op, const mlegs_field* const* y, mlegs_field* const* x, int pad, double p1);

/* VJP of CALC_BOUSSI_FORCE (mod_boussinesq.f90:317-410) at (psi, chi, b):
 * output cotangents (psin_bar, chin_bar with LN, bn_bar) -> input cotangents. */
int mlegs_boussi_force_vjp(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                           const mlegs_field* psin_bar, const mlegs_field* chin_bar, const mlegs_field* bn_bar,
                           mlegs_field* psi_bar, mlegs_field* chi_bar, mlegs_field* b_bar);

/* One steady STEP_BOUSSI_AB_CN (mod_march.f90:609-661) as a map of the state
 * (psi, chi, b, n_psi, n_chi, n_b) = in[6] -> out[6], and its VJP at state[3]
 * (psi, chi, b before the step): bar[6] -> out[6].  The map leaves the
 * context's own solver state, history and time unchanged. */
int mlegs_ab2_step_map(mlegs_ctx* ctx, const mlegs_field* const* in, mlegs_field* const* out);
int mlegs_ab2_step_vjp(mlegs_ctx* ctx, const mlegs_field* const* state, const mlegs_field* const* bar,
                       mlegs_field* const* out);
/* RICH_BOUSSI_FE_BE (535-606) as the map (psi, chi, b) = in[3] -> out[6]
 * (state and history), and its VJP at state[3]: bar[6] -> out[3]. */
int mlegs_ab2_startup_map(mlegs_ctx* ctx, const mlegs_field* const* in, mlegs_field* const* out);
int mlegs_ab2_startup_vjp(mlegs_ctx* ctx, const mlegs_field* const* state, const mlegs_field* const* bar,
                          mlegs_field* const* out);
/* Transpose of the seeded initial state psi = vortex + IDELSQH(-c_psi), chi
 * likewise, b = c_b with the CALCAT1 far-field fix: state_bar[3] -> coef_bar[3]. */
int mlegs_initial_state_T(mlegs_ctx* ctx, const mlegs_field* const* state_bar, mlegs_field* const* coef_bar);
/* J = fluctuation kinetic energy (CALC_BOUSSI_ENERGY's quadrature,
 * mod_boussinesq.f90:176-206, without the (m, k) = (0, 0) part) + 1/2 int b^2 dV
 * (CALC_BOUSSI_PE's quadrature, 112-136) and its gradient (gpsi, gchi, gb).
 * Synchronises the context's stream. */
int mlegs_energy_objective(mlegs_ctx* ctx, const mlegs_field* psi, const mlegs_field* chi, const mlegs_field* b,
                           double* J, mlegs_field* gpsi, mlegs_field* gchi, mlegs_field* gb);
/* Device-to-device copy between a field and a caller's device buffer in the
 * device layout of `space` (FFF [m][n][k], PFF [m][r][k], PFP [r][z][m], PPP
 * [r][z][j], complex doubles): to_field 1 copies dev -> f (and LN from ln_dev,
 * or LN 0 when ln_dev is null), 0 copies f -> dev (LN to ln_dev when given).
 * Ordered on the context's stream. */
int mlegs_field_device_copy(mlegs_ctx* ctx, mlegs_field* f, int to_field, int space, void* dev, double* ln_dev);

/* Kernel timing for profiling and roofline reports: launches one internal
 * kernel `reps` times on scratch fields of this context, bracketed by CUDA
 * events on the context's stream, and returns the mean device time per launch
 * (ms) and the kernel's algorithmic HBM bytes per launch.  No counterpart in
 * the reference.  kernel ids: MLEGS_K_* below. */
#define MLEGS_K_RTRAN_B2P   0   /* RTRAN(+1)  FFF -> PFF               */
#define MLEGS_K_RTRAN_P2B   1   /* RTRAN(-1)  PFF -> FFF               */
#define MLEGS_K_VERFFT_B    2   /* VERFFT(+1) PFF -> PFP               */
#define MLEGS_K_VERFFT_F    3   /* VERFFT(-1) PFP -> PFF               */
#define MLEGS_K_HORFFT_B    4   /* HORFFT(+1) PFP -> PPP               */
#define MLEGS_K_HORFFT_F    5   /* HORFFT(-1) PPP -> PFP               */
#define MLEGS_K_POINTWISE   6   /* VPRODSUB+VDOTPSUB+linear terms, PPP */
#define MLEGS_K_SOLVE       7   /* IDEL2LN banded solves               */
#define MLEGS_K_PHYS        8   /* fused HORFFT+VPRODSUB+VDOTPSUB+linear+HORFFT, PFP -> PFP */
#define MLEGS_K_HORFFT_WB   9   /* warp-per-line HORFFT(+1) PFP -> PPP */
#define MLEGS_K_HORFFT_WF  10   /* warp-per-line HORFFT(-1) PPP -> PFP */
#define MLEGS_K_SPLIT_B2P  11   /* RTRAN(+1) as split-BF16 tcgen05 GEMM (MLEGS_PREC_SPLIT contexts) */
#define MLEGS_K_SPLIT_P2B  12   /* RTRAN(-1) as split-BF16 tcgen05 GEMM (MLEGS_PREC_SPLIT contexts) */
#define MLEGS_K_PROJECT    13   /* PROJECT's five EOMUL/OEMUL products, 3 PFF -> 2 FFF */
#define MLEGS_K_PROJECT_FFF 14  /* PROJECT of FFF velocity fields via composite matrices, 3 FFF -> 2 FFF */
#define MLEGS_K_PHYS_NONLIN 15  /* MLEGS_K_PHYS as CALC_BOUSSI_NONLIN runs it: 9 inputs, no linear terms */
#define MLEGS_K_ROUNDTRIP  16   /* TOFP then TOFF of one field, FFF -> PPP -> FFF (context's precision) */
#define MLEGS_K_DMMA_PEAK  17   /* the FP64 tensor path's ceiling: register-only m8n8k4 MMAs, 4 CTAs x 8
                                   warps per SM; bytes_per_launch returns its FLOPs instead (MLEGS_ERR_ARG
                                   if a field buffer cannot hold one double per thread) */
int mlegs_kernel_time(mlegs_ctx* ctx, int kernel, int reps, double* ms_per_launch, double* bytes_per_launch);

/* Number of this library's kernel launches issued since the counter was reset. */
int64_t mlegs_launch_count(const mlegs_ctx* ctx);
void    mlegs_reset_launch_count(mlegs_ctx* ctx);
/* CUDA stream of the context (cudaStream_t), for event timing by hosts. */
void*   mlegs_stream(mlegs_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* MLEGS_B200_H */
