/*
 * laph_gpu.h -- C ABI of liblaph_gpu.so, the B200 (sm_100a) implementation of
 * the per-timeslice LapH eigensystem path of HISKP-LQCD/LapH_EigSys:
 *   smearing (HYP / APE / stout)  ->  Chebyshev-accelerated covariant
 *   Laplacian matvec  ->  lowest-nev eigensolve  ->  phase fixing.
 *
 * Every entry point returns an int status (LAPH_OK = 0) and never exits the
 * process; laph_last_error() gives a one-line message for the calling thread.
 * Plain pointers and sizes only.  "Host" pointers are ordinary CPU memory and
 * are staged through the context's stream; "device" pointers are CUDA global
 * memory of the context's device and are used in place.
 *
 * Threads: a context (laph_ctx) or a solver (laph_solver) is used by one thread
 * at a time; separate contexts and solvers, on one device or several, may be
 * driven from separate threads at once, each on its own CUDA stream.  The
 * host-only functions (file I/O, parsing, fix_phase, ...) are reentrant.
 *
 * Conventions (identical to the reference):
 *   site      = x*L*L + y*L + z                     (modules/navigation.cpp:27-88)
 *   vector    = complex128[3*V3], index 3*site+colour (modules/shell_matop.cpp:33-38)
 *   eigvecs   = column-major complex128 [3*V3][nev]   (src/ev_ts.cpp:298)
 *   eigvals   = eigenvalues of Delta = hop - 6, i.e. -lambda(-Delta) <= 0, in
 *               ascending order of lambda (recover_spectrum, modules/recover_spec.cpp:45-54)
 */
#ifndef LAPH_GPU_H_
#define LAPH_GPU_H_
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum {
  LAPH_OK = 0,
  LAPH_EINVAL = 1,     /* bad argument */
  LAPH_ECUDA = 2,      /* CUDA runtime error */
  LAPH_ENOMEM = 3,     /* device or host allocation failed */
  LAPH_EIO = 4,        /* cannot open/read/write (reference: exit(500)) */
  LAPH_ENORECORD = 5,  /* no ildg-binary-data record (reference: exit(-2)) */
  LAPH_ESIZE = 6,      /* record size does not match lattice (reference: exit(501)) */
  LAPH_ESINGLE = 7,    /* single-precision ILDG payload (reference: "Not implemented") */
  LAPH_ENOTCONV = 8,   /* eigensolver stopped at max_it before nev pairs converged */
  LAPH_ETIMEOUT = 9,   /* a bounded device wait gave up */
  LAPH_ETRACE = 10,    /* tr(V^dag V) / sum(V^dag V) check failed (reference check_trace) */
  LAPH_EPARSE = 11,    /* parameters.txt line the reference parser cannot read, or an
                          ildg-format record without its lattice and precision */
  LAPH_ENODEV = 12     /* no CUDA device */
};
const char* laph_strerror(int status);
const char* laph_last_error(void);
int laph_version(void);
/* The device architecture the library's kernels were built for, as the CUDA
 * runtime reports it (cudaFuncAttributes::binaryVersion: 100 = sm_100a). */
int laph_binary_version(int* version);
/* The device's FP64 throughput measured in place (TFLOP/s): a saturating loop
 * of fma.rn.f64 and one of mma.sync.m8n8k4.f64 (the FP64 tensor path), each
 * timed with CUDA events; the denominators of the FP64 kernels' rooflines.
 * No counterpart in the reference. */
int laph_probe_fp64(int device, double* fma_tflops, double* dmma_tflops);

/* ---- bounds-checked build ---------------------------------------------------
 * liblaph_gpu_check.so is the same library compiled with -DLAPH_CHECK: every
 * lattice neighbour index, the filter's coefficient and staging offsets and
 * the dense kernels' tile and column indices are checked against their ranges
 * in the kernels.  An index out of range is counted and the first one
 * recorded, and its access goes to index 0 instead (nothing traps, nothing
 * leaves its buffer).  No counterpart in the reference (it has no sanitizer
 * runs).  laph_check_enabled: 1 in the checked build, 0 otherwise.
 * laph_check_report: *count = indices out of range so far, summed over the
 * library's translation units; the first one's value, bound, source line and
 * unit (any pointer but count may be NULL); reset != 0 clears the records.
 * In the normal build *count is always 0.  laph_check_selftest (checked build
 * only; LAPH_EINVAL otherwise) runs a kernel that checks one index past its
 * bound, which the next report shows. */
int laph_check_enabled(void);
int laph_check_report(unsigned long long* count, long long* index, long long* bound, int* line, char* unit,
                      int unit_len, int reset);
int laph_check_selftest(int device);

/* ---- link layouts accepted at the boundary -------------------------------- */
enum {
  LAPH_LAYOUT_ROWMAJOR = 0, /* double[V3][3][3][3][2]: [site][dir][a][b][re,im]                */
  LAPH_LAYOUT_EIGEN = 1,    /* double[V3][3][9][2]: Matrix3cd memory (column-major 3x3),
                               the order write_link_matrices_ts dumps (read_write.cpp:263-274) */
  LAPH_LAYOUT_CONF = 2      /* one timeslice of the read_lime_gauge_field_doubleprec_timeslices
                               buffer: double[V3][4][3][3][2], slot 0 = U_t, 1..3 = U_x..U_z
                               (io.cpp:112-131, mapped as timeslice.cpp:34-79)              */
};
enum { LAPH_SMEAR_NONE = 0, LAPH_SMEAR_HYP = 1, LAPH_SMEAR_STOUT = 2, LAPH_SMEAR_APE = 3 };

/* ---- single-timeslice context: the MatShell drop-in ------------------------
 * Replaces the process-global IO/Nav/Tslice singletons the reference's
 * MatMult_Laplacian2D reads (modules/shell_matop.cpp:9-11): one context holds
 * one timeslice's links on one device, plus LAM_L, LAM_C and DEG.           */
typedef struct laph_ctx laph_ctx;
typedef struct {
  int L;          /* spatial extent LX = LY = LZ (par_io.cpp:110-112)               */
  double lam_l;   /* LAM_L, upper end of the Chebyshev window (shell_matop.cpp:18) */
  double lam_c;   /* LAM_C, cut (shell_matop.cpp:19)                               */
  int deg;        /* DEG, Chebyshev degree (shell_matop.cpp:143)                   */
  int device;     /* CUDA device ordinal                                           */
} laph_params;

int laph_ctx_create(laph_ctx** ctx, const laph_params* p);
int laph_ctx_destroy(laph_ctx* ctx);
int laph_ctx_set_window(laph_ctx* ctx, double lam_l, double lam_c, int deg);
/* The context's CUDA stream (a cudaStream_t): every device call of the
 * context runs on it, so callers can time the products with their own events. */
int laph_ctx_stream(laph_ctx* ctx, void** stream);

/* Load one timeslice of links (host pointer, FP64).  Replaces
 * Tslice::map_timeslice_to_eigen (modules/timeslice.cpp:34-79) for
 * layout = LAPH_LAYOUT_CONF, and Tslice::set_gauge for the others. */
int laph_set_links(laph_ctx* ctx, const double* links, int layout);
/* Read the (smeared) links back, Tslice::get_gauge (timeslice.cpp:81-83). */
int laph_get_links(laph_ctx* ctx, double* links, int layout);

/* FP64 smearing on the device.  kind = LAPH_SMEAR_HYP: p1 = alpha_1, p2 = alpha_2
 * (Tslice::smearing_hyp, timeslice.cpp:243-369); LAPH_SMEAR_STOUT: p1 = rho
 * (smearing_stout, :145-193); LAPH_SMEAR_APE: p1 = alpha (smearing_ape, :196-239).
 * compat = 1 keeps the reference's backward-staple factor U[nu][dir] of
 * stout/APE (timeslice.cpp:171-172, :221-222); compat = 0 uses the
 * gauge-covariant U[nu][not_dir].  HYP ignores compat (its staples are correct). */
int laph_smear(laph_ctx* ctx, int kind, double p1, double p2, int iters, int compat);

/* y = T_deg(B) x in FP64, B = c(hop - 6) + a, c = 2/(LAM_L - LAM_C),
 * a = 1 + c LAM_C: the body of MatMult_Laplacian2D (shell_matop.cpp:136-168,
 * :226-244).  deg >= 1 (deg = 1 gives B x).  x, y: complex128[3*V3];
 * on_device = 0 for host pointers (staged), 1 for device pointers, which must
 * not overlap (LAPH_EINVAL).  The whole recurrence is one cooperative launch. */
int laph_matmult(laph_ctx* ctx, const double* x, double* y, int deg, int on_device);
/* laph_matmult_noalloc: the same y = T_deg(B) x in FP64 without any device
 * allocation, for callers that may not call cudaMalloc where they need the
 * product (a framework that owns the device memory budget through its own
 * pool, a service that allocates only at start-up, a loop that cannot take
 * cudaMalloc's implicit synchronisation).  No counterpart in the reference.
 * links: device pointer, LAPH_LAYOUT_ROWMAJOR, one timeslice of L^3 sites;
 * x, y: device pointers, complex128[3*L^3], not overlapping (LAPH_EINVAL);
 * work is queued on `stream` (a cudaStream_t, 0 = legacy default) and the
 * call returns without waiting.  The two Chebyshev temporaries live in a
 * fixed file-scope device array of 3 MiB that holds timeslices up to L = 32;
 * larger L returns LAPH_EINVAL.  The first call in each CUDA context resolves
 * that array's address (make it before any stream capture).  Calls that
 * overlap on the GPU share the array and race: serialise them on one stream. */
int laph_matmult_noalloc(const double* links, int L, double lam_l, double lam_c, int deg, const double* x,
                         double* y, void* stream);
/* y = (-Delta) x = 6x - hop(x) in FP64 (for residuals). */
int laph_apply_neglap(laph_ctx* ctx, const double* x, double* y, int on_device);
/* MatGetDiagonal_Laplacian2D (shell_matop.cpp:248-255): fills diag with -6. */
int laph_get_diagonal(laph_ctx* ctx, double* diag, int on_device);
/* Average spatial plaquette of the context's links (config_utils.cpp:388-426). */
int laph_plaquette(laph_ctx* ctx, double* plaq);

/* The plain form: SLEPc-style Krylov-Schur (EPS_HEP, EPS_LARGEST_MAGNITUDE,
 * ncv <= 0 -> max(2 nev, nev + 15), convergence |beta s_i| <= tol |theta_i|)
 * on T_deg(B) of the context (window and deg of laph_ctx_set_window), the
 * EPSSolve of src/ev_ts.cpp:231-263 driving this library's MatMult.
 * device_basis = 0: Krylov basis in host memory, every product through
 * laph_matmult with host vectors (the reference's data flow); 1: basis in
 * device memory (SLEPc with CUDA vectors).  theta_out[nev]: eigenvalues of
 * T_deg(B) by decreasing |theta|; V_out (host, may be NULL): column-major
 * complex128 [3 V3][nev] Ritz vectors.  LAPH_ENOTCONV if max_it restarts did
 * not converge nev pairs (the reference silently sets nconv = nev). */
int laph_eps_solve(laph_ctx* ctx, int nev, int ncv, double tol, int max_it, int device_basis, uint64_t seed,
                   double* theta_out, double* V_out, int* nconv, int* restarts, long long* nmatvec);

/* The same Krylov-Schur on any Hermitian operator given as a host callback
 * mult(user, x, y): y = Op x on host complex128 vectors of length dim (returns
 * 0 on success) -- the EPSSolve that drives a registered MATOP_MULT.  Host
 * memory only; needs no device.  Same outputs as laph_eps_solve. */
int laph_eps_solve_cb(long long dim, int (*mult)(void* user, const double* x, double* y), void* user, int nev,
                      int ncv, double tol, int max_it, uint64_t seed, double* theta_out, double* V_out, int* nconv,
                      int* restarts, long long* nmatvec);

/* ---- batched block eigensolver (the "chosen" form) ------------------------
 * Solves many timeslices (possibly of different L and nev) in one batched,
 * device-resident Chebyshev-filtered subspace iteration: FP32 filter matvecs
 * (links FP32 or BF16 + per-site scale), FP64 Gram/Cholesky/Rayleigh-Ritz and
 * residuals.  Replaces, per timeslice, the body of the ev_ts loop
 * (src/ev_ts.cpp:176-336): smearing, MatShell + EPSSolve, fix_phase,
 * recover_spectrum. */
enum { LAPH_WINDOW_FIXED = 0, LAPH_WINDOW_LANCZOS = 1, LAPH_WINDOW_MLP = 2 };
enum { LAPH_LINKS_FP32 = 0, LAPH_LINKS_BF16 = 1 };

typedef struct {
  int L;             /* spatial extent of this timeslice                       */
  int nev;           /* wanted eigenpairs                                      */
} laph_problem;

typedef struct {
  int smear_kind;       /* LAPH_SMEAR_*                                          */
  double smear_p1, smear_p2;
  int smear_iters;
  int smear_compat;
  int guard;            /* block vectors beyond nev (>= 0); the block width
                           nev + guard is rounded up to a multiple of 32         */
  int link_prec;        /* LAPH_LINKS_FP32 / LAPH_LINKS_BF16                      */
  double tol;           /* target ||(-Delta)v - lambda v|| / (||v|| lambda_max)   */
  int max_it;           /* outer iterations                                       */
  int window;           /* LAPH_WINDOW_*                                          */
  double lam_cut;       /* fixed window: cut (<= 0: from the first Rayleigh-Ritz) */
  double lam_max;       /* fixed window: upper end (<= 0: Lanczos bound)          */
  int deg;              /* filter degree cap, 2..128 (default 16; 48-60 measured
                           best at 24^3-48^3; laph_solver_autotune picks it)     */
  int phase_fix;        /* apply fix_phase to the output eigenvectors             */
  uint64_t seed;        /* start block                                            */
  int block;            /* columns per CTA of the filter kernel, 1..512 (0: 32);
                           above 64 the filter runs as variant 0               */
  int filter_kernel;    /* filter variant, all with register-resident forward
                           links and L2 bulk prefetch: 0 FP64 coefficients per
                           thread; 1 FP32 coefficients staged per CTA, backward
                           links in shared memory (default; block <= 64); 2 as 1
                           with the backward links in tensor memory; 3 as 2 with
                           the vectors staged by a bulk-copy pipeline; 4 as 2 on
                           512-site bricks; 5 as 2 with each thread's next-column
                           operands in flight through cp.async (2-5: block <= 64;
                           3 and 4 need every L in {16, 32, 64, 128}, else 1
                           runs).  All give the same results bit for bit; 1 is
                           the fastest measured                                  */
  int jacobi_sweeps;    /* cap on Jacobi sweeps per Rayleigh-Ritz (0: 2); an
                           unfinished sweep set only delays convergence, since
                           residuals are always computed from the new vectors   */
  double window_margin; /* learned window: first-pass cut = margin x the
                           predicted converged cut (<= 0: the calibrated 1.4)  */
  int host_loop;        /* 0 (default): the whole solve is one CUDA graph launch
                           whose WHILE node repeats the outer iteration on the
                           device; 1: the host drives the outer iteration (one
                           filter graph and one Rayleigh-Ritz graph per pass,
                           the convergence mask read each pass), also taken
                           with LAPH_TRACE set                                   */
  int filter_tile;      /* sites per CTA of the filter (64, 128 or 256; 0: 128);
                           laph_solver_autotune picks it                        */
  double direct_resid;  /* a pass whose problem's largest wanted residual
                           (relative to lam_max) is above this filters V itself
                           in FP32, W = T_{m-1}(B) V, instead of the FP64-exact
                           part plus the FP32 correction (no S in its steps, 72
                           instead of 96 B per site-vector-step), until a direct
                           pass fails to halve the residual; < 0 turns it off,
                           and BF16 links never use it (default 1e-3)          */
} laph_solve_opts;
void laph_solve_opts_default(laph_solve_opts* o);

typedef struct {
  int status;           /* LAPH_OK or LAPH_ENOTCONV                               */
  int iters;            /* outer iterations used                                  */
  int nconv;            /* converged wanted pairs                                 */
  int deg;              /* filter degree used                                     */
  double lam_cut0, lam_max;  /* initial window                                    */
  double max_resid;     /* max over the nev wanted pairs                          */
  double trace_vdv;     /* tr(V^dag V) of the returned eigenvectors               */
  int window_fallback;  /* 1: the learned first window failed its check after
                           the first pass and the solve went on with the
                           non-learned window (lam_max back to 12)             */
} laph_result;

typedef struct laph_solver laph_solver;
/* Allocate a solver for n problems (device memory sized for all of them). */
int laph_solver_create(laph_solver** s, const laph_problem* probs, int n, const laph_solve_opts* opts, int device);
int laph_solver_destroy(laph_solver* s);
/* Links of problem i: FP64, layout as above; host (on_device = 0) or device pointer. */
int laph_solver_set_links(laph_solver* s, int i, const double* links, int layout, int on_device);
/* Run: smear + solve all problems.  Results stay on the device; results (may be
 * NULL) receives one laph_result per problem.  With the environment variable
 * LAPH_TRACE=1 each outer iteration prints one line to stderr: active, locked
 * and converged counts, the largest wanted residual, the filter degree and the
 * phase times of the small dense step. */
int laph_solver_run(laph_solver* s, laph_result* results);
/* Fetch problem i: evals[nev] (reference convention, see top), evecs column-major
 * complex128 [3*V3][nev] (may be NULL), phases[nev] (may be NULL). */
int laph_solver_get(laph_solver* s, int i, double* evals, double* evecs, double* phases, int on_device);
/* The same results without waiting: the copies are queued on a read-back
 * stream of the solver and overlap whatever the solver does next (the next
 * laph_solver_set_links / laph_solver_run), which waits only for the
 * conversion of the eigenvectors out of the solver's block, not for the
 * copies.  evals, evecs, phases: host buffers as for laph_solver_get (any may
 * be NULL); page-locked memory makes the copies truly asynchronous.  They are
 * complete after laph_solver_wait.  The first call allocates a device staging
 * pool of sum(3 V3 nev) complex128 for the batch. */
int laph_solver_get_async(laph_solver* s, int i, double* evals, double* evecs, double* phases);
int laph_solver_wait(laph_solver* s);
/* The CUDA stream (cudaStream_t) every kernel and copy of the solver runs on,
 * for callers that time or order work around laph_solver_run. */
int laph_solver_stream(laph_solver* s, void** stream);
/* Device-side timing of the last run (ms): smearing, filter, dense, total. */
int laph_solver_timings(laph_solver* s, double* ms4);
/* Counters of the last run for roofline accounting: filter site-vector-steps,
 * number of filter kernel launches, total device kernel launches. */
int laph_solver_counters(laph_solver* s, long long* c3);
/* Algorithmic bytes of the last run's filter passes (lap_cheb_mrhs): b2[0] =
 * what the correction-form recurrence must move (per unlocked site-vector and
 * step 24 B for each of X, Z, S read and Y written, the last step FP64 V read
 * and W written, W = V for locked columns, the links once per column block),
 * b2[1] = the plain recurrence's unit, 72 B per site-vector-step (X, Z read, Y
 * written) plus the links once per column block. */
int laph_solver_filter_bytes(laph_solver* s, double* b2);
/* How the last run looped: device_loop = 1 when the whole solve was one
 * graph launch (the WHILE node on the device), 0 when the host drove the
 * outer iteration; graph_launches = the graph launches it made (1, or two
 * per pass for the host loop). */
int laph_solver_loop_info(laph_solver* s, int* device_loop, long long* graph_launches);

/* Device memory a solver for probs[0..n) with opts allocates (bytes, each
 * allocation rounded up to 2 MiB), without touching a device. */
int laph_solver_footprint(const laph_problem* probs, int n, const laph_solve_opts* opts, long long* bytes);
/* Largest m <= n such that a solver for probs[0..m) fits in `fraction` of the
 * device's free memory now: the wave size for batches that do not fit at once
 * (48^3 x 96 at nev 220 needs ~650 GB).  LAPH_ENOMEM (nmax = 0) if even one
 * problem does not fit. */
int laph_solver_max_batch(const laph_problem* probs, int n, const laph_solve_opts* opts, int device, double fraction,
                          int* nmax);

/* ---- autotuner ------------------------------------------------------------
 * Picks the filter degree cap (deg), the filter's columns per CTA (block) and
 * the guard vectors (hence the block width k) for a batch, by timing solves of
 * a sample of it.  No counterpart in the reference, whose DEG, LAM_L and LAM_C
 * are set by hand in parameters.txt. */
typedef struct {
  int deg, block, guard;   /* the chosen settings (also written to opts)         */
  double ms_per_problem;   /* device time per problem with them, on the sample   */
  int trials;              /* settings timed (0 when read from the cache)        */
  int from_cache;          /* 1: taken from the cache file, nothing timed        */
  int tile;                /* filter sites per CTA (laph_solver_autotune only)    */
} laph_tune_result;
/* One trial: device ms per problem of the setting, or < 0 if it failed. */
typedef double (*laph_tune_trial)(void* user, int deg, int block, int guard);
/* The search with a caller-supplied trial: from (deg0, block0, guard0), each
 * axis in turn (deg, block, guard), every candidate of the axis timed with the
 * others at their best so far; a candidate replaces the best only when more
 * than 1% faster; no setting is timed twice.  LAPH_ENOTCONV if none succeeded. */
int laph_autotune_search(const int* deg_c, int nd, const int* block_c, int nb, const int* guard_c, int ng, int deg0,
                         int block0, int guard0, laph_tune_trial trial, void* user, laph_tune_result* out);
/* Tune opts (deg, block, guard; every other field kept) for a batch shaped like
 * probs[0..n): the sample is the first min(n, nsample) problems, links[i] their
 * FP64 host links in `layout`; each setting is timed as the faster of two runs
 * of a solver over the sample (the first also captures its CUDA graphs), a
 * setting that does not converge within opts->max_it is dropped.  model /
 * nmodel: the window model (as laph_solver_set_window_model) when
 * opts->window is LAPH_WINDOW_MLP, else ignored (may be NULL).  Candidates:
 * deg 40, 48, 56, 60, 64, 72, 80, 96 (start: opts->deg, or 60 if <= 1), block 8, 16, 32, 64
 * (start: opts->block, or 32), guard opts->guard, opts->guard + 32 and the fewest
 * (>= 4) that give the smallest block width above nev + 4, then the
 * filter's tile of 64, 128 or 256 sites per CTA (start: opts->filter_tile, or
 * 128) with the other three at their best.
 * cache_path (may be NULL): a text file of earlier results, one line per
 * device and batch shape; a hit sets opts without timing anything, a new
 * result is appended. */
int laph_solver_autotune(const laph_problem* probs, int n, const double* const* links, int layout, int nsample,
                         laph_solve_opts* opts, const float* model, int nmodel, int device, const char* cache_path,
                         laph_tune_result* out);

/* ---- learned Chebyshev window --------------------------------------------
 * A 16 -> 64 -> 64 -> 3 tanh MLP (FP32) maps per-timeslice features -- the
 * smeared plaquette's mean, variance, skewness, excess kurtosis, the 10 Ritz
 * values of a 10-step Lanczos on -Delta (/12), log V3 / log 48^3, k / dim --
 * to (log lambda_cut, lambda_max, degree) of the first filter pass.  No
 * counterpart in the reference, whose window (LAM_L, LAM_C, DEG) is set by
 * hand in parameters.txt.  Parameter layout: W1[64][16] b1[64] W2[64][64]
 * b2[64] W3[3][64] b3[3]; a model is the parameters followed by feature
 * mean[16], std[16], target mean[3], std[3]. */
int laph_mlp_nparams(void);
int laph_mlp_forward(const float* params, const float* X, int n, float* out, int device);
/* Gradient (and loss) of the mean-squared loss over n samples at params. */
int laph_mlp_grad(const float* params, const float* X, const float* Y, int n, float* grad, float* loss, int device);
/* `epochs` full-batch Adam steps (beta 0.9 / 0.999), params updated in place. */
int laph_mlp_train(float* params, const float* X, const float* Y, int n, int epochs, float lr, float* loss,
                   int device);
/* Model used by window = LAPH_WINDOW_MLP (nfloats = nparams + 38). */
int laph_solver_set_window_model(laph_solver* s, const float* model, int nfloats);
/* Features (np x 16) and 10-step Lanczos upper bounds (np) of the last run. */
int laph_solver_features(laph_solver* s, float* feats, double* bound);
/* All k Ritz values of problem i after the last run (k returned). */
int laph_solver_ritz(laph_solver* s, int i, double* theta, int* k);

/* Smearing parameters of problem i (p1, p2 as in laph_solve_opts), replacing
 * the options' for that problem only: a batch of copies of one timeslice with
 * different parameters is the batched form of tune_hyp's (alpha_1, alpha_2)
 * scan (src/tune_hyp.cpp:116-255).  Kind and iterations stay global. */
int laph_solver_set_smear(laph_solver* s, int i, double p1, double p2);

/* ---- covariant displacement ---------------------------------------------
 * W_i(x) = 1/2 (U_dir(x) V_i(x+dir) - U_dir(x-dir)^dag V_i(x-dir)) for every
 * column of V (column-major complex128 [3 V3][nev], index 3 site + colour),
 * dir 0/1/2 = x/y/z: right_displacement_one_dir (modules/config_utils.cpp:
 * 344-382), FP64 on the device.  laph_displace uses a context's current
 * (smeared) links and host or device V/W (must not overlap); laph_solver_displace
 * displaces problem i's phase-fixed eigenvectors with its smeared links, in
 * place on the device, W to host or device memory. */
int laph_displace(laph_ctx* ctx, int dir, const double* V, double* W, int nev, int on_device);
int laph_solver_displace(laph_solver* s, int i, int dir, double* W, int on_device);

/* ---- source shape (the reference's sourceshape program) ------------------
 * psi(r) = sum_x || V_{x+r} V_x^dag ||_F over the grid r_i = 0, 2, ..., L-2,
 * V_y the 3 x nev block of rows 3y .. 3y+2 of the eigensystem: replaces
 * source_shape_complete / dll_op (modules/sourceshape_funcs.cpp:30-81).
 * psi[(L/2)^3] (host) in the reference's order (r1 = x outer, r3 = z inner).
 * FP64 on the device; even L only.  evals (may be NULL): weight column n by
 * sqrt|evals[n]| first (weight_eigenvectors, sourceshape_funcs.cpp:85-96).
 * laph_sourceshape takes a column-major complex128 eigensystem [3 V3][nev]
 * in host (on_device = 0) or device memory; laph_solver_sourceshape works on
 * problem i of a solver that has run, in place on the device (weighted != 0:
 * by sqrt of its eigenvalues).  The tile products run on the FP64 tensor path;
 * the environment variable LAPH_SOURCESHAPE_KERNEL=0, read once per process,
 * selects the FP64-FMA kernel instead (same results to rounding). */
int laph_sourceshape(const double* V, int L, int nev, const double* evals, int on_device, double* psi, int device);
int laph_solver_sourceshape(laph_solver* s, int i, int weighted, double* psi);
/* avg_radii (sourceshape_funcs.cpp:100-135): psi averaged over grid points of
 * equal |r| (to 1e-11), radii in order of first appearance; r_out / psi_out
 * hold up to (L/2)^3 entries, *n_out gets the count. */
int laph_sourceshape_avg(int L, const double* psi, double* r_out, double* psi_out, int* n_out);
/* write_sourceshape_ascii / _bin (modules/read_write.cpp:205-234):
 * "<dir>/sourceshape_nev<nev>.<config>.<t>" ("#r\tpsi(r)" then "r psi" with 12
 * significant digits) and "<dir>/sourceshape_nev<nev>.%04d.%03d.bin" ((r, psi)
 * double pairs); dir NULL or "" is the working directory, as in the reference. */
int laph_write_sourceshape(const char* dir, int config, int t, int nev, int n, const double* r, const double* psi);

/* ---- host-side utilities (no device needed) ------------------------------ */
/* Seeded synthetic gauge field U = exp(i eps H), H = sum_a c_a lambda_a with
 * c_a ~ N(0,1) i.i.d. (Gell-Mann basis), for all 4 directions; output in the
 * LAPH_LAYOUT_CONF order for nt timeslices: double[nt][V3][4][3][3][2]. */
int laph_gauge_random(double* conf, int L, int nt, double eps, uint64_t seed);
/* LIME/ILDG I/O.  The reader replaces read_lime_gauge_field_doubleprec_timeslices
 * (modules/io.cpp:22-146): conf gets timeslices [t_i, t_f] in the order above.
 * The writer emits ildg-format + ildg-binary-data records (big-endian FP64). */
int laph_lime_write_gauge(const char* path, const double* conf, int L, int T);
int laph_lime_read_gauge(const char* path, int T, int L, int t_i, int t_f, double* conf);
/* Beyond the reference, whose reader stops at single-precision files
 * (modules/io.cpp:72-79): laph_lime_read_gauge_any reads FP64 or FP32 ILDG
 * binary data (FP32 widened to FP64), telling them apart by the record size
 * and, when an ildg-format record precedes the data, checking its <precision>
 * (LAPH_ESIZE on a mismatch); *precision (may be NULL) receives 32 or 64.
 * laph_lime_info parses the ildg-format XML record (lx, ly, lz, lt,
 * precision) and checks it against the size of the binary record.
 * laph_lime_write_gauge_prec writes either precision (the plain writer is 64). */
int laph_lime_read_gauge_any(const char* path, int T, int L, int t_i, int t_f, double* conf, int* precision);
int laph_lime_info(const char* path, int* lx, int* ly, int* lz, int* lt, int* precision);
int laph_lime_write_gauge_prec(const char* path, const double* conf, int L, int T, int precision);
/* write_eig_sys_bin / write_eigenvalues_bin (modules/read_write.cpp:176-250):
 * "<dir>/<prefix>.%04d.%03d".  The eigenvector writer runs check_trace first
 * and returns LAPH_ETRACE (nothing written) where the reference exits. */
int laph_write_eigsys_bin(const char* dir, const char* prefix, int config, int t, int dim, int nev, const double* V);
int laph_write_eigenvalues_bin(const char* dir, const char* prefix, int config, int t, int nev, const double* ev);
int laph_read_eigsys_bin(const char* dir, const char* prefix, int config, int t, int dim, int nev, double* V);
int laph_read_eigenvalues_bin(const char* dir, const char* prefix, int config, int t, int nev, double* ev);
/* check_trace (read_write.cpp:20-35): 1 if |tr|-nev, |Im tr|, |sum|-nev, |Im sum| <= 1e-9. */
int laph_check_trace(int dim, int nev, const double* V, double* trace, double* sum);
/* fix_phase (modules/eigensystem.cpp:4-30) on host data. */
int laph_fix_phase_host(int dim, int nev, const double* V, double* Vfix, double* phase);
/* reset_phase (modules/eigensystem.cpp:32-57) on host data: column n of V
 * rotated so that its first entry has the phase phase_want[n] (the phases
 * file of an earlier run); Vreset may equal V. */
int laph_reset_phase_host(int dim, int nev, const double* V, const double* phase_want, double* Vreset);
/* read_eigenvalues_ascii (modules/read_write.cpp:99-115): "<prefix>.%03d.%04d"
 * (timeslice, then configuration), nev whitespace-separated values.  A missing
 * file is LAPH_EIO and a short one LAPH_ESIZE (the reference skips both
 * silently). */
int laph_read_eigenvalues_ascii(const char* prefix, int config, int t, int nev, double* ev);
/* write_gauge_matrices / read_gauge_matrices (modules/read_write.cpp:117-132,
 * 253-261): V3 raw 3x3 complex128 matrices in Eigen Matrix3cd memory order
 * (column-major), 144 bytes each, no header; a short file is LAPH_ESIZE. */
int laph_write_gauge_matrices(const char* path, int V3, const double* G);
int laph_read_gauge_matrices(const char* path, int V3, double* G);
/* recover_spectrum (modules/recover_spec.cpp:45-54). */
int laph_recover_spectrum(int nev, const double* theta, int deg, double lam_l, double lam_c, double* out);

/* Timeslice block of process `rank` among `size` (src/ev_ts.cpp:103-119):
 * contiguous blocks of LT/size, the first LT % size blocks one longer. */
int laph_timeslice_split(int LT, int size, int rank, int* t0, int* count);

/* parameters.txt (modules/par_io.cpp:8-136), same key/value rules. */
typedef struct {
  char config_path[512], result_path[512], in_path[512], phase_path[512];
  int LT, LX, NEV, iter, DEG, OMP_THRDS;
  double alpha_1, alpha_2, LAM_L, LAM_C;
  /* keys added by this library */
  int smear;            /* LAPH_SMEAR_* (key "smear" = hyp|stout|ape|none; default hyp) */
  double rho, alpha;    /* stout rho, APE alpha                                        */
  double tol;           /* residual target                                             */
  int guard, block, window, solver; /* solver: 0 = block (default), 1 = plain MatShell */
  int V3, MAT_ENTRIES, V_TS;
  double alpha_1_i, alpha_1_f, alpha_2_i, alpha_2_f; /* tune_hyp scan range (par_io.cpp:75-89) */
  int autotune;         /* > 0: laph_ev_ts tunes deg / block / guard on that many
                           timeslices first (laph_solver_autotune); 0: off      */
  int filter_deg;       /* block solver's filter degree cap (0: by lattice size) */
} laph_config;
int laph_parse_parameters(const char* path, laph_config* cfg);

#ifdef __cplusplus
}
#endif
#endif
