/*
 * ddamg.h — C ABI of the B200-native DD-alphaAMG solver for the 2D Schwinger-model
 * Wilson-Dirac operator.  Drop-in for the solve path of the reference
 * (JFNCastellanos/DDalphaAMG-SM); each entry point names the reference interface it
 * replaces.
 *
 * Conventions (identical to the reference):
 *   - lattice Nx (x, slow) by Nt (t, fast); site = x*Nt + t; no halo;
 *   - mu = 0 is the t direction, mu = 1 the x direction (include/boundary.h:32-36);
 *   - fermions periodic in x, antiperiodic in t; links periodic (include/boundary.h:38-46);
 *   - a level-l vector is [site][c][alpha] with dof = c*2 + alpha (src/level.cpp:403);
 *   - every complex number is two doubles (re, im), interleaved; a field of n complex
 *     numbers is a double[2n];
 *   - several right-hand sides are stored one after another: [rhs][site][dof].
 *
 * Host pointers are caller-owned and may be pageable; *_device variants take device
 * pointers on the handle's device.  One handle owns its device memory and one CUDA stream
 * and is not thread-safe; different handles are independent.  Every call returns a
 * ddamg_status; ddamg_last_error() describes the last failure on the calling thread.
 */
#ifndef DDAMG_H
#define DDAMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DDAMG_MAX_LEVELS 6

typedef enum {
    DDAMG_OK = 0,
    DDAMG_ERR_BAD_PARAM = 1,      /* reference: exit(1)/MPI_Abort on bad input (include/params.h:22-25,101-104) */
    DDAMG_ERR_IO = 2,             /* reference: exit(1) in read_binary / readParameters (src/io.cpp:7-10) */
    DDAMG_NOT_CONVERGED = 3,      /* reference: only the returned count restarts*m (src/fgmres.cpp:93-96) */
    DDAMG_ERR_NAN = 4,            /* NaN/Inf found in an input or a residual */
    DDAMG_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait (grid barrier) gave up */
    DDAMG_ERR_CUDA = 6,           /* a CUDA runtime error */
    DDAMG_ERR_STATE = 7           /* call out of order (e.g. solve before setup) */
} ddamg_status;

typedef enum { DDAMG_PREC_DOUBLE = 0, DDAMG_PREC_MIXED = 1 } ddamg_precision;
typedef enum { DDAMG_CYCLE_V = 0, DDAMG_CYCLE_K = 1 } ddamg_cycle;

/* Solver parameters.  Geometry comes from the parameters file (include/params.h:18-111),
 * the constants from the reference's globals (src/variables.cpp:100-134); defaults are
 * the reference's values. */
typedef struct {
    int Nx, Nt;          /* lattice (reference: compile-time NS, NT from config.h) */
    int levels;          /* reference: stdin "Levels" (src/main.cpp:33-46) */
    double m0;           /* bare mass (mass::m0) */
    /* parameters-file rows: level block_x block_t ntest sap_block_x sap_block_t;
     * block_* and sap_block_* are block COUNTS (include/params.h:7-16) */
    int rows[DDAMG_MAX_LEVELS - 1][6];
    int sap_gmres_restart_length;     /* 5    SAPV::sap_gmres_restart_length */
    int sap_gmres_restarts;           /* 5    SAPV::sap_gmres_restarts */
    double sap_gmres_tolerance;       /* 1e-3 SAPV::sap_gmres_tolerance */
    int sap_test_vectors_iterations;  /* 4    AMGV::SAP_test_vectors_iterations */
    int coarse_gmres_restart_length;  /* 400  AMGV::gmres_restart_length_coarse_level */
    int coarse_gmres_restarts;        /* 10   AMGV::gmres_restarts_coarse_level */
    double coarse_gmres_tolerance;    /* 0.1  AMGV::gmres_tol_coarse_level */
    int nu1, nu2;                     /* 0, 2 AMGV::nu1, AMGV::nu2 */
    int kcycle_restart_length;        /* 5    AMGV::fgmres_k_cycle_restart_length */
    int kcycle_restarts;              /* 2    AMGV::fgmres_k_cycle_restarts */
    double kcycle_tolerance;          /* 0.1  AMGV::fgmres_k_cycle_tol */
    int fgmres_restart_length;        /* 20   FGMRESV::fgmres_restart_length */
    int fgmres_restarts;              /* 50   FGMRESV::fgmres_restarts */
    double fgmres_tolerance;          /* 1e-10 FGMRESV::fgmres_tolerance */
    double smoother_tolerance;        /* 1e-10, the tol the cycles pass to SAP (src/amg.cpp:65) */
    int cycle;                        /* ddamg_cycle; reference: AMGV::cycle */
    int precision;                    /* ddamg_precision; the reference is FP64 only */
    int max_rhs;                      /* right-hand sides one ddamg_solve call may carry (>= 1) */
    int device;                       /* CUDA device ordinal */
    /* 1 (default): in mixed precision, coarse-level SAP sweeps over >= 8 right-hand sides run
     * the block operator on tcgen05 tensor cores (TF32 inputs, FP32 accumulation), and the batched
     * level operator D_c (the residuals of the cycles, the K-cycle's inner FGMRES) runs on them where the
     * autotuner measures them faster than the CUDA-core kernel; 2: the level operator always on tensor
     * cores where the level admits them; 0: CUDA cores only.  No reference counterpart. */
    int tensor_cores;
    /* 1 (default): solves run from CUDA graphs.  The first solve of a batch width runs host driven
     * (it tunes the kernels and captures the V-cycle preconditioner into a graph that it replays);
     * from the second on, the whole solve is one graph whose conditional nodes carry the FGMRES loops
     * (the outer one and, for K-cycles, the inner FGMRES of every coarse level), with the Hessenberg
     * and Givens work in device kernels, so no Arnoldi step waits for the host.  0: kernels are
     * launched one by one from the host loop.  Off while per-kernel timing (ddamg_profile) is on.
     * No reference counterpart. */
    int cuda_graphs;
    /* polls (each an L2 read and a 32 ns sleep) after which a grid barrier of the coarsest-level GMRES kernel gives up
     * and the solve returns DDAMG_ERR_DEVICE_TIMEOUT; default 2^24 (a few seconds); <= 0 also means the
     * default.  The reference's MPI collectives wait without a bound. */
    int coarse_barrier_polls;
    /* the coarsest-level GMRES kernel: 0 (default) chosen per handle at the end of its first setup by
     * timing both on one right-hand side; 1 the cooperative-grid kernel (about two coarse sites per CTA,
     * bounded grid barriers); 2 the thread-block-cluster kernel (one cluster of 16 CTAs per right-hand
     * side, hardware cluster barriers, distributed shared memory; the cooperative kernel where the device
     * or the level does not admit it).  No reference counterpart. */
    int coarse_kernel;
} ddamg_params;

typedef struct {
    int iterations;        /* outer FGMRES iterations, as FGMRES::fgmres returns (src/fgmres.cpp:89,96) */
    int converged;         /* 1 if the true residual met the tolerance */
    double rel_residual;   /* ||b - D x|| / ||b|| with the FP64 operator */
    double setup_seconds;  /* device time of the last setup */
    double solve_seconds;  /* device time of this solve */
} ddamg_solve_info;

typedef struct ddamg_handle ddamg_t;

/* ------------------------------------------------------------------ configuration */
/* fills the reference defaults (src/variables.cpp:100-134); geometry zeroed */
ddamg_status ddamg_params_default(ddamg_params* p);
/* readParameters (include/params.h:18-111): one row per non-coarsest level; the number
 * of rows must equal levels-1 (include/params.h:101-104) */
ddamg_status ddamg_parse_params_file(const char* path, int levels, ddamg_params* p);
/* Level / AlgebraicMG construction (include/level.h:147-233, include/amg.h:96-114):
 * validates the geometry and allocates every level's device storage */
ddamg_status ddamg_create(const ddamg_params* p, ddamg_t** h);
ddamg_status ddamg_destroy(ddamg_t* h);
const char* ddamg_last_error(void);
/* the cudaStream_t the handle launches on (as void*) */
ddamg_status ddamg_get_stream(ddamg_t* h, void** stream);
/* number of kernels the library has launched so far (all handles) */
ddamg_status ddamg_launch_count(ddamg_t* h, long long* count);
/* per-kernel device timing: while enabled, the handle brackets every SAP sweep, coarsest solve
 * and level-operator launch with CUDA events on its stream; disabling folds the elapsed times
 * into per (kind, level) totals.  kind: 0 SAP colour sweep, 1 coarsest GMRES, 2 level operator,
 * 3 orthonormalisation of the test vectors, 4 coarse-link construction (the last two: setup).
 * (No reference counterpart: the reference counts FLOPs, include/utils.h:141-150.) */
ddamg_status ddamg_profile(ddamg_t* h, int enable);
ddamg_status ddamg_profile_query(ddamg_t* h, int kind, int level, double* total_ms, long long* launches);
/* the autotuner's record: for each (level, batch width) whose SAP sweeps ran on the tensor cores,
 * the measured time of one block-operator application per candidate tile shape (right-hand sides
 * per CTA, link-tile pipeline depth, independent accumulator chains) and the chosen one (*), and
 * one line per captured V-cycle graph with its kernel count; NUL-terminated text, truncated to
 * len - 1 characters.  No reference counterpart. */
ddamg_status ddamg_autotune_report(ddamg_t* h, char* buf, int len);

/* ------------------------------------------------------------------ I/O */
/* read_binary (src/io.cpp:4-55): records int32 x, t, mu, f64 re, im, x slowest; out: [site][mu] */
ddamg_status ddamg_read_binary(const char* path, int Nx, int Nt, double* out);
/* writer of the same format (the reference has none; its inputs come from HMC) */
ddamg_status ddamg_write_binary(const char* path, int Nx, int Nt, const double* field);
/* layout converters for callers holding the reference's spinors (struct spinor, include/variables.h:201-238,
 * indexed by idx, include/utils.h:46-52): halo[(x*(Nt+2)+t)*dof + d] for x in 1..Nx, t in 1..Nt
 * <-> compact[((x-1)*Nt + (t-1))*dof + d], complex interleaved; to_halo zeroes the halo sites */
ddamg_status ddamg_from_halo(const double* halo, int Nx, int Nt, int dof, double* compact);
ddamg_status ddamg_to_halo(const double* compact, int Nx, int Nt, int dof, double* halo);
/* gauge links U_mu(x) (spinor U of src/main.cpp:74-78), [site][mu] complex */
ddamg_status ddamg_load_gauge(ddamg_t* h, const double* U);

/* ------------------------------------------------------------------ operators */
/* D_phi / D_dagger_phi (src/dirac_operator.cpp:24-85); nrhs fields back to back */
ddamg_status ddamg_apply_dirac(ddamg_t* h, int dagger, const double* in, double* out, int nrhs);
ddamg_status ddamg_apply_dirac_device(ddamg_t* h, int dagger, const void* in, void* out, int nrhs);
/* the same stencil in FP32 on device buffers of float pairs (mixed-precision smoother operator) */
ddamg_status ddamg_apply_dirac_f32_device(ddamg_t* h, int dagger, const void* in, void* out, int nrhs);
/* Level::D_operator (src/level.cpp:394-426) at level l >= 0, FP64 */
ddamg_status ddamg_apply_level_op(ddamg_t* h, int level, const double* in, double* out);
/* the same on nrhs right-hand sides in device memory ([rhs][site][dof], complex), on the handle's
 * stream: fp32 = 0 the FP64 operator (double2 data), fp32 = 1 the working-precision FP32 operator of a
 * mixed-precision handle (float2 data; with tensor_cores and nrhs >= 8 the batched tensor-core kernel
 * where the autotuner measured it faster, TF32 inputs with FP32 accumulation).  Level::D_operator
 * (src/level.cpp:394-426) for a batch. */
ddamg_status ddamg_apply_level_op_device(ddamg_t* h, int level, int fp32, const void* in, void* out, int nrhs);
/* Level::Pdagg_v (src/level.cpp:145-189): level l -> l+1 */
ddamg_status ddamg_restrict(ddamg_t* h, int level, const double* in, double* out);
/* Level::P_vc (src/level.cpp:92-141): level l+1 -> l */
ddamg_status ddamg_prolong(ddamg_t* h, int level, const double* in, double* out);
/* SAP_C::SAP (src/sap.cpp:81-165) at level l: x is the initial guess on entry and the
 * result on exit; *iters gets SAP's return value */
ddamg_status ddamg_sap(ddamg_t* h, int level, const double* v, double* x, int nu, double tol, int* iters);
/* SAP_C::SAP (src/sap.cpp:81-165) on nrhs vectors at once ([rhs][site][dof]), in the level's
 * working precision (FP32 in mixed precision below the coarsest level, where batches of >= 8
 * right-hand sides of a coarse level use the tensor-core block operator); x: initial guesses in,
 * results out.  nrhs <= max(max_rhs, test vectors of any level). */
ddamg_status ddamg_sap_batched(ddamg_t* h, int level, const double* v, double* x, int nrhs, int nu, double tol);

/* ------------------------------------------------------------------ setup */
/* AlgebraicMG::setUpPhase (src/amg.cpp:4-62) with test vectors drawn on the device from a
 * counter-based generator (splitmix64) seeded by `seed`: re, im ~ U(-1, 1) as in src/amg.cpp:7 */
ddamg_status ddamg_setup(ddamg_t* h, uint64_t seed);
/* the same with every random vector supplied, in the order setUpPhase draws them
 * (src/amg.cpp:12-41): level-0 vectors, then the extra vectors of each level >= 1 */
ddamg_status ddamg_setup_with_vectors(ddamg_t* h, const double* rnd, int64_t n_complex);
/* number of complex values ddamg_setup_with_vectors consumes */
ddamg_status ddamg_setup_random_count(ddamg_t* h, int64_t* n_complex);
/* Level::tvec access (include/level.h:251): [ntest][site][dof] */
ddamg_status ddamg_get_test_vectors(ddamg_t* h, int level, double* out);
ddamg_status ddamg_set_test_vectors(ddamg_t* h, int level, const double* in);
/* Level::orthonormalize (src/level.cpp:193-284) */
ddamg_status ddamg_orthonormalize(ddamg_t* h, int level);
/* Level::makeCoarseLinks (src/level.cpp:431-542): builds level+1's operator */
ddamg_status ddamg_build_coarse_links(ddamg_t* h, int level);
/* coarse links of level l >= 1 in the reference layout (include/level.h:349-365):
 * which = 1: G1[site][alf][bet][c][b]; 2: G2 and 3: G3 [site][alf][bet][c][b][mu] */
ddamg_status ddamg_get_coarse_links(ddamg_t* h, int level, int which, double* out);

/* ------------------------------------------------------------------ solvers */
/* coarsest solve Level::GMRES_level_l (include/level.h:70-140), x0 = b (src/amg.cpp:69) */
ddamg_status ddamg_coarse_solve(ddamg_t* h, const double* b, double* x, int* iters);
/* No counterpart in the reference.  The coarsest solve above without any device allocation, for
 * callers that cannot allocate device memory while they solve (a host framework that hands out all
 * device memory from its own pool, or a time-critical loop that cannot absorb the device
 * synchronisation of cudaMalloc / cudaFree).  The caller passes device pointers: links in the
 * library's coarse layout [site][d][j][i] (d = self, +t, +x, -t, -x; j input dof, i output dof,
 * 5*dof*dof complex per site), b and x (sites*dof complex); stream may be 0.  Scratch comes from
 * one fixed 32 MiB array of complex doubles compiled into the library: the solve must fit in
 * (m+2)*n + (m+1)*m + 3*G*(m+2) + 2 <= 2097152 complex values (n = Nx*Nt*dof, G = min(SMs,
 * (sites+1)/2)) or the call returns DDAMG_ERR_BAD_PARAM; e.g. m = 400 with G = 148 allows n up to
 * about 4,370.  The array is device memory of every GPU that runs this code, held until the process
 * exits.  The first call on a device looks the array's address up (cudaGetSymbolAddress) with that
 * device current.  All calls share the one array and it keeps the last call's contents (its barrier
 * and status words are cleared at each call): calls that overlap on the GPU, on any stream, race and
 * give wrong results.  The call synchronizes its stream before it returns (it reads the solve's
 * status words), so it must not be made while that stream is being captured into a graph;
 * *iterations gets the GMRES iteration count. */
ddamg_status ddamg_coarse_gmres_noalloc(const void* links, const void* b, void* x, int Nx, int Nt, int dof,
                                        double m0, int m, int restarts, double tol, void* stream,
                                        int* iterations);
/* changes coarse_barrier_polls of a live handle (launches made after the call use it; V-cycle graphs
 * captured earlier are dropped and captured again).  No reference counterpart. */
ddamg_status ddamg_set_coarse_barrier_polls(ddamg_t* h, int polls);
/* Which D_W kernel the library uses, process-wide (no reference counterpart): 0 the default, 1 the
 * register kernels (one or two sites per thread, neighbours through L1/L2), 2 the staged-tile kernel
 * (persistent CTAs; bulk asynchronous copies bring 8 x 64-site tiles of psi with their halo and the
 * links into shared memory, two stages deep), used where the lattice divides into its tiles. */
ddamg_status ddamg_set_stencil_kernel(int kind);
ddamg_status ddamg_get_stencil_kernel(int* kind);

/* ------------------------------------------------------------------ run metadata */
/* Iteration counters of the last run of each method, in the order the metadata file lists them;
 * -1 for a method not run on the handle (src/variables.cpp:9-17). */
typedef enum {
    DDAMG_COUNT_CG = 0,         /* ddamg_cg_normal        (iter_counters::CGIt, Methods::CG) */
    DDAMG_COUNT_BICG = 1,       /* ddamg_bicgstab         (iter_counters::BiCGIt) */
    DDAMG_COUNT_GMRES = 2,      /* ddamg_gmres_plain      (iter_counters::GMRESIt) */
    DDAMG_COUNT_SAP = 3,        /* ddamg_sap_fine         (iter_counters::SAPIt) */
    DDAMG_COUNT_FGMRES_SAP = 4, /* ddamg_fgmres_sap       (iter_counters::FGMRES_SAPIt) */
    DDAMG_COUNT_VCYCLE = 5,     /* ddamg_solve, V-cycle   (iter_counters::vCycleIt; most iterations over the batch) */
    DDAMG_COUNT_KCYCLE = 6,     /* ddamg_solve, K-cycle   (iter_counters::kCycleIt) */
    DDAMG_COUNT_KINDS = 7
} ddamg_counter;
ddamg_status ddamg_get_counters(ddamg_t* h, long long counts[DDAMG_COUNT_KINDS]);
/* writeMetadata (src/io.cpp:72-145): the run metadata file, line for line in the reference's format
 * (host, date, rank grid 1 x 1, m0, tolerance, one row per non-coarsest level, the solver constants and
 * the iteration counters of the handle).  The reference's FLOP counters are not kept: every FLOPS
 * column holds -1, the reference's value for a method that did not run.  path NULL: the reference's
 * file name metadata_<Nx>x<Nt>_Levels<L>_{V,K}cycle.dat in the working directory.  The Host line is
 * $HOSTNAME, else gethostname(). */
ddamg_status ddamg_write_metadata(ddamg_t* h, const char* path, int cycle, double tol);
/* the same from parameters and counters alone (no handle, no device) */
ddamg_status ddamg_write_metadata_params(const ddamg_params* p, const long long counts[DDAMG_COUNT_KINDS], int cycle,
                                         double tol, const char* path);
/* one cycle from psi = 0: AlgebraicMG::v_cycle / k_cycle (src/amg.cpp:64-174) */
ddamg_status ddamg_vcycle(ddamg_t* h, const double* eta, double* psi);
ddamg_status ddamg_kcycle(ddamg_t* h, const double* eta, double* psi);
/* stand-alone multigrid, AlgebraicMG::applyMultilevel (src/amg.cpp:177-243) as Methods::Vcycle /
 * Kcycle drive it (src/methods.cpp:106-127): up to max_cycles cycles of the handle's kind (V or K) on
 * the iterate x (initial guess in, result out), each followed by the true residual with the FP64
 * operator, until ||rhs - D x|| < tol ||rhs||.  In FP64 each cycle acts on x itself as the reference's
 * does; in mixed precision each cycle runs on the FP64 residual from zero and its result is added to x.
 * *cycles gets the cycles run (the reference only prints it), *rel_residual the last relative residual
 * (either may be NULL); DDAMG_NOT_CONVERGED if max_cycles were not enough.  A zero rhs gives x = 0 after
 * 0 cycles (the reference would iterate max_cycles times). */
ddamg_status ddamg_apply_multilevel(ddamg_t* h, const double* rhs, double* x, int max_cycles, double tol,
                                    int* cycles, double* rel_residual);
/* FGMRES_AMG_v_cycle / _k_cycle::fgmres (include/amg.h:147-270, src/fgmres.cpp:5-97) from
 * x0 = 0 for nrhs right-hand sides; info may be NULL or point to nrhs entries */
ddamg_status ddamg_solve(ddamg_t* h, const double* b, double* x, int nrhs, ddamg_solve_info* info);
ddamg_status ddamg_solve_device(ddamg_t* h, const void* b, void* x, int nrhs, ddamg_solve_info* info);
/* FGMRES_fine_level (include/fgmres.h:153-236): unpreconditioned GMRES(m) on D_W */
ddamg_status ddamg_gmres_plain(ddamg_t* h, const double* b, double* x, int m, int restarts, double tol,
                               ddamg_solve_info* info);
/* FGMRES_SAP (include/sap.h:236-333) as Methods::FGMRES_sap runs it (src/methods.cpp:83-104): FGMRES(m) x
 * restarts on D_W from x0 = 0 to tol, preconditioned by one fine-level SAP iteration from zero over
 * sap_x x sap_t Schwarz blocks (block COUNTS; the reference fixes 4 x 4, SAPV::sap_block_x/t,
 * include/variables.h:131-132), each block solved by GMRES(sap_gmres_restart_length) x
 * sap_gmres_restarts to sap_gmres_tolerance.  The blocks must divide the lattice, their number must be
 * even (or 1), and a block may hold at most 256 sites, or more if its Krylov basis fits in one CTA's
 * shared memory (about 1000 sites at restart length 5).  The SAP runs in the handle's level-0
 * precision (FP32 in mixed mode), the outer FGMRES in FP64.  info may be NULL. */
ddamg_status ddamg_fgmres_sap(ddamg_t* h, const double* b, double* x, int sap_x, int sap_t, int m, int restarts,
                              double tol, ddamg_solve_info* info);
/* SAP_C::SAP of SAP_fine_level (src/sap.cpp:81-165) over sap_x x sap_t fine-level blocks, as Methods::SAP
 * runs it (src/methods.cpp:60-80): x is the initial guess on entry and the result on exit; FP64;
 * *iters gets SAP's return value (same block limits as ddamg_fgmres_sap) */
ddamg_status ddamg_sap_fine(ddamg_t* h, const double* v, double* x, int sap_x, int sap_t, int nu, double tol,
                            int* iters);

/* bi_cgstab (src/conjugate_gradient.cpp:87-176, driven as Methods::BiCG, src/methods.cpp:3-19):
 * BiCGstab on D_W from x0 (NULL: zero) until ||s|| < tol ||b||; info->iterations is the
 * reference's return value (k+1, or max_iter without convergence -> DDAMG_NOT_CONVERGED) */
ddamg_status ddamg_bicgstab(ddamg_t* h, const double* b, const double* x0, double* x, int max_iter, double tol,
                            ddamg_solve_info* info);
/* conjugate_gradient (src/conjugate_gradient.cpp:4-83): CG on D^dagger D x = phi (the operator of
 * D_D_dagger_phi, src/dirac_operator.cpp:88-92) from x0 = phi until ||r|| < tol ||phi||.
 * Methods::CG (src/methods.cpp:42-58) calls it with phi = D^dagger b; info->rel_residual is
 * ||phi - D^dagger D x|| / ||phi||; info->iterations is k+1 at convergence, max_iter without it
 * (the reference returns 0 there), with DDAMG_NOT_CONVERGED */
ddamg_status ddamg_cg_normal(ddamg_t* h, const double* phi, double* x, int max_iter, double tol,
                             ddamg_solve_info* info);

/* ------------------------------------------------------------------ gradient (no reference counterpart) */
/* L = Re(eta^dagger D^-1 b): solves D psi = b and D^dagger lambda = eta through the same
 * multigrid (D^dagger = sigma_3 D sigma_3) and forms dL/dtheta_mu(x) = out[site*2 + mu] */
ddamg_status ddamg_gradient(ddamg_t* h, const double* eta, const double* b, double* dL_dtheta,
                            ddamg_solve_info* info);
/* the link-derivative kernel alone, given psi = D^-1 b and lambda = D^-dagger eta */
ddamg_status ddamg_link_derivative(ddamg_t* h, const double* psi, const double* lambda, double* dL_dtheta);

/* ------------------------------------------------------------------ HMC (no reference counterpart: the
 * reference reads HMC configurations generated elsewhere) */
typedef struct {
    int accepted;         /* the trajectory's end point was accepted */
    double dH;            /* H(end) - H(start) */
    double plaquette;     /* mean cos(theta_P) of the returned field */
    int cg_iterations;    /* CG iterations over all force evaluations and the final action */
    double seconds;       /* wall time of the trajectory */
} ddamg_hmc_info;
/* one HMC trajectory of the two-flavour Schwinger model, S = beta sum_P (1 - cos theta_P) +
 * phi^dagger (D^dagger D)^-1 phi with phi = D^dagger eta: Gaussian momenta and eta from seed, leapfrog
 * with md_steps steps of tau / md_steps, forces from the gauge plaquettes and the link derivative of
 * the CG solution (ddamg_cg_normal to cg_tol), Metropolis accept/reject.  theta: [site][mu] in/out
 * (unchanged when rejected or on an error); the handle's gauge field becomes the returned one and its
 * multigrid setup must be redone before the next solve. */
ddamg_status ddamg_hmc_trajectory(ddamg_t* h, double* theta, double beta, int md_steps, double tau, uint64_t seed,
                                  double cg_tol, ddamg_hmc_info* info);
/* dS/dtheta_mu(x) of that action at theta for a given phi: force[site*2 + mu] (the integrator's force).
 * The handle's gauge field and multigrid setup are the same afterwards as before, on success and on
 * error; DDAMG_NOT_CONVERGED if the CG solve misses cg_tol within 100000 iterations. */
ddamg_status ddamg_hmc_force(ddamg_t* h, const double* theta, const double* phi, double beta, double cg_tol,
                             double* force);

/* ------------------------------------------------------------------ inputs (no reference counterpart) */
/* U(1) Metropolis of S = beta sum_P (1 - cos theta_P), hot start theta ~ U[-pi, pi), on the
 * device; theta: [site][mu]; *acceptance: acceptance rate of the last sweep (may be NULL) */
ddamg_status ddamg_gauge_metropolis(int Nx, int Nt, double beta, int sweeps, uint64_t seed, double delta,
                                    double* theta, double* acceptance, int device);
/* complex Gaussian right-hand sides, E|z|^2 = 1 */
ddamg_status ddamg_gaussian_field(int64_t n_complex, uint64_t seed, double* out);

#ifdef __cplusplus
}
#endif
#endif
