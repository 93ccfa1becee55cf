/*
 * ddamg_oracle — CPU restatement of the DD-alphaAMG solve for the 2D
 * Schwinger-model Wilson-Dirac operator (reference: JFNCastellanos/DDalphaAMG-SM).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
 * The library itself never calls into it.
 *
 * Pinning: every operation here is compared with the reference's own code
 * (compiled by oracle/Makefile `ref`, driven by oracle/ref_harness.cpp) through
 * the fixtures in tests/golden/ (generator: tests/golden/make_golden.py).
 *
 * Conventions (all follow the reference):
 *  - lattice Nx (x, slow) by Nt (t, fast); site = x*Nt + t; no halo;
 *  - mu = 0 is the t direction, mu = 1 the x direction (include/boundary.h:32-36);
 *  - fermion fields are periodic in x and antiperiodic in t (include/boundary.h:38-46);
 *  - a level-l vector is [site][c][alpha], dof = c*2 + alpha (src/level.cpp:403);
 *  - complex numbers are interleaved (re, im) doubles in every buffer.
 */
#ifndef DDAMG_ORACLE_H
#define DDAMG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_LEVELS 8

typedef struct orc_mg orc_mg;

/* solver constants, defaults from src/variables.cpp:100-134 */
typedef struct {
    int sap_gmres_m;          /* 5    SAPV::sap_gmres_restart_length */
    int sap_gmres_restarts;   /* 5    SAPV::sap_gmres_restarts */
    double sap_gmres_tol;     /* 1e-3 SAPV::sap_gmres_tolerance */
    int sap_tv_iters;         /* 4    AMGV::SAP_test_vectors_iterations */
    int coarse_m;             /* 400  AMGV::gmres_restart_length_coarse_level */
    int coarse_restarts;      /* 10   AMGV::gmres_restarts_coarse_level */
    double coarse_tol;        /* 0.1  AMGV::gmres_tol_coarse_level */
    int nu1, nu2;             /* 0, 2 */
    int kc_m, kc_restarts;    /* 5, 2 AMGV::fgmres_k_cycle_* */
    double kc_tol;            /* 0.1 */
    double smoother_tol;      /* 1e-10, the tol the cycles pass to SAP (src/amg.cpp:65) */
} orc_constants;

void orc_default_constants(orc_constants* c);

/* rows: (levels-1) x 6 ints, one parameters-file row each:
 * level block_x block_t ntest sap_block_x sap_block_t (include/params.h:34) */
orc_mg* orc_create(int levels, double m0, int Nx, int Nt, const int* rows, const double* U,
                   const orc_constants* c);
void orc_destroy(orc_mg* mg);
int orc_level_sites(const orc_mg* mg, int l);
int orc_level_dof(const orc_mg* mg, int l);
int orc_level_ntest(const orc_mg* mg, int l);

/* fine operators */
void orc_dirac(const orc_mg* mg, int dagger, const double* in, double* out);
/* generic level operator Level::D_operator */
void orc_level_op(const orc_mg* mg, int l, const double* in, double* out);
/* transfers */
void orc_restrict(const orc_mg* mg, int l, const double* in, double* out);
void orc_prolong(const orc_mg* mg, int l, const double* in, double* out);
/* setup pieces */
void orc_set_tvec(orc_mg* mg, int l, const double* tv);
void orc_get_tvec(const orc_mg* mg, int l, double* tv);
void orc_orthonormalize(orc_mg* mg, int l);
void orc_make_coarse_links(orc_mg* mg, int l);
/* which: 1 = G1 (A), 2 = G2 (B), 3 = G3 (C); reference layout per site */
void orc_get_links(const orc_mg* mg, int l, int which, double* out);
void orc_set_links(orc_mg* mg, int l, int which, const double* in);
/* rnd: every random vector the setup draws, in setUpPhase order */
int orc_setup(orc_mg* mg, const double* rnd, long n_rnd_complex);
long orc_setup_random_count(const orc_mg* mg);
/* solvers; each returns the reference's iteration count */
int orc_sap(const orc_mg* mg, int l, const double* v, double* x, int nu, double tol);
int orc_coarse_gmres(const orc_mg* mg, const double* b, double* x);
void orc_vcycle(const orc_mg* mg, const double* eta, double* psi);
void orc_kcycle(const orc_mg* mg, const double* eta, double* psi);
int orc_solve(const orc_mg* mg, int cycle, int m, int restarts, double tol, const double* b, double* x);
/* plain GMRES(m) on D_W with no preconditioner (FGMRES_fine_level, include/fgmres.h:153-236) */
int orc_gmres_plain(const orc_mg* mg, int m, int restarts, double tol, const double* b, double* x);

/* stand-alone multigrid, AlgebraicMG::applyMultilevel (src/amg.cpp:177-243): up to `it` cycles
 * (cycle 0 = V, 1 = K) on the iterate out (initial guess on entry) until the true residual is below
 * tol ||rhs||; returns the cycles run, *rel_residual the last relative residual */
int orc_apply_multilevel(const orc_mg* mg, int cycle, int it, double tol, const double* rhs, double* out,
                         double* rel_residual);
/* FGMRES_SAP (include/sap.h:236-333, Methods::FGMRES_sap src/methods.cpp:83-104): FGMRES(m) on D_W
 * from x0 = 0, preconditioned by one fine-level SAP iteration over sap_x x sap_t blocks (counts) */
int orc_fgmres_sap(const orc_mg* mg, int sap_x, int sap_t, int m, int restarts, double tol, const double* b,
                   double* x);
/* SAP_C::SAP with SAP_fine_level over sap_x x sap_t blocks (Methods::SAP, src/methods.cpp:60-80) */
int orc_sap_fine(const orc_mg* mg, int sap_x, int sap_t, const double* v, double* x, int nu, double tol);
/* D_phi / D_dagger_phi without a hierarchy: U [site][mu] */
void orc_dirac_plain(int Nx, int Nt, double m0, const double* U, int dagger, const double* in, double* out);

/* comparison solvers (src/conjugate_gradient.cpp): BiCGstab on D_W from x0, returning k+1 or
 * max_iter; CG on D^dagger D x = phi from x0 = phi, returning k+1 or 0 */
int orc_bicgstab(const orc_mg* mg, const double* phi, const double* x0, double* x, int max_iter, double tol);
int orc_cg_normal(const orc_mg* mg, const double* phi, double* x, int max_iter, double tol);

/* link derivative of L = Re(eta^dagger D^-1 b) given psi = D^-1 b and
 * lambda = D^-dagger eta; out[site*2+mu] = dL/dtheta_mu(site) */
void orc_link_gradient(const orc_mg* mg, const double* psi, const double* lambda, double* out);

/* ---------- inputs (no reference counterpart: the reference reads files) ---------- */
/* counter-based RNG: splitmix64 finaliser (Steele, Lea & Flood 2014) keyed by seed and stream */
uint64_t orc_rng(uint64_t seed, uint64_t stream, uint64_t counter);
/* U(1) Metropolis for S = beta * sum_P (1 - cos theta_P); hot start theta ~ U[-pi, pi).
 * theta: [site][mu]. returns the acceptance rate of the last sweep. */
double orc_metropolis(int Nx, int Nt, double beta, int sweeps, uint64_t seed, double delta, double* theta);
double orc_plaquette(int Nx, int Nt, const double* theta);
/* complex Gaussian, E|z|^2 = 1 (re, im ~ N(0, 1/2)) */
void orc_gaussian(long n, uint64_t seed, double* out);
/* complex with re, im ~ U(-1, 1) (the test-vector distribution of src/amg.cpp:7) */
void orc_uniform(long n, uint64_t seed, double* out);
/* reference binary record format (src/io.cpp:32-44) */
int orc_write_binary(const char* path, int Nx, int Nt, const double* field);
int orc_read_binary(const char* path, int Nx, int Nt, double* field);

#ifdef __cplusplus
}
#endif
#endif
