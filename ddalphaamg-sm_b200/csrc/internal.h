// Kernel launchers and level geometry shared by the library's translation units.
#pragma once

#include "common.cuh"

namespace ddamg {

// Geometry of one multigrid level (include/params.h:34-69 derives the same numbers).
struct Geom {
    int level = 0;
    int Nx = 0, Nt = 0, sites = 0;
    int colors = 1, dof = 2;         // dof = 2 * colors
    int ntest = 0;                   // test vectors = colours of level+1 (non-coarsest)
    int agg_x = 0, agg_t = 0;        // aggregation block counts
    int el_x = 0, el_t = 0;          // sites per aggregate and direction
    int sap_x = 0, sap_t = 0;        // SAP block counts
    int sel_x = 0, sel_t = 0;        // sites per SAP block and direction
    __host__ __device__ long size() const { return (long)sites * dof; }
};

// Coarse links live as [site][d][j][i]: 5 dof x dof matrices per site, column j (input dof)
// major and row i (output dof) fastest so a warp reads one column coalesced.
// d = 0 self (G1 = A), 1 = +t (G2, mu=0), 2 = +x (G2, mu=1), 3 = -t (G3, mu=0), 4 = -x (G3, mu=1).
// The level operator is out = (m0+2) v - sum_d s_d M_d v(nbr_d) with s_d the antiperiodic
// sign of hops that cross t = Nt-1 <-> 0.

// ------------------------------------------------------------ fine level (kernels_fine.cu)
template <typename V>
void launch_wilson(cudaStream_t s, const V* U, const V* in, V* out, const V* b, int Nx, int Nt, double m0,
                   int dagger, int nrhs);
// D_W kernel choice (process-wide): 0 default, 1 register kernels, 2 staged tiles (bulk copies into
// shared memory); the staged kernel's bounded-wait status word (1: a copy never arrived)
void set_stencil_variant(int v);
int stencil_variant();
int stencil_status_read();
void launch_link_derivative(cudaStream_t s, const double2* U, const double2* psi, const double2* lam, double* out,
                            int Nx, int Nt);
void launch_metropolis_init(cudaStream_t s, double* th, int Nx, int Nt, uint64_t seed);
void launch_metropolis_sub(cudaStream_t s, double* th, int Nx, int Nt, double beta, double delta, uint64_t seed,
                           int sweep, int sub, unsigned long long* acc);
void launch_theta_to_links(cudaStream_t s, const double* th, double2* U, long n);
void launch_fill_uniform(cudaStream_t s, double2* out, long n_complex, uint64_t seed, long offset_complex);
template <typename A, typename B> void launch_convert(cudaStream_t s, const A* in, B* out, long n);

// ------------------------------------------------------------ vector algebra (kernels_blas.cu)
// Reductions use a fixed grid and a second pass, so results are deterministic.
constexpr int kRedBlocks = 296;  // 2 x 148 SMs
// out[r*k + i] = sum_e w_r[e] * conj(B_r,i[e]) for i < k; basis vector i of rhs r at B + r*bstride + i*ldb
template <typename V>
void launch_multidot(cudaStream_t s, const V* B, long ldb, long bstride, int k, const V* w, long wstride, long n,
                     int nrhs, double2* partial, double2* out);
// out[r] = sum_e |x_r[e]|^2
template <typename V>
void launch_norm2(cudaStream_t s, const V* x, long xstride, long n, int nrhs, double2* partial, double* out);
// w_r -= sum_i coef[r*k+i] * B_r,i   (coef in FP64 on the device)
template <typename V>
void launch_multiaxpy(cudaStream_t s, const V* B, long ldb, long bstride, int k, const double2* coef, V* w,
                      long wstride, long n, int nrhs, double sign);
// y_r = alpha_r * x_r with alpha from the device
template <typename V>
void launch_scale(cudaStream_t s, const double2* alpha, const V* x, V* y, long n, int nrhs);
// r = a - b
template <typename V> void launch_sub(cudaStream_t s, const V* a, const V* b, V* r, long n);
// y += x
template <typename V> void launch_add(cudaStream_t s, const V* x, V* y, long n);
// SAP convergence flags: done[r] = it + 1 the first time sqrt(rr[r]) < tol * sqrt(vv[r])
void launch_flag_converged(cudaStream_t s, const double* rr, const double* vv, double tol, int nrhs, int it,
                           int* done);
// y = alpha x with alpha a host value
template <typename V> void launch_scale_host(cudaStream_t s, double2 alpha, const V* x, V* y, long n);
void launch_sigma3(cudaStream_t s, const double2* x, double2* y, long sites);
size_t sap_smem_bytes(int m, int NE, bool fp64);

// ------------------------------------------------------------ coarse levels (kernels_coarse.cu)
template <typename V>
void launch_coarse_op(cudaStream_t s, const V* links, const V* in, V* out, const V* b, int Nx, int Nt, int dof,
                      double m0, int nrhs);
// P^dagger: fine level g -> coarse; tv = [ntest][sites][dof]
template <typename V>
void launch_restrict(cudaStream_t s, const Geom& g, const V* tv, const V* in, V* out, int nrhs);
// P (add = 0: out = P vc, add = 1: out += P vc)
template <typename V>
void launch_prolong(cudaStream_t s, const Geom& g, const V* tv, const V* vc, V* out, int add, int nrhs);
void launch_orthonormalize(cudaStream_t s, const Geom& g, double2* tv);
// next-level links from level g's operator (U for level 0, links otherwise) and test vectors
void launch_build_coarse_links(cudaStream_t s, const Geom& g, const double2* U, const double2* links,
                               const double2* tv, double2* next_links);

// ------------------------------------------------------------ SAP (kernels_sap.cu)
// One colour sweep of SAP_C::SAP: x_B += D_B^-1 r_B for every block of the colour, block
// GMRES(m) x restarts to tol with x0 = r_B (src/sap.cpp:48-77).  blocks: device list.
constexpr int kSapMaxM = 8;  // block GMRES restart length supported by the SAP block solvers
struct SapArgs {
    int m, restarts;
    double tol;
    double m0;
    const int* blocks;  // block indices of this colour
    int nblocks;
    const int* done;    // per-rhs skip flags (may be null)
    const void* vres = nullptr;  // coarse sweeps of sap_block2_kernel: form r_B = v_B - (D x)_B from this v
};
template <typename V>
void launch_sap_sweep_fine(cudaStream_t s, const Geom& g, const V* U, const V* r, V* x, const SapArgs& a,
                           int nrhs);
// variant = rb * 4 + kernel: rb right-hand sides per CTA, kernel 0 the block solver with the
// single-thread Hessenberg update (sap_block_kernel), 1 the latency-trimmed block solver
// (sap_block2_kernel); 0 lets the launcher choose from the batch width and the block size
template <typename V>
void launch_sap_sweep_coarse(cudaStream_t s, const Geom& g, const V* links, const V* r, V* x, const SapArgs& a,
                             int nrhs, int variant = 0);
// the autotuner's candidate variants
constexpr int kSapVariantCount = 6;
constexpr int kSapVariants[kSapVariantCount] = {4 * 1 + 0, 4 * 1 + 1, 4 * 2 + 1, 4 * 4 + 0, 4 * 4 + 1, 4 * 8 + 0};
// autotuner of the variant: times one sweep per admissible candidate into the scratch field xs;
// us[kSapVariantCount]; returns the fastest variant
template <typename V>
int tune_sap_rb(cudaStream_t s, const Geom& g, const V* links, const V* r, V* xs, const SapArgs& a, int nrhs,
                double* us);

// ------------------------------------------------------------ tensor-core SAP (kernels_tcsap.cu)
// Batched FP32 coarse-level SAP colour sweep whose block operator runs on tcgen05 tensor cores
// (TF32 inputs, FP32 accumulation), with the per-(block, rhs) GMRES bookkeeping on CUDA cores.
// Block vectors are [kb][r][s][dof] (kb: block of the colour, r: rhs, s: site in the block).
struct TcSapWork {
    float2 *b = nullptr, *x = nullptr, *w = nullptr, *V = nullptr;  // V holds m+1 block vectors
    long vec = 0;                                                    // float2 per block vector
    int *act = nullptr, *fin = nullptr, *arn = nullptr, *maxit = nullptr;
    double *normb = nullptr, *err = nullptr;
    double2 *H = nullptr, *gm = nullptr, *cn = nullptr, *sn = nullptr;
    float* tiles = nullptr;  // operator tiles of the level, kTcTileFloats per (site, direction)
    int* status = nullptr;   // set when a bounded wait inside the apply kernel gave up
};
constexpr int kTcTileFloats = 64 * 64;
// the level's geometry admits the tensor-core sweep (dof <= 32, at most 1024 unknowns per block,
// and a block-vector window that fits in shared memory)
bool tc_sap_supported(const Geom& g);
void launch_pack_tc_links(cudaStream_t s, const Geom& g, const float2* links, float* tiles);
// shape: index of the apply kernel's tile shape (from tune_sap_tc; out of range: a default)
void launch_sap_sweep_tc(cudaStream_t s, const Geom& g, const TcSapWork& w, const float2* r, float2* x,
                         const SapArgs& a, int nrhs, int shape);
// autotuner: times each admissible tile shape on the sweep's data and returns the fastest;
// us[tc_sweep_shapes()] receives the times (negative: not admissible)
int tune_sap_tc(cudaStream_t s, const Geom& g, const TcSapWork& w, const float2* r, const SapArgs& a, int nrhs,
                double* us);
int tc_sweep_shapes();
// the level operator out = D_c in (or b - D_c in) for nrhs right-hand sides on tcgen05 tensor cores
// (TF32 inputs, FP32 accumulation), from the SAP sweeps' packed operator tiles; shape: 0..tc_op_shapes()-1
// (64, 32 or 16 right-hand sides per CTA)
bool tc_op_supported(const Geom& g);
int tc_op_shapes();
int tc_op_shape_rg(int shape);
void launch_coarse_op_tc(cudaStream_t s, const Geom& g, const float* tiles, const float2* in, float2* out,
                         const float2* b, double m0, int nrhs, int shape, int* status);
void tc_sweep_shape(int idx, int* rg, int* stages, int* chains);

// ------------------------------------------------------------ comparison solvers (kernels_krylov.cu)
// BiCGstab on D_W and CG on D^dagger D (src/conjugate_gradient.cpp) with device-resident scalars
struct KrylovState {
    double2 alpha, beta, omega, rho, rho_prev, rnorm2;
    double norm_b, err;
    int k, done, iters;  // done: 0 running, 1 BiCGstab converged with x += alpha d pending, 2 converged, 3 max_iter
    unsigned ticket;     // CTAs finished in the current kernel (the last one reduces)
};
struct KrylovWork {
    double2 *b = nullptr, *rt = nullptr, *x = nullptr, *r = nullptr, *s = nullptr, *t = nullptr, *y = nullptr;
    double2* d[2] = {nullptr, nullptr};
    double2* Ad[2] = {nullptr, nullptr};
    double2* part = nullptr;  // 3 partial sums per CTA
    KrylovState* st = nullptr;
};
int krylov_grid(int sites);
// solver 0 = BiCGstab (x holds x0 on entry), 1 = CG on D^dagger D x = b (x0 = b)
void launch_krylov_init(cudaStream_t s, int solver, const KrylovWork& w, const double2* U, int Nx, int Nt, double m0,
                        double tol, int max_iter);
void launch_krylov_iterations(cudaStream_t s, int solver, const KrylovWork& w, const double2* U, int Nx, int Nt,
                              double m0, double tol, int max_iter, int count);
// one-thread kernel for the body of a graph while node: condition = (the solve is still running)
void launch_krylov_continue(cudaStream_t s, cudaGraphConditionalHandle hc, const KrylovWork& w);

// ------------------------------------------------------------ HMC (kernels_hmc.cu)
void launch_gauge_force(cudaStream_t s, const double* th, double* F, int Nx, int Nt, double beta);
void launch_hmc_momentum(cudaStream_t s, double* p, const double* Fg, const double* Ff, double eps, long nlinks);
void launch_hmc_theta(cudaStream_t s, double* th, const double* p, double eps, long nlinks);

// ------------------------------------------------------------ device-driven FGMRES (kernels_fgmres.cu)
// Per-level state of one lockstep FGMRES (R right-hand sides, restart length m) whose Arnoldi
// bookkeeping runs on the device; loops are CUDA graph conditional nodes.
enum FgCtl {
    kFgJ = 0,            // Arnoldi step of the current restart
    kFgK = 1,            // restart
    kFgNan = 2,          // a NaN or Inf was met (reported by the host after the solve)
    kFgRunsOuter = 3,    // restart bodies run (cumulative)
    kFgRunsInner = 4,    // Arnoldi-step bodies run (cumulative; for K-cycles those of restart 0)
    kFgRunsFirst = 5,    // K-cycle restarts whose preconditioner starts from zero (restart 0)
    kFgRunsLater = 6,    // K-cycle restarts whose preconditioner starts from the previous Z_j
    kFgRunsInnerLater = 7,  // K-cycle Arnoldi-step bodies of restarts after the first
    kFgCtlWords = 8
};
struct FgDev {
    double2 *H = nullptr, *gm = nullptr, *cn = nullptr, *sn = nullptr;  // R x (m+1) x m, R x (m+1), R x m
    double2* coef = nullptr;   // R x m back-substitution result
    double2* alpha = nullptr;  // R scale factors of the next basis vector
    double2* dots = nullptr;   // 2 x R x (m+1): the two Gram-Schmidt passes of the current step
    double* nrm = nullptr;     // 2R squared norms
    double *norm_b = nullptr, *err = nullptr;
    int *maxIt = nullptr, *done = nullptr, *arn = nullptr, *ret = nullptr;
    int* ctl = nullptr;  // kFgCtlWords
};
void launch_fg_start(cudaStream_t s, const FgDev& f, int R, int m, int restarts, cudaGraphConditionalHandle hc);
// hc_sel (if select): condition of the if/else node that picks the restart-0 loop (k == 0) or the later one
void launch_fg_restart(cudaStream_t s, const FgDev& f, int R, int m, cudaGraphConditionalHandle hc0,
                       cudaGraphConditionalHandle hc1, cudaGraphConditionalHandle hc_sel, int select);
// counter: the FgCtl run counter of the body this step belongs to
void launch_fg_arnoldi(cudaStream_t s, const FgDev& f, int R, int m, double tol, cudaGraphConditionalHandle hc,
                       int counter);
void launch_fg_backsub(cudaStream_t s, const FgDev& f, int R, int m);
void launch_fg_restart_end(cudaStream_t s, const FgDev& f, int R, int m, int restarts, double tol,
                           cudaGraphConditionalHandle hc);
// multi-dot / multi-axpy over basis vectors 0..j with j = *jdev; results and coefficients at
// [r*ldk + i]; kmax bounds k = j + 1
template <typename V>
void launch_multidot_dev(cudaStream_t s, const V* B, long ldb, long bstride, int kmax, const int* jdev, int ldk,
                         const V* w, long wstride, long n, int nrhs, double2* partial, double2* out);
template <typename V>
void launch_multiaxpy_dev(cudaStream_t s, const V* B, long ldb, long bstride, const int* jdev, const double2* coef,
                          int ldk, V* w, long wstride, long n, int nrhs);
// Vb[j*slot + r*n + e] = alpha_r x[r*n + e]
template <typename V>
void launch_scale_slot(cudaStream_t s, const double2* alpha, const V* x, V* Vb, long slot, const int* jdev, long n,
                       int nrhs);
// to_slot = 0: dst[e] = src[j*slot + e]; 1: dst[j*slot + e] = src[e]
template <typename A, typename B>
void launch_slot_copy(cudaStream_t s, const A* src, B* dst, long slot, const int* jdev, int to_slot, long count);

// ------------------------------------------------------------ coarsest GMRES (kernels_gmres.cu)
struct CoarseGmresWork {
    double2* V = nullptr;      // (m+1) x n
    double2* w = nullptr;      // n
    double2* r = nullptr;      // n
    double2* partial = nullptr;  // grid x (m+2)
    double2* H = nullptr;      // (m+1) x m (column major, ld m+1)
    unsigned* bar = nullptr;   // barrier counter + generation
    int* status = nullptr;     // [0] error flag, [1] iterations
    int grid = 0;
    int block = 0;             // threads per CTA (set by coarse_gmres_prepare)
    int ncache = 0, nbs = 0;   // link matrices / basis slots of a CTA's sites in shared memory (coarse_gmres_prepare)
    long long spin_limit = 0;  // polls before a grid barrier gives up (<= 0: the default, 2^24)
};
void coarse_gmres_prepare(CoarseGmresWork& w, int n, int m, int dof, int device);
// the same solve on one thread-block cluster per right-hand side (kernels_gmres.cu)
struct CoarseClusterWork {
    int C = 0;             // CTAs per cluster (16 or 8)
    int clusters = 0;      // clusters of one launch (each loops over its share of the right-hand sides)
    size_t smem = 0;
    long wstride = 0;      // complex values of workspace per cluster: basis (m+1) n, w n, Hessenberg (m+1) m
    double2* ws = nullptr;
    int* status = nullptr;  // [1]: iterations
};
// false if the device cannot run the cluster kernel for this level (dof > 32, shared memory, cluster size)
bool coarse_cluster_prepare(CoarseClusterWork& w, int n, int m, int dof, int max_rhs);
void launch_coarse_gmres_cluster(cudaStream_t s, const CoarseClusterWork& w, const double2* links, const double2* b,
                                 double2* x, int R, int Nx, int Nt, int dof, double m0, int m, int restarts,
                                 double tol);
// x = GMRES(m) x restarts solution of D x = b from x0 = b; returns on the stream
void launch_coarse_gmres(cudaStream_t s, const CoarseGmresWork& w, const double2* links, const double2* b,
                         double2* x, int Nx, int Nt, int dof, double m0, int m, int restarts, double tol);

}  // namespace ddamg
