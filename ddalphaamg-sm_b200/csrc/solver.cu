// Host side of the library: the multigrid hierarchy (Level / AlgebraicMG of the reference),
// the SAP driver, V- and K-cycles, FGMRES, the adaptive setup, and the extern "C" API.
// All device work is issued on the handle's stream; data-dependent branches that would
// otherwise need a host round trip (SAP early exit) are device-side flags.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iomanip>
#include <map>
#include <set>
#include <memory>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include <unistd.h>

#include "internal.h"

namespace ddamg {

std::atomic<long long> g_launches{0};
static thread_local std::string t_last_error;
void set_error(const std::string& msg) { t_last_error = msg; }

template <typename V> struct LevelBufs {
    V* U = nullptr;      // level 0 links [site][mu]
    V* links = nullptr;  // level >= 1: [site][5][dof][dof]
    V* tv = nullptr;     // [ntest][size]
    V* eta = nullptr;    // cycle input  (W x size)
    V* psi = nullptr;    // cycle output (W x size)
    V* xfer = nullptr;   // transfer buffer in the previous level's precision... (W x size)
    V* r = nullptr;      // SAP / cycle residual (W x size)
    V* t = nullptr;      // D x temporary (W x size)
    // K-cycle FGMRES workspace (level >= 1)
    V* kV = nullptr;
    V* kZ = nullptr;
    V* kw = nullptr;
    V* kr = nullptr;
    // fixed copies of the current basis vector and preconditioned vector (device-driven FGMRES)
    V* kin = nullptr;
    V* kzf = nullptr;
};

struct LevelData {
    Geom g;
    bool fp32 = false;  // working precision of this level's smoother / operator
    LevelBufs<double2> d;
    LevelBufs<float2> f;
    int* red = nullptr;
    int* black = nullptr;
    int nred = 0, nblack = 0;
    int* done = nullptr;    // W flags
    double* vv = nullptr;   // W norms
    double* rr = nullptr;   // W norms
    bool tc = false;        // batched FP32 SAP sweeps of this level use the tensor-core block operator
    TcSapWork tcw;
    std::map<int, int> tc_shape;  // batch width -> tile shape chosen by the autotuner
    std::map<int, int> rb_choice; // 2 * batch width + fp32 -> right-hand sides per CTA (CUDA cores)
    std::map<int, int> tc_op;     // batch width -> level-operator kernel: -1 CUDA cores, else tensor-core shape
    FgDev fg;                     // device-driven FGMRES state (level 0: the outer solve; >= 1: K-cycle)
};
constexpr int kTcMinRhs = 8;  // fewer right-hand sides leave too little link reuse for the tensor cores
// A Schwarz-block layout of the fine level other than the parameters file's: the block counts of
// SAP_fine_level as FGMRES_SAP and Methods::SAP build it (include/sap.h:185-233), with its red and
// black block lists on the device
struct SapLayout {
    Geom g;
    int* red = nullptr;
    int* black = nullptr;
    int nred = 0, nblack = 0;
};
template <typename V> LevelBufs<V>& B(LevelData& L);
template <> LevelBufs<double2>& B<double2>(LevelData& L) { return L.d; }
template <> LevelBufs<float2>& B<float2>(LevelData& L) { return L.f; }

}  // namespace ddamg

// timing kinds: 0 SAP colour sweep, 1 coarsest GMRES, 2 level operator, 3 orthonormalisation,
// 4 coarse-link construction
constexpr int kProfKinds = 5;

struct ddamg_handle {
    ddamg_params p;
    int L = 0;          // levels
    int W = 1;          // widest batch (max_rhs, test vectors)
    cudaStream_t s = nullptr;
    std::vector<ddamg::LevelData> lv;
    std::vector<void*> allocs;
    bool gauge = false, setup_done = false;
    // outer FGMRES (FP64, fine level)
    double2 *oV = nullptr, *oZ = nullptr, *ow = nullptr, *orr = nullptr, *ob = nullptr, *ox = nullptr;
    double2* ohost_tmp = nullptr;
    // scalars
    double2* dpart = nullptr;  // reduction partials
    double2* dh = nullptr;     // multidot results (2 x (max m + 1))
    double2* dcoef = nullptr;  // coefficients for multiaxpy
    double* dn = nullptr;      // norms
    double2* hpin = nullptr;   // pinned host mirror (downloads)
    double2* hpin2 = nullptr;  // pinned host staging (uploads)
    double2* dalpha = nullptr; // per-rhs scale factors
    double2* grad = nullptr;   // gradient work: psi, lambda, sigma_3 eta (3 fine vectors)
    ddamg::KrylovWork kry;                          // BiCGstab / CG comparison solvers (allocated on first use)
    ddamg::CoarseGmresWork cg;                      // lane 0: the handle's stream
    ddamg::CoarseClusterWork ccl;                   // the cluster kernel's workspace (if the device runs it)
    int coarse_kind = -1;                           // coarsest solver: -1 not chosen yet, 0 cooperative grid, 1 cluster
    int coarse_kind_batch = -1;                     // the same for several right-hand sides at once
    std::vector<ddamg::CoarseGmresWork> cg_lane;    // lanes 1..: concurrent coarsest solves of a batch
    std::vector<cudaStream_t> lane_s;
    std::vector<cudaEvent_t> lane_ev;
    std::vector<cudaStream_t> setup_s;  // extra streams of the setup's grouped coarse smoothing
    std::vector<cudaEvent_t> setup_ev;
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_setup_s = 0;
    long long launches_at_create = 0;
    // per-kernel event timing (ddamg_profile)
    struct ProfRec {
        int kind, level;
        cudaEvent_t a, b;
    };
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_next = 0;
    std::vector<ProfRec> prof_recs;
    std::string tune_log;  // autotuner decisions, one line per (level, batch width)
    // V-cycle preconditioner graphs, one per batch width; a width is captured on its second use
    // (the first runs directly: autotuning and first-use set-up happen there)
    struct CycleGraph {
        cudaGraphExec_t exec;
        long long kernels;
    };
    std::map<int, CycleGraph> graphs;
    std::set<int> graph_warm;
    bool graphs_off = false;  // a capture failed: launch directly from then on
    double prof_ms[kProfKinds][DDAMG_MAX_LEVELS] = {};
    long long prof_n[kProfKinds][DDAMG_MAX_LEVELS] = {};
    // fine-level Schwarz layouts by block counts (FGMRES_SAP, stand-alone fine SAP), made on first use
    std::map<std::pair<int, int>, ddamg::SapLayout> fine_sap;
    // iterations of the last run of each method (ddamg_counter), -1 before the first
    long long counts[DDAMG_COUNT_KINDS] = {-1, -1, -1, -1, -1, -1, -1};
    // device-driven solves: one graph per batch width whose conditional nodes run the FGMRES loops
    // (built on the second solve of a width; the first runs host driven and does the tuning)
    struct CapBody {
        int level, kind;  // kind: 0 the top graph, else the FgCtl run counter of the body
        long long kernels;
    };
    struct SolveGraph {
        cudaGraphExec_t exec;
        std::vector<CapBody> bodies;
    };
    std::map<int, SolveGraph> solve_graphs;
    std::set<int> solve_warm;
    bool solve_graphs_off = false;
    bool capturing = false;                 // h->s is recording a device-driven solve graph
    cudaGraph_t cap_top = nullptr;          // its top-level graph (conditional handles live there)
    std::vector<CapBody>* cap_bodies = nullptr;
    int cap_cur = -1;                       // body the capture is recording into
    long long cap_mark = 0;                 // g_launches when that segment began
    double2* ovin = nullptr;                // fixed copies of V_j and Z_j of the outer FGMRES
    double2* ozf = nullptr;
};

namespace ddamg {

static void* dalloc(ddamg_handle* h, size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) return nullptr;
    DDAMG_CUDA_TRY(cudaMalloc(&p, bytes));
    DDAMG_CUDA_TRY(cudaMemsetAsync(p, 0, bytes, h->s));
    h->allocs.push_back(p);
    return p;
}
template <typename V> static V* dalloc_t(ddamg_handle* h, size_t count) {
    return static_cast<V*>(dalloc(h, count * sizeof(V)));
}
static void sync(ddamg_handle* h) { DDAMG_CUDA_TRY(cudaStreamSynchronize(h->s)); }

// ------------------------------------------------------------------ per-kernel timing
static cudaEvent_t prof_event(ddamg_handle* h) {
    if (h->ev_next == h->ev_pool.size()) {
        cudaEvent_t e;
        DDAMG_CUDA_TRY(cudaEventCreate(&e));
        h->ev_pool.push_back(e);
    }
    return h->ev_pool[h->ev_next++];
}
struct ProfScope {
    ddamg_handle* h;
    int idx = -1;
    ProfScope(ddamg_handle* hh, int kind, int level) : h(hh) {
        if (!h->prof) return;
        cudaEvent_t a = prof_event(h), b = prof_event(h);
        DDAMG_CUDA_TRY(cudaEventRecord(a, h->s));
        h->prof_recs.push_back({kind, level, a, b});
        idx = (int)h->prof_recs.size() - 1;
    }
    ~ProfScope() {
        if (idx >= 0) cudaEventRecord(h->prof_recs[idx].b, h->s);
    }
};
static void prof_flush(ddamg_handle* h) {
    if (h->prof_recs.empty()) return;
    sync(h);
    for (auto& r : h->prof_recs) {
        float ms = 0;
        DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, r.a, r.b));
        h->prof_ms[r.kind][r.level] += ms;
        h->prof_n[r.kind][r.level] += 1;
    }
    h->prof_recs.clear();
    h->ev_next = 0;
}
static void bad(const std::string& m) { throw ParamFailure{m}; }

// ------------------------------------------------------------------ geometry
static void build_geometry(ddamg_handle* h) {
    const ddamg_params& p = h->p;
    if (p.levels < 2 || p.levels > DDAMG_MAX_LEVELS) bad("levels must be in [2, " + std::to_string(DDAMG_MAX_LEVELS) + "]");
    if (p.Nx < 2 || p.Nt < 2) bad("lattice too small");
    if (p.max_rhs < 1) bad("max_rhs must be >= 1");
    h->L = p.levels;
    h->lv.resize(p.levels);
    for (int l = 0; l < p.levels; l++) {
        Geom& g = h->lv[l].g;
        g.level = l;
        if (l == 0) {
            g.Nx = p.Nx;
            g.Nt = p.Nt;
            g.colors = 1;
        } else {
            const int* r = p.rows[l - 1];
            g.Nx = r[1];
            g.Nt = r[2];
            g.colors = r[3];
        }
        g.dof = 2 * g.colors;
        g.sites = g.Nx * g.Nt;
        if (l < p.levels - 1) {
            const int* r = p.rows[l];
            if (r[0] != l) bad("parameters row " + std::to_string(l) + " has level " + std::to_string(r[0]));
            g.agg_x = r[1];
            g.agg_t = r[2];
            g.ntest = r[3];
            g.sap_x = r[4];
            g.sap_t = r[5];
            if (g.agg_x <= 0 || g.agg_t <= 0 || g.Nx % g.agg_x || g.Nt % g.agg_t)
                bad("level " + std::to_string(l) + ": aggregation blocks must divide the lattice");
            if (g.sap_x <= 0 || g.sap_t <= 0 || g.Nx % g.sap_x || g.Nt % g.sap_t)
                bad("level " + std::to_string(l) + ": SAP blocks must divide the lattice");
            if (g.ntest < 1 || g.ntest > 16) bad("test vectors per level must be in [1, 16]");
            g.el_x = g.Nx / g.agg_x;
            g.el_t = g.Nt / g.agg_t;
            g.sel_x = g.Nx / g.sap_x;
            g.sel_t = g.Nt / g.sap_t;
            const int nb = g.sap_x * g.sap_t;
            // the reference fills RedBlocks[block/2] (src/sap.cpp:30-37): an odd count > 1 overruns it
            if (nb > 1 && nb % 2) bad("level " + std::to_string(l) + ": the number of SAP blocks must be even");
            const int NE = g.sel_x * g.sel_t * g.dof;
            if (NE > 4096) bad("SAP block has more than 4096 unknowns");
            const size_t sm = sap_smem_bytes(p.sap_gmres_restart_length, NE, true);
            if (sm > 227 * 1024) bad("SAP block Krylov basis does not fit in shared memory");
            const int dc = 2 * g.ntest;
            const size_t bl = 16 * ((size_t)5 * dc * dc + 2 * (size_t)g.dof * g.ntest + (size_t)g.dof * dc);
            if (bl > 227 * 1024) bad("coarse-link construction does not fit in shared memory");
            const size_t on = 16 * (size_t)g.ntest * g.el_x * g.el_t * g.colors;
            if (on > 227 * 1024) bad("aggregate too large for the orthonormalisation kernel");
        }
        if (l > 0 && g.dof > 64) bad("at most 32 test vectors");
    }
    for (int l = 1; l < p.levels; l++) {
        const Geom& pg = h->lv[l - 1].g;
        const Geom& g = h->lv[l].g;
        if (g.Nx != pg.agg_x || g.Nt != pg.agg_t || g.colors != pg.ntest) bad("inconsistent level sizes");
    }
    if (p.sap_gmres_restart_length > 8) bad("SAP block GMRES restart length above 8 is not supported");
    if (p.sap_gmres_restart_length < 1 || p.sap_gmres_restarts < 1 || p.coarse_gmres_restart_length < 1 ||
        p.coarse_gmres_restarts < 1 || p.kcycle_restart_length < 1 || p.kcycle_restarts < 1 ||
        p.fgmres_restart_length < 1 || p.fgmres_restarts < 1)
        bad("restart lengths and counts must be >= 1");
    if (p.nu1 < 0 || p.nu2 < 0 || p.sap_test_vectors_iterations < 0) bad("smoothing counts must be >= 0");
    if (p.cycle != DDAMG_CYCLE_V && p.cycle != DDAMG_CYCLE_K) bad("cycle must be 0 (V) or 1 (K)");
    if (p.precision != DDAMG_PREC_DOUBLE && p.precision != DDAMG_PREC_MIXED) bad("precision must be 0 or 1");
    if (p.tensor_cores < 0 || p.tensor_cores > 2) bad("tensor_cores must be 0, 1 or 2");
    if (p.coarse_kernel < 0 || p.coarse_kernel > 2) bad("coarse_kernel must be 0 (chosen), 1 (cooperative grid) or 2 (cluster)");
    int W = p.max_rhs;
    for (int l = 0; l < p.levels - 1; l++) W = std::max(W, h->lv[l].g.ntest);
    h->W = W;
}

static void allocate(ddamg_handle* h) {
    const ddamg_params& p = h->p;
    const int W = h->W, L = h->L;
    const bool mixed = p.precision == DDAMG_PREC_MIXED;
    for (int l = 0; l < L; l++) {
        LevelData& D = h->lv[l];
        const Geom& g = D.g;
        D.fp32 = mixed && l < L - 1;
        const long n = g.size();
        if (l == 0) D.d.U = dalloc_t<double2>(h, 2L * g.sites);
        else D.d.links = dalloc_t<double2>(h, (size_t)g.sites * 5 * g.dof * g.dof);
        if (l < L - 1) D.d.tv = dalloc_t<double2>(h, (size_t)g.ntest * n);
        D.d.eta = dalloc_t<double2>(h, (size_t)W * n);
        D.d.psi = dalloc_t<double2>(h, (size_t)W * n);
        D.d.r = dalloc_t<double2>(h, (size_t)W * n);
        D.d.t = dalloc_t<double2>(h, (size_t)W * n);
        if (D.fp32) {
            if (l == 0) D.f.U = dalloc_t<float2>(h, 2L * g.sites);
            else D.f.links = dalloc_t<float2>(h, (size_t)g.sites * 5 * g.dof * g.dof);
            D.f.tv = dalloc_t<float2>(h, (size_t)g.ntest * n);
            D.f.eta = dalloc_t<float2>(h, (size_t)W * n);
            D.f.psi = dalloc_t<float2>(h, (size_t)W * n);
            D.f.r = dalloc_t<float2>(h, (size_t)W * n);
            D.f.t = dalloc_t<float2>(h, (size_t)W * n);
        }
        // transfer buffer in the previous level's precision when it differs from this level's
        if (l > 0 && h->lv[l - 1].fp32 && !D.fp32) D.f.xfer = dalloc_t<float2>(h, (size_t)W * n);
        if (l > 0 && p.cycle == DDAMG_CYCLE_K) {
            const int km = p.kcycle_restart_length;
            const size_t Rn = (size_t)p.max_rhs * n;
            if (D.fp32) {
                D.f.kV = dalloc_t<float2>(h, (km + 1) * Rn);
                D.f.kZ = dalloc_t<float2>(h, km * Rn);
                D.f.kw = dalloc_t<float2>(h, Rn);
                D.f.kr = dalloc_t<float2>(h, Rn);
                D.f.kin = dalloc_t<float2>(h, Rn);
                D.f.kzf = dalloc_t<float2>(h, Rn);
            } else {
                D.d.kV = dalloc_t<double2>(h, (km + 1) * Rn);
                D.d.kZ = dalloc_t<double2>(h, km * Rn);
                D.d.kw = dalloc_t<double2>(h, Rn);
                D.d.kr = dalloc_t<double2>(h, Rn);
                D.d.kin = dalloc_t<double2>(h, Rn);
                D.d.kzf = dalloc_t<double2>(h, Rn);
            }
        }
        if (l == 0 || p.cycle == DDAMG_CYCLE_K) {
            const int fm = l == 0 ? p.fgmres_restart_length : p.kcycle_restart_length;
            const size_t R = (size_t)p.max_rhs;
            FgDev& f = D.fg;
            f.H = dalloc_t<double2>(h, R * (fm + 1) * fm);
            f.gm = dalloc_t<double2>(h, R * (fm + 1));
            f.cn = dalloc_t<double2>(h, R * fm);
            f.sn = dalloc_t<double2>(h, R * fm);
            f.coef = dalloc_t<double2>(h, R * fm);
            f.alpha = dalloc_t<double2>(h, R);
            f.dots = dalloc_t<double2>(h, 2 * R * (fm + 1));
            f.nrm = dalloc_t<double>(h, 2 * R);
            f.norm_b = dalloc_t<double>(h, R);
            f.err = dalloc_t<double>(h, R);
            f.maxIt = dalloc_t<int>(h, R);
            f.done = dalloc_t<int>(h, R);
            f.arn = dalloc_t<int>(h, R);
            f.ret = dalloc_t<int>(h, R);
            f.ctl = dalloc_t<int>(h, kFgCtlWords);
        }
        D.done = dalloc_t<int>(h, W);
        D.vv = dalloc_t<double>(h, W);
        D.rr = dalloc_t<double>(h, W);
        if (l < L - 1) {
            // red iff (bx + bt) even (src/sap.cpp:27-38); a single block is both colours
            std::vector<int> red, black;
            const int nb = g.sap_x * g.sap_t;
            for (int b = 0; b < nb; b++) {
                const int bx = b / g.sap_t, bt = b % g.sap_t;
                if (nb == 1) {
                    red.push_back(b);
                    black.push_back(b);
                } else if ((bx + bt) % 2 == 0) red.push_back(b);
                else black.push_back(b);
            }
            D.red = dalloc_t<int>(h, red.size());
            D.black = dalloc_t<int>(h, black.size());
            DDAMG_CUDA_TRY(cudaMemcpyAsync(D.red, red.data(), red.size() * sizeof(int), cudaMemcpyHostToDevice, h->s));
            DDAMG_CUDA_TRY(
                cudaMemcpyAsync(D.black, black.data(), black.size() * sizeof(int), cudaMemcpyHostToDevice, h->s));
            D.nred = (int)red.size();
            D.nblack = (int)black.size();
            sync(h);
        }
        if (D.fp32 && l >= 1 && l < L - 1 && p.tensor_cores && W >= kTcMinRhs && tc_sap_supported(g)) {
            TcSapWork& T = D.tcw;
            const int m = p.sap_gmres_restart_length;
            const long tasks = (long)std::max(D.nred, D.nblack) * W;
            T.vec = tasks * g.sel_x * g.sel_t * g.dof;
            T.b = dalloc_t<float2>(h, T.vec);
            T.x = dalloc_t<float2>(h, T.vec);
            T.w = dalloc_t<float2>(h, T.vec);
            T.V = dalloc_t<float2>(h, (size_t)(m + 1) * T.vec);
            T.act = dalloc_t<int>(h, tasks);
            T.fin = dalloc_t<int>(h, tasks);
            T.arn = dalloc_t<int>(h, tasks);
            T.maxit = dalloc_t<int>(h, tasks);
            T.normb = dalloc_t<double>(h, tasks);
            T.err = dalloc_t<double>(h, tasks);
            T.H = dalloc_t<double2>(h, (size_t)(m + 1) * m * tasks);
            T.gm = dalloc_t<double2>(h, (size_t)(m + 1) * tasks);
            T.cn = dalloc_t<double2>(h, (size_t)m * tasks);
            T.sn = dalloc_t<double2>(h, (size_t)m * tasks);
            T.tiles = dalloc_t<float>(h, (size_t)g.sites * 5 * kTcTileFloats);
            T.status = dalloc_t<int>(h, 1);
            D.tc = true;
        }
    }
    // outer FGMRES, all right-hand sides of one call in lockstep
    const long n0 = h->lv[0].g.size();
    const int m = p.fgmres_restart_length;
    const size_t Rn0 = (size_t)p.max_rhs * n0;
    h->oV = dalloc_t<double2>(h, (m + 1) * Rn0);
    h->oZ = dalloc_t<double2>(h, m * Rn0);
    h->ow = dalloc_t<double2>(h, Rn0);
    h->orr = dalloc_t<double2>(h, Rn0);
    h->ob = dalloc_t<double2>(h, Rn0);
    h->ox = dalloc_t<double2>(h, Rn0);
    h->ovin = dalloc_t<double2>(h, Rn0);
    h->ozf = dalloc_t<double2>(h, Rn0);
    const int mm = std::max(m, std::max(p.kcycle_restart_length, 1)) + 2;
    h->dpart = dalloc_t<double2>(h, (size_t)kRedBlocks * (2 * (size_t)W * mm + 2));
    h->dh = dalloc_t<double2>(h, 2 * (size_t)W * mm + 2);
    h->dcoef = dalloc_t<double2>(h, (size_t)W * mm + 2);
    h->dalpha = dalloc_t<double2>(h, (size_t)W + 2);
    h->dn = dalloc_t<double>(h, 2 * W + 4);
    DDAMG_CUDA_TRY(cudaMallocHost(&h->hpin, sizeof(double2) * (2 * (size_t)W * mm + 2 * W + 8)));
    DDAMG_CUDA_TRY(cudaMallocHost(&h->hpin2, sizeof(double2) * ((size_t)W * (mm + 1) + 8)));
    // coarsest GMRES
    const Geom& gc = h->lv[L - 1].g;
    const int cm = p.coarse_gmres_restart_length;
    coarse_gmres_prepare(h->cg, (int)gc.size(), cm, gc.dof, p.device);
    h->cg.V = dalloc_t<double2>(h, (size_t)(cm + 1) * gc.size());
    h->cg.w = dalloc_t<double2>(h, gc.size());
    h->cg.r = dalloc_t<double2>(h, gc.size());
    h->cg.partial = dalloc_t<double2>(h, (size_t)3 * h->cg.grid * (cm + 2));
    h->cg.H = dalloc_t<double2>(h, (size_t)(cm + 1) * cm);
    h->cg.bar = dalloc_t<unsigned>(h, 2);
    h->cg.status = dalloc_t<int>(h, 2);
    h->cg.spin_limit = p.coarse_barrier_polls;
    if (coarse_cluster_prepare(h->ccl, (int)gc.size(), cm, gc.dof, p.max_rhs)) {
        h->ccl.ws = dalloc_t<double2>(h, (size_t)h->ccl.clusters * h->ccl.wstride);
        h->ccl.status = dalloc_t<int>(h, 2);
    }
    // extra lanes so the coarsest solves of a batch run side by side (each a cooperative grid)
    const int lanes = std::min(p.max_rhs, 8);
    DDAMG_CUDA_TRY(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
    for (int k = 1; k < lanes; k++) {
        CoarseGmresWork w = h->cg;
        w.V = dalloc_t<double2>(h, (size_t)(cm + 1) * gc.size());
        w.w = dalloc_t<double2>(h, gc.size());
        w.r = nullptr;
        w.partial = dalloc_t<double2>(h, (size_t)3 * h->cg.grid * (cm + 2));
        w.H = dalloc_t<double2>(h, (size_t)(cm + 1) * cm);
        w.bar = dalloc_t<unsigned>(h, 2);
        w.status = dalloc_t<int>(h, 2);
        h->cg_lane.push_back(w);
        cudaStream_t ls;
        cudaEvent_t le;
        DDAMG_CUDA_TRY(cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking));
        DDAMG_CUDA_TRY(cudaEventCreateWithFlags(&le, cudaEventDisableTiming));
        h->lane_s.push_back(ls);
        h->lane_ev.push_back(le);
    }
    sync(h);
}

// ------------------------------------------------------------------ operators
// The batched FP32 level operator of a level with tensor-core tiles: the first call per batch width
// times the CUDA-core kernel and each tensor-core shape on the call's own operands (three runs each,
// outside any graph capture: the first solve of a width runs directly) and keeps the fastest; the
// last run of the chosen kernel leaves the result.
static int tc_op_for(ddamg_handle* h, int l, const float2* in, float2* out, const float2* b, int nrhs) {
    LevelData& D = h->lv[l];
    auto it = D.tc_op.find(nrhs);
    if (it != D.tc_op.end()) return it->second;
    if (h->capturing) return -1;
    const Geom& g = D.g;
    cudaStream_t s = h->s;
    cudaEvent_t e0, e1;
    DDAMG_CUDA_TRY(cudaEventCreate(&e0));
    DDAMG_CUDA_TRY(cudaEventCreate(&e1));
    auto run = [&](int k) {
        if (k < 0) launch_coarse_op<float2>(s, D.f.links, in, out, b, g.Nx, g.Nt, g.dof, h->p.m0, nrhs);
        else launch_coarse_op_tc(s, g, D.tcw.tiles, in, out, b, h->p.m0, nrhs, k, D.tcw.status);
    };
    std::ostringstream o;
    o << "level " << l << " rhs " << nrhs << " level operator:";
    int best = -1;
    double best_us = 0;
    const bool forced = h->p.tensor_cores == 2;  // tensor cores whatever the timing
    for (int k = forced ? 0 : -1; k < tc_op_shapes(); k++) {
        if (k >= 0 && tc_op_shape_rg(k) / 2 >= nrhs * 2) continue;  // at most 4x padding
        run(k);
        DDAMG_CUDA_TRY(cudaEventRecord(e0, s));
        for (int q = 0; q < 3; q++) run(k);
        DDAMG_CUDA_TRY(cudaEventRecord(e1, s));
        DDAMG_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        const double us = 1e3 * ms / 3;
        if ((best == -1 && (k == -1 || forced)) || us < best_us) {
            best = k;
            best_us = us;
        }
        if (k < 0) o << " [CUDA cores: " << us << " us]";
        else o << " [tensor cores, rhs/cta " << tc_op_shape_rg(k) << ": " << us << " us]";
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    run(best);
    D.tc_op[nrhs] = best;
    o << " -> " << (best < 0 ? std::string("CUDA cores") : "tensor cores rhs/cta " + std::to_string(tc_op_shape_rg(best)));
    h->tune_log += o.str() + "\n";
    return best;
}
// allow_tc = false keeps the CUDA-core kernel (the setup's smoothing: TF32 would coarsen the test vectors)
template <typename V>
static void level_op(ddamg_handle* h, int l, const V* in, V* out, const V* b, int nrhs, bool allow_tc = true) {
    ProfScope ps(h, 2, l);
    LevelData& D = h->lv[l];
    const Geom& g = D.g;
    if (l == 0) {
        launch_wilson<V>(h->s, B<V>(D).U, in, out, b, g.Nx, g.Nt, h->p.m0, 0, nrhs);
        return;
    }
    if constexpr (std::is_same<V, float2>::value) {
        if (allow_tc && D.tc && nrhs >= kTcMinRhs && h->p.tensor_cores && tc_op_supported(g)) {
            auto it = D.tc_op.find(nrhs);
            if (it == D.tc_op.end()) {  // tuned on this call, which it also completes
                tc_op_for(h, l, in, out, b, nrhs);
                if (D.tc_op.count(nrhs)) return;
            } else if (it->second >= 0) {
                launch_coarse_op_tc(h->s, g, D.tcw.tiles, in, out, b, h->p.m0, nrhs, it->second, D.tcw.status);
                return;
            }
        }
    }
    launch_coarse_op<V>(h->s, B<V>(D).links, in, out, b, g.Nx, g.Nt, g.dof, h->p.m0, nrhs);
}

// tile shape of the tensor-core sweep for this batch width: tuned on first use (the tuner times the
// candidate shapes on the sweep's own data and syncs the stream), then cached
static int tc_shape_for(ddamg_handle* h, int l, const float2* r, const SapArgs& a, int nrhs) {
    LevelData& D = h->lv[l];
    auto it = D.tc_shape.find(nrhs);
    if (it != D.tc_shape.end()) return it->second;
    std::vector<double> us(tc_sweep_shapes());
    const int best = tune_sap_tc(h->s, D.g, D.tcw, r, a, nrhs, us.data());
    D.tc_shape[nrhs] = best;
    std::ostringstream o;
    o << "level " << l << " rhs " << nrhs << ":";
    for (int i = 0; i < (int)us.size(); i++) {
        int rg, na, nch;
        tc_sweep_shape(i, &rg, &na, &nch);
        if (us[i] < 0) continue;
        o << " [rhs/cta " << rg << " stages " << na << " chains " << nch << ": " << us[i] << " us"
          << (i == best ? " *" : "") << "]";
    }
    h->tune_log += o.str() + "\n";
    return best;
}

// the variant (right-hand sides per CTA and block-solver kernel) of the CUDA-core coarse sweep for this
// batch width and precision: tuned on first use (one timed sweep per candidate into the level's scratch
// field t; syncs), then cached
template <typename V> static int rb_for(ddamg_handle* h, int l, const V* r, const SapArgs& a, int nrhs) {
    LevelData& D = h->lv[l];
    const int key = nrhs * 2 + (std::is_same<V, float2>::value ? 1 : 0);
    auto it = D.rb_choice.find(key);
    if (it != D.rb_choice.end()) return it->second;
    double us[kSapVariantCount];
    const int best = tune_sap_rb<V>(h->s, D.g, B<V>(D).links, r, B<V>(D).t, a, nrhs, us);
    D.rb_choice[key] = best;
    std::ostringstream o;
    o << "level " << l << " rhs " << nrhs << (key & 1 ? " fp32" : " fp64") << " CUDA-core sweep:";
    static const char* kname[2] = {"block", "block2"};
    for (int i = 0; i < kSapVariantCount; i++)
        if (us[i] >= 0)
            o << " [rhs/cta " << kSapVariants[i] / 4 << " " << kname[kSapVariants[i] % 4] << ": " << us[i] << " us"
              << (kSapVariants[i] == best ? " *" : "") << "]";
    h->tune_log += o.str() + "\n";
    return best;
}

// SAP_C::SAP (src/sap.cpp:81-165) on nrhs independent vectors; returns the reference's value
// for rhs 0 when want_iters (one host sync), else nu.  lay: a fine-level block layout other than the
// level's; allow_tc: batched FP32 coarse sweeps may use the tensor-core block operator.
// A black sweep may form its blocks' residuals from the iterate only if no two blocks of one colour
// touch: every block count is even (checkerboard across the periodic wrap) or 1 (the block is its own
// neighbour across the wrap, and reads the iterate before it updates it)
static bool fusable_residual(const Geom& g) {
    return (g.sap_x == 1 || g.sap_x % 2 == 0) && (g.sap_t == 1 || g.sap_t % 2 == 0);
}
template <typename V>
static int sap_t(ddamg_handle* h, int l, const V* v, V* x, int nu, double tol, bool x_zero, int nrhs, bool want_iters,
                 const SapLayout* lay = nullptr, bool allow_tc = true) {
    LevelData& D = h->lv[l];
    const Geom& g = lay ? lay->g : D.g;  // the block layout of the sweeps (the operator is the level's)
    const long n = g.size();
    V* r = B<V>(D).r;
    DDAMG_CUDA_TRY(cudaMemsetAsync(D.done, 0, sizeof(int) * nrhs, h->s));
    const bool check = tol > 0.0;
    if (check) launch_norm2<V>(h->s, v, n, n, nrhs, h->dpart, D.vv);
    const bool tc = std::is_same<V, float2>::value && D.tc && allow_tc && nrhs >= kTcMinRhs;
    // with the sweep variant already tuned, the first red sweep also forms its blocks' residuals itself
    // (r = v - D x is read only there); the first use tunes on the global residual
    bool fuse0 = false;
    if (!x_zero && l > 0 && !lay && !tc && fusable_residual(g)) {
        auto itv = D.rb_choice.find(nrhs * 2 + (std::is_same<V, float2>::value ? 1 : 0));
        fuse0 = itv != D.rb_choice.end() && itv->second % 4 == 1;
    }
    if (x_zero) DDAMG_CUDA_TRY(cudaMemcpyAsync(r, v, sizeof(V) * n * nrhs, cudaMemcpyDeviceToDevice, h->s));
    else if (!fuse0) level_op<V>(h, l, x, r, v, nrhs, allow_tc);  // r = v - D x
    SapArgs a{h->p.sap_gmres_restart_length, h->p.sap_gmres_restarts, h->p.sap_gmres_tolerance, h->p.m0, nullptr, 0,
              D.done};
    for (int it = 0; it < nu; it++) {
        bool fused = false;  // this iteration's black sweep forms its blocks' residuals itself
        for (int colour = 0; colour < 2; colour++) {
            a.blocks = colour == 0 ? (lay ? lay->red : D.red) : (lay ? lay->black : D.black);
            a.nblocks = colour == 0 ? (lay ? lay->nred : D.nred) : (lay ? lay->nblack : D.nblack);
            a.vres = ((colour == 1 && fused) || (colour == 0 && it == 0 && fuse0)) ? static_cast<const void*>(v)
                                                                                 : nullptr;
            int var = 0;
            {
                ProfScope ps(h, 0, l);
                if (l == 0) launch_sap_sweep_fine<V>(h->s, g, B<V>(D).U, r, x, a, nrhs);
                else if (tc)
                    launch_sap_sweep_tc(h->s, g, D.tcw, reinterpret_cast<const float2*>(r),
                                        reinterpret_cast<float2*>(x), a, nrhs,
                                        tc_shape_for(h, l, reinterpret_cast<const float2*>(r), a, nrhs));
                else {
                    var = rb_for<V>(h, l, r, a, nrhs);
                    launch_sap_sweep_coarse<V>(h->s, g, B<V>(D).links, r, x, a, nrhs, var);
                }
            }
            // the residual after the last black sweep only feeds the convergence test; the one after a
            // red sweep is left to the black sweep where sap_block2_kernel runs it (each block forms its
            // own r_B = v_B - (D x)_B, so the global operator application is saved)
            const bool last = (colour == 1 && it == nu - 1);
            if (colour == 0 && l > 0 && !lay && var % 4 == 1 && fusable_residual(g)) {
                fused = true;
                continue;
            }
            if (!last || (check && want_iters)) level_op<V>(h, l, x, r, v, nrhs, allow_tc);
        }
        if (check && (it < nu - 1 || want_iters)) {
            launch_norm2<V>(h->s, r, n, n, nrhs, h->dpart, D.rr);
            launch_flag_converged(h->s, D.rr, D.vv, tol, nrhs, it, D.done);
        }
    }
    if (!want_iters) return nu;
    int done0 = 0;
    DDAMG_CUDA_TRY(cudaMemcpyAsync(&done0, D.done, sizeof(int), cudaMemcpyDeviceToHost, h->s));
    sync(h);
    return done0 ? done0 - 1 : nu;
}

static int coarse_solve(ddamg_handle* h, const double2* b, double2* x) {
    ProfScope ps(h, 1, h->L - 1);
    LevelData& D = h->lv[h->L - 1];
    const Geom& g = D.g;
    if (h->coarse_kind == 1)
        launch_coarse_gmres_cluster(h->s, h->ccl, D.d.links, b, x, 1, g.Nx, g.Nt, g.dof, h->p.m0,
                                    h->p.coarse_gmres_restart_length, h->p.coarse_gmres_restarts,
                                    h->p.coarse_gmres_tolerance);
    else
        launch_coarse_gmres(h->s, h->cg, D.d.links, b, x, g.Nx, g.Nt, g.dof, h->p.m0,
                            h->p.coarse_gmres_restart_length, h->p.coarse_gmres_restarts,
                            h->p.coarse_gmres_tolerance);
    return 0;
}
static void coarse_solve_batch(ddamg_handle* h, const double2* b, double2* x, int R) {
    if (R == 1) {
        coarse_solve(h, b, x);
        return;
    }
    ProfScope ps(h, 1, h->L - 1);
    LevelData& D = h->lv[h->L - 1];
    const Geom& g = D.g;
    if (h->coarse_kind_batch == 1) {  // one launch: each cluster loops over its share of the right-hand sides
        launch_coarse_gmres_cluster(h->s, h->ccl, D.d.links, b, x, R, g.Nx, g.Nt, g.dof, h->p.m0,
                                    h->p.coarse_gmres_restart_length, h->p.coarse_gmres_restarts,
                                    h->p.coarse_gmres_tolerance);
        return;
    }
    const long n = g.size();
    const int K = 1 + (int)h->cg_lane.size();
    DDAMG_CUDA_TRY(cudaEventRecord(h->fork_ev, h->s));
    for (int k = 1; k < K && k < R; k++) DDAMG_CUDA_TRY(cudaStreamWaitEvent(h->lane_s[k - 1], h->fork_ev, 0));
    for (int r = 0; r < R; r++) {
        const int k = r % K;
        cudaStream_t st = k == 0 ? h->s : h->lane_s[k - 1];
        const CoarseGmresWork& w = k == 0 ? h->cg : h->cg_lane[k - 1];
        launch_coarse_gmres(st, w, D.d.links, b + r * n, x + r * n, g.Nx, g.Nt, g.dof, h->p.m0,
                            h->p.coarse_gmres_restart_length, h->p.coarse_gmres_restarts,
                            h->p.coarse_gmres_tolerance);
    }
    for (int k = 1; k < K && k < R; k++) {
        DDAMG_CUDA_TRY(cudaEventRecord(h->lane_ev[k - 1], h->lane_s[k - 1]));
        DDAMG_CUDA_TRY(cudaStreamWaitEvent(h->s, h->lane_ev[k - 1], 0));
    }
}
static void check_coarse_status(ddamg_handle* h, int* iters) {
    const int K = 1 + (int)h->cg_lane.size();
    std::vector<int> st(2 * K + 2, 0);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(st.data(), h->cg.status, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->s));
    for (int k = 1; k < K; k++)
        DDAMG_CUDA_TRY(cudaMemcpyAsync(st.data() + 2 * k, h->cg_lane[k - 1].status, 2 * sizeof(int),
                                       cudaMemcpyDeviceToHost, h->s));
    if (h->ccl.status)
        DDAMG_CUDA_TRY(
            cudaMemcpyAsync(st.data() + 2 * K, h->ccl.status, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->s));
    sync(h);
    for (int k = 0; k < K; k++)
        if (st[2 * k] != 0) throw TimeoutFailure();
    if (iters) *iters = h->coarse_kind == 1 ? st[2 * K + 1] : st[1];
}
// the coarsest solver, chosen once per handle at the end of its first setup: the cooperative-grid
// kernel and the cluster kernel each solve random right-hand sides twice, one and (with max_rhs > 1) a
// batch of max_rhs, and the faster second run wins for each (the cluster kernel only where the device
// runs its clusters)
static void tune_coarse(ddamg_handle* h) {
    if (h->coarse_kind >= 0) return;
    const int Rb = std::max(1, h->p.max_rhs);
    if (!h->ccl.ws || h->p.coarse_kernel == 1) {
        h->coarse_kind = h->coarse_kind_batch = 0;
        h->tune_log += h->ccl.ws ? "coarsest solve: cooperative grid (requested)\n"
                                 : "coarsest solve: cooperative grid (no cluster kernel for this level)\n";
        return;
    }
    if (h->p.coarse_kernel == 2) {
        h->coarse_kind = h->coarse_kind_batch = 1;
        h->tune_log += "coarsest solve: cluster of " + std::to_string(h->ccl.C) + " CTAs (requested)\n";
        return;
    }
    LevelData& D = h->lv[h->L - 1];
    const Geom& g = D.g;
    cudaStream_t s = h->s;
    launch_fill_uniform(s, D.d.eta, g.size() * Rb, 0x5eedc0a25ull, 0);
    auto time_it = [&](int kind, int R) {
        float ms = 0;
        h->coarse_kind = h->coarse_kind_batch = kind;
        for (int rep = 0; rep < 2; rep++) {
            DDAMG_CUDA_TRY(cudaEventRecord(h->ev0, s));
            coarse_solve_batch(h, D.d.eta, D.d.psi, R);
            DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, s));
            sync(h);
            DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        }
        check_coarse_status(h, nullptr);
        return 1e3 * ms;
    };
    const double u0 = time_it(0, 1), u1 = time_it(1, 1);
    const int k1 = u1 < u0 ? 1 : 0;
    int kb = k1;
    double b0 = 0, b1 = 0;
    if (Rb > 1) {
        b0 = time_it(0, Rb);
        b1 = time_it(1, Rb);
        kb = b1 < b0 ? 1 : 0;
    }
    h->coarse_kind = k1;
    h->coarse_kind_batch = kb;
    char buf[320];
    snprintf(buf, sizeof(buf),
             "coarsest solve, 1 rhs: cooperative grid %d CTAs %.1f us, cluster %d CTAs %.1f us -> %s\n", h->cg.grid, u0,
             h->ccl.C, u1, k1 ? "cluster" : "cooperative grid");
    h->tune_log += buf;
    if (Rb > 1) {
        snprintf(buf, sizeof(buf),
                 "coarsest solve, %d rhs: cooperative grid on %d streams %.1f us, %d clusters %.1f us -> %s\n", Rb,
                 1 + (int)h->cg_lane.size(), b0, std::min(Rb, h->ccl.clusters), b1, kb ? "cluster" : "cooperative grid");
        h->tune_log += buf;
    }
}

// the tensor-core sweeps record a bounded wait that gave up in a status word per level
static void check_tc_status(ddamg_handle* h) {
    for (int l = 0; l < h->L; l++) {
        LevelData& D = h->lv[l];
        if (!D.tc) continue;
        int st = 0;
        DDAMG_CUDA_TRY(cudaMemcpyAsync(&st, D.tcw.status, sizeof(int), cudaMemcpyDeviceToHost, h->s));
        sync(h);
        if (st != 0) throw TimeoutFailure();
    }
}

// ------------------------------------------------------------------ FGMRES (host driven)
// FGMRES::fgmres (src/fgmres.cpp:5-97) for R right-hand sides in lockstep, with CGS2 for the
// Arnoldi step.  Every right-hand side keeps its own Hessenberg matrix, rotations, break point
// (maxIt, not reset between restarts: src/fgmres.cpp:14,56) and convergence state; one that has
// finished is fed zero vectors so the shared launches leave it unchanged.  The small dense work
// (Givens, back substitution) runs on the host in FP64: one sync per Arnoldi step.
// A(in, out, R): out = A in.  M(in, out, R, restart): out = M in, where out still holds the
// previous restart's Z_j (the K-cycle's initial guess, src/amg.cpp:43-45).
template <typename V> struct Krylov {
    V* Vb;  // (m+1) x R x n
    V* Z;   // m x R x n
    V* w;   // R x n
    V* r;   // R x n
};
template <typename V>
static void fgmres_host(ddamg_handle* h, long n, int R, int m, int restarts, double tol,
                        const std::function<void(const V*, V*, int)>& A,
                        const std::function<void(const V*, V*, int, int)>* M, const V* b, const V* x0, bool x0_zero,
                        V* x, Krylov<V> K, int* iters, double* rel) {
    cudaStream_t s = h->s;
    const long Rn = (long)R * n;
    if (x0_zero) DDAMG_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(V) * Rn, s));
    else if (x0 != x) DDAMG_CUDA_TRY(cudaMemcpyAsync(x, x0, sizeof(V) * Rn, cudaMemcpyDeviceToDevice, s));
    DDAMG_CUDA_TRY(cudaMemsetAsync(K.Z, 0, sizeof(V) * Rn * m, s));  // setZeros (include/fgmres.h:119-143)
    if (x0_zero) DDAMG_CUDA_TRY(cudaMemcpyAsync(K.r, b, sizeof(V) * Rn, cudaMemcpyDeviceToDevice, s));
    else {
        A(x, K.w, R);
        launch_sub<V>(s, b, K.w, K.r, Rn);
    }
    launch_norm2<V>(s, b, n, n, R, h->dpart, h->dn);
    launch_norm2<V>(s, K.r, n, n, R, h->dpart, h->dn + R);
    double* hn_pin = reinterpret_cast<double*>(h->hpin);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(hn_pin, h->dn, sizeof(double) * 2 * R, cudaMemcpyDeviceToHost, s));
    sync(h);
    std::vector<double> norm_b(R), err(R);
    for (int r = 0; r < R; r++) {
        norm_b[r] = std::sqrt(hn_pin[r]);
        err[r] = std::sqrt(hn_pin[R + r]);
        if (!(err[r] == err[r]) || !(norm_b[r] == norm_b[r])) throw ParamFailure{"NaN in the right-hand side"};
    }
    std::vector<double2> H((size_t)R * (m + 1) * m), gm((size_t)R * (m + 1)), cn((size_t)R * m), sn((size_t)R * m);
    std::vector<int> maxIt(R, m), ret(R, restarts * m);
    std::vector<char> done(R, 0), arn(R, 0);
    for (int r = 0; r < R; r++) done[r] = norm_b[r] == 0.0;  // zero right-hand side: x = x0 = 0
    double2* alpha = h->hpin2;            // R values uploaded to h->dalpha
    double2* coef = h->hpin2 + R;         // R x m back-substitution results uploaded to h->dcoef
    auto upload_alpha = [&]() {
        DDAMG_CUDA_TRY(cudaMemcpyAsync(h->dalpha, alpha, sizeof(double2) * R, cudaMemcpyHostToDevice, s));
    };
    for (int k = 0; k < restarts; k++) {
        bool any = false;
        for (int r = 0; r < R; r++) {
            arn[r] = !done[r];
            any |= !done[r];
            alpha[r] = make_double2(done[r] ? 0.0 : 1.0 / err[r], 0.0);
            gm[(size_t)r * (m + 1)] = make_double2(err[r], 0.0);
        }
        if (!any) break;
        upload_alpha();
        launch_scale<V>(s, h->dalpha, K.r, K.Vb, n, R);  // V_0 = r / beta
        for (int j = 0; j < m; j++) {
            bool anyarn = false;
            for (int r = 0; r < R; r++) anyarn |= arn[r] != 0;
            if (!anyarn) break;
            const V* vj = K.Vb + (long)j * Rn;
            V* zj = K.Z + (long)j * Rn;
            if (M) (*M)(vj, zj, R, k);
            else DDAMG_CUDA_TRY(cudaMemcpyAsync(zj, vj, sizeof(V) * Rn, cudaMemcpyDeviceToDevice, s));
            A(zj, K.w, R);
            double2* h1 = h->dh;
            double2* h2 = h->dh + (long)R * (j + 1);
            launch_multidot<V>(s, K.Vb, Rn, n, j + 1, K.w, n, n, R, h->dpart, h1);
            launch_multiaxpy<V>(s, K.Vb, Rn, n, j + 1, h1, K.w, n, n, R, -1.0);
            launch_multidot<V>(s, K.Vb, Rn, n, j + 1, K.w, n, n, R, h->dpart, h2);
            launch_multiaxpy<V>(s, K.Vb, Rn, n, j + 1, h2, K.w, n, n, R, -1.0);
            launch_norm2<V>(s, K.w, n, n, R, h->dpart, h->dn);
            DDAMG_CUDA_TRY(
                cudaMemcpyAsync(h->hpin, h->dh, sizeof(double2) * 2 * R * (j + 1), cudaMemcpyDeviceToHost, s));
            double* dn_pin = reinterpret_cast<double*>(h->hpin + 2 * R * (j + 1));
            DDAMG_CUDA_TRY(cudaMemcpyAsync(dn_pin, h->dn, sizeof(double) * R, cudaMemcpyDeviceToHost, s));
            sync(h);
            for (int r = 0; r < R; r++) {
                alpha[r] = make_double2(0.0, 0.0);
                if (!arn[r]) continue;
                double2* Hr = H.data() + (size_t)r * (m + 1) * m;
                double2* gr = gm.data() + (size_t)r * (m + 1);
                double2* cr = cn.data() + (size_t)r * m;
                double2* sr = sn.data() + (size_t)r * m;
                auto Hij = [&](int i, int jj) -> double2& { return Hr[(size_t)i * m + jj]; };
                for (int i = 0; i <= j; i++)
                    Hij(i, j) = h->hpin[(size_t)r * (j + 1) + i] + h->hpin[(size_t)R * (j + 1) + r * (j + 1) + i];
                const double hn = std::sqrt(dn_pin[r]);
                if (!(hn == hn)) throw ParamFailure{"NaN in the Krylov basis"};
                Hij(j + 1, j) = make_double2(hn, 0.0);
                if (hn > 0) alpha[r] = make_double2(1.0 / hn, 0.0);
                for (int i = 0; i < j; i++) {  // FGMRES::rotation (src/fgmres.cpp:99-115)
                    double2 tmp = cmulc(cr[i], Hij(i, j)) + cmulc(sr[i], Hij(i + 1, j));
                    Hij(i + 1, j) = cmul(cr[i], Hij(i + 1, j)) - cmul(sr[i], Hij(i, j));
                    Hij(i, j) = tmp;
                }
                const double den = std::sqrt(cnorm2(Hij(j, j)) + cnorm2(Hij(j + 1, j)));
                sr[j] = make_double2(Hij(j + 1, j).x / den, Hij(j + 1, j).y / den);
                cr[j] = make_double2(Hij(j, j).x / den, Hij(j, j).y / den);
                Hij(j, j) = cmulc(cr[j], Hij(j, j)) + cmulc(sr[j], Hij(j + 1, j));
                Hij(j + 1, j) = make_double2(0.0, 0.0);
                gr[j + 1] = -cmul(sr[j], gr[j]);
                gr[j] = cmulc(cr[j], gr[j]);
                if (std::sqrt(cnorm2(gr[j + 1])) < tol * norm_b[r]) {
                    maxIt[r] = j + 1;
                    arn[r] = 0;
                    alpha[r] = make_double2(0.0, 0.0);  // V_{j+1} is not used again
                }
            }
            upload_alpha();
            launch_scale<V>(s, h->dalpha, K.w, K.Vb + (long)(j + 1) * Rn, n, R);
        }
        // solve_upper_triangular (src/fgmres.cpp:118-128); x += sum_j eta_j Z_j
        for (int r = 0; r < R; r++) {
            double2* cf = coef + (size_t)r * m;
            for (int i = 0; i < m; i++) cf[i] = make_double2(0.0, 0.0);
            if (done[r]) continue;
            const double2* Hr = H.data() + (size_t)r * (m + 1) * m;
            const double2* gr = gm.data() + (size_t)r * (m + 1);
            for (int i = maxIt[r] - 1; i >= 0; i--) {
                double2 e = gr[i];
                for (int jj = i + 1; jj < maxIt[r]; jj++) e = e - cmul(Hr[(size_t)i * m + jj], cf[jj]);
                cf[i] = cdiv(e, Hr[(size_t)i * m + i]);
            }
        }
        DDAMG_CUDA_TRY(cudaMemcpyAsync(h->dcoef, coef, sizeof(double2) * R * m, cudaMemcpyHostToDevice, s));
        launch_multiaxpy<V>(s, K.Z, Rn, n, m, h->dcoef, x, n, n, R, +1.0);
        A(x, K.w, R);
        launch_sub<V>(s, b, K.w, K.r, Rn);
        launch_norm2<V>(s, K.r, n, n, R, h->dpart, h->dn);
        DDAMG_CUDA_TRY(cudaMemcpyAsync(hn_pin, h->dn, sizeof(double) * R, cudaMemcpyDeviceToHost, s));
        sync(h);
        for (int r = 0; r < R; r++) {
            if (done[r]) continue;
            err[r] = std::sqrt(hn_pin[r]);
            if (!(err[r] == err[r])) throw ParamFailure{"NaN residual"};
            if (err[r] < tol * norm_b[r]) {
                ret[r] = k * m + maxIt[r];
                done[r] = 1;
            }
        }
    }
    for (int r = 0; r < R; r++) {
        if (iters) iters[r] = (norm_b[r] == 0.0) ? 0 : ret[r];
        if (rel) rel[r] = norm_b[r] > 0 ? err[r] / norm_b[r] : 0.0;
    }
}

// ------------------------------------------------------------------ FGMRES (device driven)
// While h->capturing, h->s records into a graph that replaces the host loop above: the loops become
// conditional nodes whose conditions the control kernels of kernels_fgmres.cu set.  Recording is split
// into segments: before a conditional node is added the capture is ended (its dependency set kept),
// the node's body is recorded on the same stream, and the capture then resumes after the node.  Each
// segment's kernels are counted against the body it belongs to, so the launches a solve ran follow
// from the bodies' run counters.
struct CapPoint {
    std::vector<cudaGraphNode_t> deps;
    cudaGraph_t graph;
};
static CapPoint cap_pause(ddamg_handle* h) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    DDAMG_CUDA_TRY(cudaStreamGetCaptureInfo(h->s, &st, nullptr, &g, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) throw CudaFailure{};
    CapPoint p{std::vector<cudaGraphNode_t>(deps, deps + nd), g};
    cudaGraph_t out = nullptr;
    DDAMG_CUDA_TRY(cudaStreamEndCapture(h->s, &out));
    (*h->cap_bodies)[h->cap_cur].kernels += g_launches - h->cap_mark;
    return p;
}
static void cap_begin(ddamg_handle* h, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, int body) {
    DDAMG_CUDA_TRY(cudaStreamBeginCaptureToGraph(h->s, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                                 cudaStreamCaptureModeRelaxed));
    h->cap_cur = body;
    h->cap_mark = g_launches;
}
static int cap_new_body(ddamg_handle* h, int level, int kind) {
    h->cap_bodies->push_back({level, kind, 0});
    return (int)h->cap_bodies->size() - 1;
}
static cudaGraphConditionalHandle cap_handle(ddamg_handle* h) {
    cudaGraphConditionalHandle hc;
    DDAMG_CUDA_TRY(cudaGraphConditionalHandleCreate(&hc, h->cap_top, 0, 0));
    return hc;
}
// ends the current segment, adds a conditional node after it (a while node, an if node, or with two
// bodies an if/else node) and records each body into its graph as a new body of (level, kind); the
// capture resumes after the node
static void cap_conditional(ddamg_handle* h, cudaGraphConditionalHandle hc, cudaGraphConditionalNodeType type,
                            int level, const std::vector<std::pair<int, std::function<void()>>>& bodies) {
    const int cur = h->cap_cur;
    CapPoint p = cap_pause(h);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hc;
    np.conditional.type = type;
    np.conditional.size = (unsigned)bodies.size();
    cudaGraphNode_t node;
    DDAMG_CUDA_TRY(cudaGraphAddNode(&node, p.graph, p.deps.empty() ? nullptr : p.deps.data(), p.deps.size(), &np));
    for (size_t k = 0; k < bodies.size(); k++) {
        cap_begin(h, np.conditional.phGraph_out[k], {}, cap_new_body(h, level, bodies[k].first));
        bodies[k].second();
        cap_pause(h);
    }
    cap_begin(h, p.graph, {node}, cur);
}

// FGMRES::fgmres as fgmres_host computes it, recorded into the graph under construction.  M(in, out, R,
// first): out = M in with in and out fixed buffers; first = restart 0 (the K-cycle starts from zero
// there and from the previous Z_j after a restart), `select` says whether the two differ.  With select
// each restart picks one of two recorded Arnoldi loops through an if/else node (one conditional
// evaluation per restart instead of one per step: an if node costs about 6.5 us on the device, a
// while iteration about 3.5 us).
template <typename V>
static void fgmres_dev(ddamg_handle* h, int lvl, long n, int R, int m, int restarts, double tol,
                       const std::function<void(const V*, V*, int)>& A,
                       const std::function<void(const V*, V*, int, bool)>& M, bool select, const V* b, const V* x0,
                       bool x0_zero, V* x, Krylov<V> K, V* vin, V* zf) {
    cudaStream_t s = h->s;
    const long Rn = (long)R * n;
    const FgDev& f = h->lv[lvl].fg;
    const int* jdev = f.ctl + kFgJ;
    if (x0_zero) DDAMG_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(V) * Rn, s));
    else if (x0 != x) DDAMG_CUDA_TRY(cudaMemcpyAsync(x, x0, sizeof(V) * Rn, cudaMemcpyDeviceToDevice, s));
    DDAMG_CUDA_TRY(cudaMemsetAsync(K.Z, 0, sizeof(V) * Rn * m, s));
    if (x0_zero) DDAMG_CUDA_TRY(cudaMemcpyAsync(K.r, b, sizeof(V) * Rn, cudaMemcpyDeviceToDevice, s));
    else {
        A(x, K.w, R);
        launch_sub<V>(s, b, K.w, K.r, Rn);
    }
    launch_norm2<V>(s, b, n, n, R, h->dpart, f.nrm);
    launch_norm2<V>(s, K.r, n, n, R, h->dpart, f.nrm + R);
    const cudaGraphConditionalHandle hc_outer = cap_handle(h), hc_in0 = cap_handle(h);
    cudaGraphConditionalHandle hc_in1{}, hc_sel{};
    if (select) {
        hc_in1 = cap_handle(h);
        hc_sel = cap_handle(h);
    }
    // one Arnoldi step; `later`: a K-cycle restart after the first, whose preconditioner starts from the
    // previous restart's Z_j
    auto step = [&](bool later, cudaGraphConditionalHandle hc, int counter) {
        launch_slot_copy<V, V>(s, K.Vb, vin, Rn, jdev, 0, Rn);
        if (later) launch_slot_copy<V, V>(s, K.Z, zf, Rn, jdev, 0, Rn);
        M(vin, zf, R, !later);
        launch_slot_copy<V, V>(s, zf, K.Z, Rn, jdev, 1, Rn);
        A(zf, K.w, R);
        double2* d1 = f.dots;
        double2* d2 = f.dots + (long)R * (m + 1);
        launch_multidot_dev<V>(s, K.Vb, Rn, n, m, jdev, m + 1, K.w, n, n, R, h->dpart, d1);
        launch_multiaxpy_dev<V>(s, K.Vb, Rn, n, jdev, d1, m + 1, K.w, n, n, R);
        launch_multidot_dev<V>(s, K.Vb, Rn, n, m, jdev, m + 1, K.w, n, n, R, h->dpart, d2);
        launch_multiaxpy_dev<V>(s, K.Vb, Rn, n, jdev, d2, m + 1, K.w, n, n, R);
        launch_norm2<V>(s, K.w, n, n, R, h->dpart, f.nrm);
        launch_fg_arnoldi(s, f, R, m, tol, hc, counter);
        launch_scale_slot<V>(s, f.alpha, K.w, K.Vb, Rn, jdev, n, R);  // V_{j+1}
    };
    launch_fg_start(s, f, R, m, restarts, hc_outer);
    cap_conditional(h, hc_outer, cudaGraphCondTypeWhile, lvl, {{kFgRunsOuter, [&]() {
        launch_fg_restart(s, f, R, m, hc_in0, hc_in1, hc_sel, select ? 1 : 0);
        launch_scale<V>(s, f.alpha, K.r, K.Vb, n, R);  // V_0 = r / beta
        if (!select) {
            cap_conditional(h, hc_in0, cudaGraphCondTypeWhile, lvl,
                            {{kFgRunsInner, [&]() { step(false, hc_in0, kFgRunsInner); }}});
        } else {
            // the restart's loop is chosen once per restart, not per step: an if/else node over two loops
            cap_conditional(h, hc_sel, cudaGraphCondTypeIf, lvl,
                            {{kFgRunsFirst,
                              [&]() {
                                  cap_conditional(h, hc_in0, cudaGraphCondTypeWhile, lvl,
                                                  {{kFgRunsInner, [&]() { step(false, hc_in0, kFgRunsInner); }}});
                              }},
                             {kFgRunsLater, [&]() {
                                  cap_conditional(
                                      h, hc_in1, cudaGraphCondTypeWhile, lvl,
                                      {{kFgRunsInnerLater, [&]() { step(true, hc_in1, kFgRunsInnerLater); }}});
                              }}});
        }
        launch_fg_backsub(s, f, R, m);
        launch_multiaxpy<V>(s, K.Z, Rn, n, m, f.coef, x, n, n, R, +1.0);
        A(x, K.w, R);
        launch_sub<V>(s, b, K.w, K.r, Rn);
        launch_norm2<V>(s, K.r, n, n, R, h->dpart, f.nrm);
        launch_fg_restart_end(s, f, R, m, restarts, tol, hc_outer);
    }}});
}

// ------------------------------------------------------------------ cycles
static void cycle(ddamg_handle* h, int l, const void* eta, void* psi, bool psi_zero, int kind, int R);

// the next level's input: restrict r (level l, type V) into level l+1's eta (its own type)
template <typename V> static void* restrict_into_next(ddamg_handle* h, int l, const V* r, int R) {
    LevelData& D = h->lv[l];
    LevelData& N = h->lv[l + 1];
    const bool cur32 = std::is_same<V, float2>::value;
    if (N.fp32 == cur32) {
        V* out = B<V>(N).eta;
        launch_restrict<V>(h->s, D.g, B<V>(D).tv, r, out, R);
        return out;
    }
    // only float -> double happens (mixed: FP32 level above the FP64 coarsest level)
    launch_restrict<V>(h->s, D.g, B<V>(D).tv, r, reinterpret_cast<V*>(N.f.xfer), R);
    launch_convert<float2, double2>(h->s, N.f.xfer, N.d.eta, N.g.size() * R);
    return N.d.eta;
}
template <typename V> static void prolong_from_next(ddamg_handle* h, int l, const void* psi_next, V* psi, int R) {
    LevelData& D = h->lv[l];
    LevelData& N = h->lv[l + 1];
    const bool cur32 = std::is_same<V, float2>::value;
    if (N.fp32 == cur32) {
        launch_prolong<V>(h->s, D.g, B<V>(D).tv, static_cast<const V*>(psi_next), psi, 1, R);
        return;
    }
    launch_convert<double2, float2>(h->s, static_cast<const double2*>(psi_next), N.f.xfer, N.g.size() * R);
    launch_prolong<V>(h->s, D.g, B<V>(D).tv, reinterpret_cast<const V*>(N.f.xfer), psi, 1, R);
}
static void* next_psi(ddamg_handle* h, int l) {
    LevelData& N = h->lv[l + 1];
    return N.fp32 ? (void*)N.f.psi : (void*)N.d.psi;
}

// AlgebraicMG::v_cycle / k_cycle (src/amg.cpp:64-174) on R vectors of level l
template <typename V>
static void cycle_t(ddamg_handle* h, int l, const V* eta, V* psi, bool psi_zero, int kind, int R) {
    const ddamg_params& p = h->p;
    if (l == h->L - 1) {
        coarse_solve_batch(h, reinterpret_cast<const double2*>(eta), reinterpret_cast<double2*>(psi), R);
        return;
    }
    LevelData& D = h->lv[l];
    const long n = D.g.size();
    if (psi_zero) DDAMG_CUDA_TRY(cudaMemsetAsync(psi, 0, sizeof(V) * n * R, h->s));
    bool zero = psi_zero;
    if (p.nu1 > 0) {
        sap_t<V>(h, l, eta, psi, p.nu1, p.smoother_tolerance, zero, R, false);
        zero = false;
    }
    V* r = B<V>(D).r;
    // r = eta - D psi (psi == 0 gives r = eta exactly)
    const V* rin = eta;
    if (!zero) {
        level_op<V>(h, l, psi, r, eta, R);
        rin = r;
    }
    void* en = restrict_into_next<V>(h, l, rin, R);
    void* pn = next_psi(h, l);
    LevelData& N = h->lv[l + 1];
    if (kind == DDAMG_CYCLE_V) {
        cycle(h, l + 1, en, pn, true, kind, R);
    } else {
        // FGMRES_k_cycle at level l+1 (include/amg.h:16-94), x0 = rhs
        const long nn = N.g.size();
        auto run = [&](auto tag) {
            typedef decltype(tag) W;
            LevelBufs<W>& nb = B<W>(N);
            std::function<void(const W*, W*, int)> A = [h, l](const W* in, W* out, int RR) {
                level_op<W>(h, l + 1, in, out, nullptr, RR);
            };
            std::function<void(const W*, W*, int, int)> M = [h, l](const W* in, W* out, int RR, int restart) {
                cycle(h, l + 1, in, out, restart == 0, DDAMG_CYCLE_K, RR);
            };
            Krylov<W> K{nb.kV, nb.kZ, nb.kw, nb.kr};
            if (h->capturing) {
                std::function<void(const W*, W*, int, bool)> Md = [h, l](const W* in, W* out, int RR, bool first) {
                    cycle(h, l + 1, in, out, first, DDAMG_CYCLE_K, RR);
                };
                fgmres_dev<W>(h, l + 1, nn, R, p.kcycle_restart_length, p.kcycle_restarts, p.kcycle_tolerance, A, Md,
                              true, static_cast<const W*>(en), static_cast<const W*>(en), false, static_cast<W*>(pn), K,
                              nb.kin, nb.kzf);
                return;
            }
            fgmres_host<W>(h, nn, R, p.kcycle_restart_length, p.kcycle_restarts, p.kcycle_tolerance, A, &M,
                           static_cast<const W*>(en), static_cast<const W*>(en), false, static_cast<W*>(pn), K,
                           nullptr, nullptr);
        };
        if (N.fp32) run(float2{});
        else run(double2{});
    }
    prolong_from_next<V>(h, l, pn, psi, R);
    if (p.nu2 > 0) sap_t<V>(h, l, eta, psi, p.nu2, p.smoother_tolerance, false, R, false);
}
// (the coarsest solves record a bounded wait that gave up in their status words; the callers of the
// cycle check them once the whole solve is done: check_coarse_status)
static void cycle(ddamg_handle* h, int l, const void* eta, void* psi, bool psi_zero, int kind, int R) {
    if (h->lv[l].fp32)
        cycle_t<float2>(h, l, static_cast<const float2*>(eta), static_cast<float2*>(psi), psi_zero, kind, R);
    else cycle_t<double2>(h, l, static_cast<const double2*>(eta), static_cast<double2*>(psi), psi_zero, kind, R);
}

// One cycle on the level-0 buffers eta -> psi (fixed addresses, so a captured graph stays valid
// across calls and set-ups).  V-cycles replay a CUDA graph per batch width: the first application
// of a width runs directly, the second is captured and every later one replays it.
static void level0_cycle(ddamg_handle* h, int R) {
    LevelData& D = h->lv[0];
    auto direct = [&]() {
        if (D.fp32) cycle(h, 0, D.f.eta, D.f.psi, true, h->p.cycle, R);
        else cycle(h, 0, D.d.eta, D.d.psi, true, h->p.cycle, R);
    };
    if (!h->p.cuda_graphs || h->graphs_off || h->p.cycle != DDAMG_CYCLE_V || h->prof || h->capturing) {
        direct();
        return;
    }
    auto it = h->graphs.find(R);
    if (it != h->graphs.end()) {
        DDAMG_CUDA_TRY(cudaGraphLaunch(it->second.exec, h->s));
        g_launches += it->second.kernels;
        return;
    }
    if (!h->graph_warm.count(R)) {
        direct();
        h->graph_warm.insert(R);
        return;
    }
    const long long launches0 = g_launches;
    cudaGraph_t graph = nullptr;
    bool failed = cudaStreamBeginCapture(h->s, cudaStreamCaptureModeRelaxed) != cudaSuccess;
    if (!failed) {
        try {
            direct();
        } catch (...) {
            failed = true;
        }
        if (cudaStreamEndCapture(h->s, &graph) != cudaSuccess || !graph) failed = true;
    }
    cudaGraphExec_t exec = nullptr;
    if (!failed && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) failed = true;
    if (graph) cudaGraphDestroy(graph);
    const long long kernels = g_launches - launches0;  // recorded, not yet run
    g_launches -= kernels;
    if (failed) {  // this configuration cannot be captured: keep launching directly
        cudaGetLastError();
        h->graphs_off = true;
        h->tune_log += "cycle graph capture failed: launching kernels directly\n";
        direct();
        return;
    }
    h->graphs[R] = {exec, kernels};
    h->tune_log += "cycle graph rhs " + std::to_string(R) + ": " + std::to_string(kernels) + " kernels\n";
    DDAMG_CUDA_TRY(cudaGraphLaunch(exec, h->s));
    g_launches += kernels;
}

// the outer preconditioner (FGMRES_AMG_*::preconditioner, include/amg.h:240-269): zero, one cycle
static void outer_prec(ddamg_handle* h, const double2* in, double2* out, int R) {
    LevelData& D = h->lv[0];
    const long n = D.g.size() * R;
    if (D.fp32) launch_convert<double2, float2>(h->s, in, D.f.eta, n);
    else DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, in, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->s));
    level0_cycle(h, R);
    if (D.fp32) launch_convert<float2, double2>(h->s, D.f.psi, out, n);
    else DDAMG_CUDA_TRY(cudaMemcpyAsync(out, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->s));
}

// ------------------------------------------------------------------ setup
static void make_fp32_copies(ddamg_handle* h) {
    for (int l = 0; l < h->L; l++) {
        LevelData& D = h->lv[l];
        if (!D.fp32) continue;
        if (l == 0) launch_convert<double2, float2>(h->s, D.d.U, D.f.U, 2L * D.g.sites);
        else launch_convert<double2, float2>(h->s, D.d.links, D.f.links, (long)D.g.sites * 5 * D.g.dof * D.g.dof);
        if (D.tc) launch_pack_tc_links(h->s, D.g, D.f.links, D.tcw.tiles);
        if (l < h->L - 1) launch_convert<double2, float2>(h->s, D.d.tv, D.f.tv, (long)D.g.ntest * D.g.size());
    }
}

static long setup_random_count(const ddamg_handle* h) {
    long n = (long)h->lv[0].g.ntest * h->lv[0].g.size();
    for (int l = 1; l < h->L - 1; l++) {
        int extra = h->lv[l].g.ntest - h->lv[l - 1].g.ntest;
        if (extra > 0) n += (long)extra * h->lv[l].g.size();
    }
    return n;
}

// The setup's smoothing at a coarse level: SAP with right-hand side 0 on every test vector
// (src/amg.cpp:49-52).  The vectors are independent, so groups of the CUDA-core sweep's tuned width
// run their sweeps and residual updates on separate streams, and one group's CTAs fill the SMs that
// the last wave of another group's sweep leaves idle.  With v = 0 the reference's test
// ||r|| < tol ||v|| never passes, so every vector takes exactly nu iterations and no norms are
// needed, as in sap_t.  Returns false (nothing done) where the single-stream path applies.
template <typename V>
static bool sap_setup_split(ddamg_handle* h, int l, const V* v, V* x, int nu, int nrhs) {
    if (l == 0 || h->prof || nrhs < 2) return false;
    LevelData& D = h->lv[l];
    const Geom& g = D.g;
    const long n = g.size();
    V* r = B<V>(D).r;
    SapArgs a{h->p.sap_gmres_restart_length, h->p.sap_gmres_restarts, h->p.sap_gmres_tolerance, h->p.m0, D.red,
              D.nred, D.done};
    DDAMG_CUDA_TRY(cudaMemsetAsync(D.done, 0, sizeof(int) * nrhs, h->s));
    // r = v - D x for every vector (CUDA cores: test-vector quality); once the sweep variant is tuned, the
    // groups' first red sweeps form it themselves where the residual can be fused
    const int rkey = nrhs * 2 + (std::is_same<V, float2>::value ? 1 : 0);
    const bool pre_fuse = D.rb_choice.count(rkey) != 0 && D.rb_choice[rkey] % 4 == 1 && fusable_residual(g);
    if (!pre_fuse) level_op<V>(h, l, x, r, v, nrhs, false);
    const int var = rb_for<V>(h, l, r, a, nrhs);  // tuned on first use on red sweeps (times into scratch, syncs)
    const int rb = var / 4;
    const int G = nrhs / rb;
    // the groups of one Schwarz block share its links through L2 only while they run side by side,
    // which one launch guarantees (block-major CTA order) and separate streams do not: split only when
    // one colour's links fit in L2 (128x128 sites at dof 32, 671 MB per colour, lost 38 % of its setup)
    const double colour_link_bytes = 0.5 * (double)g.sites * 5 * g.dof * g.dof * sizeof(V);
    if (G < 2 || G * rb != nrhs || colour_link_bytes > 100e6) {  // one stream: the plain sweep loop
        if (pre_fuse) level_op<V>(h, l, x, r, v, nrhs, false);
        for (int it = 0; it < nu; it++)
            for (int colour = 0; colour < 2; colour++) {
                a.blocks = colour == 0 ? D.red : D.black;
                a.nblocks = colour == 0 ? D.nred : D.nblack;
                launch_sap_sweep_coarse<V>(h->s, g, B<V>(D).links, r, x, a, nrhs, var);
                if (!(colour == 1 && it == nu - 1)) level_op<V>(h, l, x, r, v, nrhs, false);
            }
        return true;
    }
    while ((int)h->setup_s.size() < G - 1) {
        cudaStream_t q;
        cudaEvent_t e;
        DDAMG_CUDA_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        DDAMG_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->setup_s.push_back(q);
        h->setup_ev.push_back(e);
    }
    DDAMG_CUDA_TRY(cudaEventRecord(h->fork_ev, h->s));
    for (int k = 1; k < G; k++) DDAMG_CUDA_TRY(cudaStreamWaitEvent(h->setup_s[k - 1], h->fork_ev, 0));
    for (int k = 0; k < G; k++) {
        cudaStream_t st = k == 0 ? h->s : h->setup_s[k - 1];
        const long off = (long)k * rb * n;
        SapArgs ak = a;
        ak.done = D.done + k * rb;
        const bool fuse = var % 4 == 1 && fusable_residual(g);
        for (int it = 0; it < nu; it++)
            for (int colour = 0; colour < 2; colour++) {
                ak.blocks = colour == 0 ? D.red : D.black;
                ak.nblocks = colour == 0 ? D.nred : D.nblack;
                ak.vres = ((colour == 1 && fuse) || (colour == 0 && it == 0 && pre_fuse))
                              ? static_cast<const void*>(v + off)
                              : nullptr;
                launch_sap_sweep_coarse<V>(st, g, B<V>(D).links, r + off, x + off, ak, rb, var);
                if (colour == 0 && fuse) continue;  // the black sweep forms its blocks' residuals
                if (!(colour == 1 && it == nu - 1))
                    launch_coarse_op<V>(st, B<V>(D).links, x + off, r + off, v + off, g.Nx, g.Nt, g.dof, h->p.m0, rb);
            }
    }
    for (int k = 1; k < G; k++) {
        DDAMG_CUDA_TRY(cudaEventRecord(h->setup_ev[k - 1], h->setup_s[k - 1]));
        DDAMG_CUDA_TRY(cudaStreamWaitEvent(h->s, h->setup_ev[k - 1], 0));
    }
    return true;
}

// AlgebraicMG::setUpPhase (src/amg.cpp:4-56).  rnd: device stream of random complex values
// (or null with a seed: drawn on the device with the same counter RNG as the oracle).
static void setup(ddamg_handle* h, const double2* rnd_host, uint64_t seed) {
    if (!h->gauge) throw ParamFailure{"load the gauge field before the setup"};
    cudaStream_t s = h->s;
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev0, s));
    long pos = 0;
    auto draw = [&](double2* dst, long count) {
        if (rnd_host)
            DDAMG_CUDA_TRY(cudaMemcpyAsync(dst, rnd_host + pos, sizeof(double2) * count, cudaMemcpyHostToDevice, s));
        else launch_fill_uniform(s, dst, count, seed, pos);
        pos += count;
    };
    LevelData& L0 = h->lv[0];
    draw(L0.d.tv, (long)L0.g.ntest * L0.g.size());
    for (int l = 1; l < h->L - 1; l++) {
        LevelData& D = h->lv[l];
        LevelData& P = h->lv[l - 1];
        const int from_prev = std::min(D.g.ntest, P.g.ntest);
        // tvec_l[cc] = P^dagger tvec_{l-1}[cc] before level l-1 is smoothed (src/amg.cpp:25-41)
        launch_restrict<double2>(s, P.g, P.d.tv, P.d.tv, D.d.tv, from_prev);
        for (int cc = from_prev; cc < D.g.ntest; cc++) draw(D.d.tv + (long)cc * D.g.size(), D.g.size());
    }
    for (int l = 0; l < h->L - 1; l++) {
        LevelData& D = h->lv[l];
        const long n = D.g.size();
        const int nv = D.g.ntest;
        const int nu = h->p.sap_test_vectors_iterations;
        // SAP(rhs = 0, tvec, nu = SAP_test_vectors_iterations) on all test vectors at once
        // (src/amg.cpp:45-52), in the level's working precision: in mixed precision the smoother is FP32
        // (its operator converted from this level's FP64 links, built just before by level l-1), and the
        // smoothed vectors are promoted to FP64 for the orthonormalisation and the coarse links
        if (D.fp32) {
            if (l > 0) {
                launch_convert<double2, float2>(s, D.d.links, D.f.links, (long)D.g.sites * 5 * D.g.dof * D.g.dof);
                if (D.tc) launch_pack_tc_links(s, D.g, D.f.links, D.tcw.tiles);
            }
            launch_convert<double2, float2>(s, D.d.tv, D.f.tv, n * nv);
            DDAMG_CUDA_TRY(cudaMemsetAsync(D.f.eta, 0, sizeof(float2) * n * nv, s));
            // CUDA cores only: TF32 block operators would coarsen the test vectors
            if (!sap_setup_split<float2>(h, l, D.f.eta, D.f.tv, nu, nv))
                sap_t<float2>(h, l, D.f.eta, D.f.tv, nu, 1e-10, false, nv, false, nullptr, false);
            launch_convert<float2, double2>(s, D.f.tv, D.d.tv, n * nv);
        } else {
            DDAMG_CUDA_TRY(cudaMemsetAsync(D.d.eta, 0, sizeof(double2) * n * nv, s));
            if (!sap_setup_split<double2>(h, l, D.d.eta, D.d.tv, nu, nv))
                sap_t<double2>(h, l, D.d.eta, D.d.tv, nu, 1e-10, false, nv, false);
        }
        {
            ProfScope ps(h, 3, l);
            launch_orthonormalize(s, D.g, D.d.tv);
        }
        ProfScope ps(h, 4, l);
        launch_build_coarse_links(s, D.g, D.d.U, D.d.links, D.d.tv, h->lv[l + 1].d.links);
    }
    make_fp32_copies(h);
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, s));
    sync(h);
    float ms = 0;
    DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->last_setup_s = ms * 1e-3;
    h->setup_done = true;
    tune_coarse(h);  // once per handle, outside the setup's timed region
}

// ------------------------------------------------------------------ solve
// The device-driven solve of R right-hand sides from h->ob into h->ox: built once per width (false if
// this runtime cannot record or instantiate it; the host-driven loop is used from then on)
static bool solve_graph(ddamg_handle* h, int R, const std::function<void(const double2*, double2*, int)>& A,
                        const std::function<void(const double2*, double2*, int, bool)>& M, Krylov<double2> K) {
    if (h->solve_graphs.count(R)) return true;
    const ddamg_params& p = h->p;
    const long n = h->lv[0].g.size();
    const long long l0 = g_launches;
    ddamg_handle::SolveGraph sg{nullptr, {}};
    cudaGraph_t top = nullptr;
    bool ok = cudaGraphCreate(&top, 0) == cudaSuccess;
    if (ok) {
        h->capturing = true;
        h->cap_top = top;
        h->cap_bodies = &sg.bodies;
        try {
            cap_begin(h, top, {}, cap_new_body(h, 0, 0));
            for (int l = 0; l < h->L; l++)
                if (h->lv[l].fg.ctl)
                    DDAMG_CUDA_TRY(cudaMemsetAsync(h->lv[l].fg.ctl + kFgRunsOuter, 0,
                                               (kFgCtlWords - kFgRunsOuter) * sizeof(int), h->s));
            fgmres_dev<double2>(h, 0, n, R, p.fgmres_restart_length, p.fgmres_restarts, p.fgmres_tolerance, A, M,
                                false, h->ob, nullptr, true, h->ox, K, h->ovin, h->ozf);
            cap_pause(h);
        } catch (...) {
            ok = false;
            cudaStreamCaptureStatus st;
            if (cudaStreamIsCapturing(h->s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(h->s, &junk);
                if (junk && junk != top) cudaGraphDestroy(junk);
            }
        }
        h->capturing = false;
        h->cap_bodies = nullptr;
        h->cap_top = nullptr;
    }
    if (ok && cudaGraphInstantiate(&sg.exec, top, 0) != cudaSuccess) ok = false;
    if (ok && cudaGraphUpload(sg.exec, h->s) != cudaSuccess) ok = false;
    if (top) cudaGraphDestroy(top);
    g_launches = l0;  // recorded, not run
    if (!ok) {
        cudaGetLastError();
        if (sg.exec) cudaGraphExecDestroy(sg.exec);
        h->solve_graphs_off = true;
        h->tune_log += "solve graph for rhs " + std::to_string(R) + ": not supported here, host-driven FGMRES\n";
        return false;
    }
    long long kernels = 0;
    for (const auto& bd : sg.bodies) kernels += bd.kernels;
    h->tune_log += "solve graph rhs " + std::to_string(R) + ": " + std::to_string(sg.bodies.size()) + " bodies, " +
                   std::to_string(kernels) + " kernels recorded (FGMRES loops on the device)\n";
    h->solve_graphs[R] = sg;
    return true;
}
// after the solve graph's launch: its per-rhs results and the bodies' run counters (launch count)
static void read_solve_graph(ddamg_handle* h, int R, std::vector<int>& it, std::vector<double>& rel) {
    const ddamg_handle::SolveGraph& sg = h->solve_graphs.at(R);
    std::vector<std::array<int, kFgCtlWords>> ctl(h->L);
    for (int l = 0; l < h->L; l++)
        if (h->lv[l].fg.ctl)
            DDAMG_CUDA_TRY(cudaMemcpyAsync(ctl[l].data(), h->lv[l].fg.ctl, sizeof(int) * kFgCtlWords,
                                           cudaMemcpyDeviceToHost, h->s));
    const FgDev& f = h->lv[0].fg;
    std::vector<int> ret(R);
    std::vector<double> err(R), nb(R);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(ret.data(), f.ret, sizeof(int) * R, cudaMemcpyDeviceToHost, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(err.data(), f.err, sizeof(double) * R, cudaMemcpyDeviceToHost, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(nb.data(), f.norm_b, sizeof(double) * R, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    long long launched = 0;
    for (const auto& bd : sg.bodies) launched += bd.kernels * (bd.kind == 0 ? 1 : ctl[bd.level][bd.kind]);
    g_launches += launched;
    for (int l = 0; l < h->L; l++)
        if (h->lv[l].fg.ctl && ctl[l][kFgNan]) throw NanFailure{"NaN in the right-hand side or the Krylov basis"};
    for (int r = 0; r < R; r++) {
        it[r] = nb[r] == 0.0 ? 0 : ret[r];
        rel[r] = nb[r] > 0 ? err[r] / nb[r] : 0.0;
    }
}

static ddamg_status solve_device(ddamg_handle* h, const double2* b, double2* x, int nrhs, ddamg_solve_info* info) {
    if (!h->setup_done) throw ParamFailure{"run the setup before solving"};
    const ddamg_params& p = h->p;
    const long n = h->lv[0].g.size();
    const Geom& g0 = h->lv[0].g;
    std::function<void(const double2*, double2*, int)> A = [h, &g0](const double2* in, double2* out, int R) {
        launch_wilson<double2>(h->s, h->lv[0].d.U, in, out, nullptr, g0.Nx, g0.Nt, h->p.m0, 0, R);
    };
    std::function<void(const double2*, double2*, int, int)> M = [h](const double2* in, double2* out, int R, int) {
        outer_prec(h, in, out, R);
    };
    Krylov<double2> K{h->oV, h->oZ, h->ow, h->orr};
    std::vector<int> it(nrhs);
    std::vector<double> rel(nrhs);
    const bool graph = p.cuda_graphs && !h->prof && !h->solve_graphs_off;
    bool use_graph = false;
    if (graph && h->solve_warm.count(nrhs)) {  // built (host work, once per width) before the timed region
        std::function<void(const double2*, double2*, int, bool)> Md = [h](const double2* in, double2* out, int R,
                                                                          bool) { outer_prec(h, in, out, R); };
        use_graph = solve_graph(h, nrhs, A, Md, K);
    }
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev0, h->s));
    if (use_graph) {
        if (b != h->ob)
            DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ob, b, sizeof(double2) * n * nrhs, cudaMemcpyDeviceToDevice, h->s));
        DDAMG_CUDA_TRY(cudaGraphLaunch(h->solve_graphs.at(nrhs).exec, h->s));
        if (x != h->ox)
            DDAMG_CUDA_TRY(cudaMemcpyAsync(x, h->ox, sizeof(double2) * n * nrhs, cudaMemcpyDeviceToDevice, h->s));
        DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, h->s));
        read_solve_graph(h, nrhs, it, rel);
    } else {
        fgmres_host<double2>(h, n, nrhs, p.fgmres_restart_length, p.fgmres_restarts, p.fgmres_tolerance, A, &M, b,
                             nullptr, true, x, K, it.data(), rel.data());
        if (graph) h->solve_warm.insert(nrhs);
        DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, h->s));
    }
    check_coarse_status(h, nullptr);
    check_tc_status(h);
    sync(h);
    float ms = 0;
    DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    ddamg_status st = DDAMG_OK;
    h->counts[p.cycle == DDAMG_CYCLE_K ? DDAMG_COUNT_KCYCLE : DDAMG_COUNT_VCYCLE] = *std::max_element(it.begin(), it.end());
    for (int r = 0; r < nrhs; r++) {
        const bool conv = rel[r] < p.fgmres_tolerance;
        if (!conv) st = DDAMG_NOT_CONVERGED;
        if (info) {
            info[r].iterations = it[r];
            info[r].converged = conv ? 1 : 0;
            info[r].rel_residual = rel[r];
            info[r].setup_seconds = h->last_setup_s;
            info[r].solve_seconds = ms * 1e-3;
        }
    }
    return st;
}

}  // namespace ddamg

// ====================================================================== C API
using namespace ddamg;

#define API_BEGIN try {
#define API_END                                                                                  \
    }                                                                                            \
    catch (const ParamFailure& e) {                                                              \
        set_error(e.msg);                                                                        \
        return DDAMG_ERR_BAD_PARAM;                                                              \
    }                                                                                            \
    catch (const CudaFailure&) {                                                                 \
        return DDAMG_ERR_CUDA;                                                                   \
    }                                                                                            \
    catch (const TimeoutFailure&) {                                                              \
        set_error("a bounded device-side wait gave up (grid barrier timeout)");                  \
        return DDAMG_ERR_DEVICE_TIMEOUT;                                                         \
    }                                                                                            \
    catch (const NanFailure& e) {                                                                \
        set_error(e.msg);                                                                        \
        return DDAMG_ERR_NAN;                                                                    \
    }                                                                                            \
    catch (const NotConvergedFailure& e) {                                                       \
        set_error(e.msg);                                                                        \
        return DDAMG_NOT_CONVERGED;                                                              \
    }                                                                                            \
    catch (const IoFailure& e) {                                                                 \
        set_error(e.msg);                                                                        \
        return DDAMG_ERR_IO;                                                                     \
    }                                                                                            \
    catch (const std::exception& e) {                                                            \
        set_error(e.what());                                                                     \
        return DDAMG_ERR_STATE;                                                                  \
    }                                                                                            \
    return DDAMG_OK;

#define CHECK_HANDLE(h)                                                                          \
    if (!(h)) {                                                                                  \
        set_error("null handle");                                                                \
        return DDAMG_ERR_BAD_PARAM;                                                              \
    }                                                                                            \
    DDAMG_CUDA_TRY(cudaSetDevice((h)->p.device));

static void need_level(ddamg_handle* h, int l, bool allow_coarsest) {
    if (l < 0 || l >= h->L || (!allow_coarsest && l == h->L - 1)) throw ParamFailure{"level out of range"};
}
static void need_setup(ddamg_handle* h) {
    if (!h->setup_done) throw ParamFailure{"run the setup first"};
}

extern "C" {

const char* ddamg_last_error(void) { return t_last_error.c_str(); }

ddamg_status ddamg_params_default(ddamg_params* p) {
    if (!p) return DDAMG_ERR_BAD_PARAM;
    std::memset(p, 0, sizeof(*p));
    p->sap_gmres_restart_length = 5;
    p->sap_gmres_restarts = 5;
    p->sap_gmres_tolerance = 1e-3;
    p->sap_test_vectors_iterations = 4;
    p->coarse_gmres_restart_length = 400;
    p->coarse_gmres_restarts = 10;
    p->coarse_gmres_tolerance = 0.1;
    p->nu1 = 0;
    p->nu2 = 2;
    p->kcycle_restart_length = 5;
    p->kcycle_restarts = 2;
    p->kcycle_tolerance = 0.1;
    p->fgmres_restart_length = 20;
    p->fgmres_restarts = 50;
    p->fgmres_tolerance = 1e-10;
    p->smoother_tolerance = 1e-10;
    p->cycle = DDAMG_CYCLE_V;
    p->precision = DDAMG_PREC_DOUBLE;
    p->max_rhs = 1;
    p->device = 0;
    p->tensor_cores = 1;
    p->cuda_graphs = 1;
    p->coarse_barrier_polls = 1 << 24;
    p->coarse_kernel = 0;
    return DDAMG_OK;
}

ddamg_status ddamg_parse_params_file(const char* path, int levels, ddamg_params* p) {
    if (!path || !p) return DDAMG_ERR_BAD_PARAM;
    std::ifstream f(path);
    if (!f) {
        set_error(std::string("File ") + path + " not found");
        return DDAMG_ERR_IO;
    }
    int v[6], count = 0;
    while (f >> v[0] >> v[1] >> v[2] >> v[3] >> v[4] >> v[5]) {
        if (count >= DDAMG_MAX_LEVELS - 1) {
            set_error("too many rows in the parameters file");
            return DDAMG_ERR_BAD_PARAM;
        }
        for (int k = 0; k < 6; k++) p->rows[count][k] = v[k];
        count++;
    }
    if (!f.eof()) {
        set_error("malformed parameters file (expected 6 integers per row)");
        return DDAMG_ERR_BAD_PARAM;
    }
    if (count != levels - 1) {
        set_error("The number of levels in the inputs file does not match the number of levels assigned");
        return DDAMG_ERR_BAD_PARAM;
    }
    p->levels = levels;
    return DDAMG_OK;
}

ddamg_status ddamg_create(const ddamg_params* p, ddamg_t** out) {
    if (!p || !out) return DDAMG_ERR_BAD_PARAM;
    *out = nullptr;
    auto* h = new ddamg_handle();
    h->p = *p;
    try {
        DDAMG_CUDA_TRY(cudaSetDevice(p->device));
        build_geometry(h);
        DDAMG_CUDA_TRY(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
        DDAMG_CUDA_TRY(cudaEventCreate(&h->ev0));
        DDAMG_CUDA_TRY(cudaEventCreate(&h->ev1));
        allocate(h);
    } catch (const ParamFailure& e) {
        set_error(e.msg);
        ddamg_destroy(h);
        return DDAMG_ERR_BAD_PARAM;
    } catch (const CudaFailure&) {
        ddamg_destroy(h);
        return DDAMG_ERR_CUDA;
    }
    h->launches_at_create = g_launches;
    *out = h;
    return DDAMG_OK;
}

ddamg_status ddamg_destroy(ddamg_t* h) {
    if (!h) return DDAMG_OK;
    cudaSetDevice(h->p.device);
    if (h->s) cudaStreamSynchronize(h->s);
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second.exec);
    for (auto& kv : h->solve_graphs) cudaGraphExecDestroy(kv.second.exec);
    for (void* a : h->allocs) cudaFree(a);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : h->lane_ev) cudaEventDestroy(e);
    for (cudaStream_t q : h->lane_s) cudaStreamDestroy(q);
    for (cudaStream_t q : h->setup_s) cudaStreamDestroy(q);
    for (cudaEvent_t e : h->setup_ev) cudaEventDestroy(e);
    if (h->fork_ev) cudaEventDestroy(h->fork_ev);
    if (h->hpin) cudaFreeHost(h->hpin);
    if (h->hpin2) cudaFreeHost(h->hpin2);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
    return DDAMG_OK;
}

ddamg_status ddamg_get_stream(ddamg_t* h, void** stream) {
    CHECK_HANDLE(h);
    API_BEGIN
    *stream = (void*)h->s;
    API_END
}
ddamg_status ddamg_profile(ddamg_t* h, int enable) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (enable && !h->prof) {
        for (auto& row : h->prof_ms)
            for (double& v : row) v = 0;
        for (auto& row : h->prof_n)
            for (long long& v : row) v = 0;
    }
    if (!enable) prof_flush(h);
    h->prof = enable != 0;
    API_END
}
ddamg_status ddamg_profile_query(ddamg_t* h, int kind, int level, double* total_ms, long long* launches) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (kind < 0 || kind >= kProfKinds || level < 0 || level >= h->L) throw ParamFailure{"kind or level out of range"};
    prof_flush(h);
    if (total_ms) *total_ms = h->prof_ms[kind][level];
    if (launches) *launches = h->prof_n[kind][level];
    API_END
}
ddamg_status ddamg_autotune_report(ddamg_t* h, char* buf, int len) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!buf || len < 1) throw ParamFailure{"buffer required"};
    const std::string& t = h->tune_log;
    const int n = std::min<int>((int)t.size(), len - 1);
    std::memcpy(buf, t.data(), n);
    buf[n] = 0;
    API_END
}
ddamg_status ddamg_launch_count(ddamg_t* h, long long* count) {
    if (!count) return DDAMG_ERR_BAD_PARAM;
    *count = g_launches;
    (void)h;
    return DDAMG_OK;
}

ddamg_status ddamg_read_binary(const char* path, int Nx, int Nt, double* out) {
    if (!path || !out || Nx <= 0 || Nt <= 0) return DDAMG_ERR_BAD_PARAM;
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        set_error(std::string("File ") + path + " not found");
        return DDAMG_ERR_IO;
    }
    for (long i = 0; i < 2L * Nx * Nt; i++) {
        int32_t hdr[3];
        double re_im[2];
        f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
        f.read(reinterpret_cast<char*>(re_im), sizeof(re_im));
        if (!f) {
            set_error(std::string("short file ") + path);
            return DDAMG_ERR_IO;
        }
        out[2 * i] = re_im[0];
        out[2 * i + 1] = re_im[1];
    }
    return DDAMG_OK;
}
ddamg_status ddamg_from_halo(const double* halo, int Nx, int Nt, int dof, double* compact) {
    if (!halo || !compact || Nx <= 0 || Nt <= 0 || dof <= 0) {
        set_error("ddamg_from_halo: bad argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    for (int x = 1; x <= Nx; x++)
        for (int t = 1; t <= Nt; t++)
            for (int d = 0; d < dof; d++) {
                const long h = ((long)x * (Nt + 2) + t) * dof + d, c = ((long)(x - 1) * Nt + (t - 1)) * dof + d;
                compact[2 * c] = halo[2 * h];
                compact[2 * c + 1] = halo[2 * h + 1];
            }
    return DDAMG_OK;
}
ddamg_status ddamg_to_halo(const double* compact, int Nx, int Nt, int dof, double* halo) {
    if (!halo || !compact || Nx <= 0 || Nt <= 0 || dof <= 0) {
        set_error("ddamg_to_halo: bad argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    std::fill(halo, halo + 2L * (Nx + 2) * (Nt + 2) * dof, 0.0);
    for (int x = 1; x <= Nx; x++)
        for (int t = 1; t <= Nt; t++)
            for (int d = 0; d < dof; d++) {
                const long h = ((long)x * (Nt + 2) + t) * dof + d, c = ((long)(x - 1) * Nt + (t - 1)) * dof + d;
                halo[2 * h] = compact[2 * c];
                halo[2 * h + 1] = compact[2 * c + 1];
            }
    return DDAMG_OK;
}
ddamg_status ddamg_write_binary(const char* path, int Nx, int Nt, const double* field) {
    if (!path || !field || Nx <= 0 || Nt <= 0) return DDAMG_ERR_BAD_PARAM;
    std::ofstream f(path, std::ios::binary);
    if (!f) return DDAMG_ERR_IO;
    for (int x = 0; x < Nx; x++)
        for (int t = 0; t < Nt; t++)
            for (int mu = 0; mu < 2; mu++) {
                int32_t hdr[3] = {x, t, mu};
                long i = ((long)x * Nt + t) * 2 + mu;
                f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
                f.write(reinterpret_cast<const char*>(field + 2 * i), 2 * sizeof(double));
            }
    return f ? DDAMG_OK : DDAMG_ERR_IO;
}

ddamg_status ddamg_load_gauge(ddamg_t* h, const double* U) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!U) throw ParamFailure{"null gauge field"};
    LevelData& D = h->lv[0];
    const long n = 2L * D.g.sites;
    for (long i = 0; i < 2 * n; i++)
        if (!std::isfinite(U[i])) {
            set_error("non-finite value in the gauge field");
            return DDAMG_ERR_NAN;
        }
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.U, U, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    if (D.fp32) launch_convert<double2, float2>(h->s, D.d.U, D.f.U, n);
    sync(h);
    h->gauge = true;
    h->setup_done = false;
    API_END
}

static ddamg_status apply_dirac_dev(ddamg_t* h, int dagger, const double2* in, double2* out, int nrhs) {
    const Geom& g = h->lv[0].g;
    launch_wilson<double2>(h->s, h->lv[0].d.U, in, out, nullptr, g.Nx, g.Nt, h->p.m0, dagger, nrhs);
    return DDAMG_OK;
}

ddamg_status ddamg_apply_dirac(ddamg_t* h, int dagger, const double* in, double* out, int nrhs) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (nrhs < 1 || nrhs > h->W) throw ParamFailure{"nrhs out of range"};
    const long n = h->lv[0].g.size() * nrhs;
    LevelData& D = h->lv[0];
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, in, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    apply_dirac_dev(h, dagger, D.d.eta, D.d.psi, nrhs);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    API_END
}
ddamg_status ddamg_apply_dirac_device(ddamg_t* h, int dagger, const void* in, void* out, int nrhs) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    apply_dirac_dev(h, dagger, static_cast<const double2*>(in), static_cast<double2*>(out), nrhs);
    API_END
}
ddamg_status ddamg_apply_dirac_f32_device(ddamg_t* h, int dagger, const void* in, void* out, int nrhs) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    LevelData& D = h->lv[0];
    if (!D.f.U) {
        D.f.U = dalloc_t<float2>(h, 2L * D.g.sites);
        launch_convert<double2, float2>(h->s, D.d.U, D.f.U, 2L * D.g.sites);
    }
    launch_wilson<float2>(h->s, D.f.U, static_cast<const float2*>(in), static_cast<float2*>(out), nullptr, D.g.Nx,
                          D.g.Nt, h->p.m0, dagger, nrhs);
    API_END
}

ddamg_status ddamg_apply_level_op_device(ddamg_t* h, int level, int fp32, const void* in, void* out, int nrhs) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, true);
    if (level == 0 && !h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (level > 0) need_setup(h);
    if (!in || !out || nrhs < 1) throw ParamFailure{"ddamg_apply_level_op_device: bad argument"};
    LevelData& D = h->lv[level];
    if (fp32) {
        if (!D.fp32) throw ParamFailure{"this level has no FP32 operator (a mixed-precision handle has one below the coarsest level)"};
        level_op<float2>(h, level, static_cast<const float2*>(in), static_cast<float2*>(out), nullptr, nrhs);
    } else {
        level_op<double2>(h, level, static_cast<const double2*>(in), static_cast<double2*>(out), nullptr, nrhs);
    }
    check_tc_status(h);
    API_END
}
ddamg_status ddamg_apply_level_op(ddamg_t* h, int level, const double* in, double* out) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, true);
    if (level == 0 && !h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (level > 0) need_setup(h);
    LevelData& D = h->lv[level];
    const long n = D.g.size();
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, in, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    level_op<double2>(h, level, D.d.eta, D.d.psi, nullptr, 1);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    API_END
}

ddamg_status ddamg_restrict(ddamg_t* h, int level, const double* in, double* out) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    need_setup(h);
    LevelData& D = h->lv[level];
    LevelData& N = h->lv[level + 1];
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, in, sizeof(double2) * D.g.size(), cudaMemcpyHostToDevice, h->s));
    launch_restrict<double2>(h->s, D.g, D.d.tv, D.d.eta, N.d.psi, 1);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, N.d.psi, sizeof(double2) * N.g.size(), cudaMemcpyDeviceToHost, h->s));
    sync(h);
    API_END
}
ddamg_status ddamg_prolong(ddamg_t* h, int level, const double* in, double* out) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    need_setup(h);
    LevelData& D = h->lv[level];
    LevelData& N = h->lv[level + 1];
    DDAMG_CUDA_TRY(cudaMemcpyAsync(N.d.eta, in, sizeof(double2) * N.g.size(), cudaMemcpyHostToDevice, h->s));
    launch_prolong<double2>(h->s, D.g, D.d.tv, N.d.eta, D.d.psi, 0, 1);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, D.d.psi, sizeof(double2) * D.g.size(), cudaMemcpyDeviceToHost, h->s));
    sync(h);
    API_END
}

ddamg_status ddamg_sap(ddamg_t* h, int level, const double* v, double* x, int nu, double tol, int* iters) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    if (level == 0 && !h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (level > 0) need_setup(h);
    if (nu < 0) throw ParamFailure{"nu must be >= 0"};
    LevelData& D = h->lv[level];
    const long n = D.g.size();
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, v, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.psi, x, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    int it = sap_t<double2>(h, level, D.d.eta, D.d.psi, nu, tol, false, 1, true);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    if (iters) *iters = it;
    API_END
}

ddamg_status ddamg_sap_batched(ddamg_t* h, int level, const double* v, double* x, int nrhs, int nu, double tol) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    if (level == 0 && !h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (level > 0) need_setup(h);
    if (nu < 0) throw ParamFailure{"nu must be >= 0"};
    if (nrhs < 1 || nrhs > h->W) throw ParamFailure{"nrhs must be in [1, max(max_rhs, test vectors)]"};
    LevelData& D = h->lv[level];
    const long n = D.g.size() * nrhs;
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, v, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.psi, x, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    if (D.fp32) {
        launch_convert<double2, float2>(h->s, D.d.eta, D.f.eta, n);
        launch_convert<double2, float2>(h->s, D.d.psi, D.f.psi, n);
        sap_t<float2>(h, level, D.f.eta, D.f.psi, nu, tol, false, nrhs, false);
        launch_convert<float2, double2>(h->s, D.f.psi, D.d.psi, n);
    } else {
        sap_t<double2>(h, level, D.d.eta, D.d.psi, nu, tol, false, nrhs, false);
    }
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    check_tc_status(h);
    API_END
}

ddamg_status ddamg_setup(ddamg_t* h, uint64_t seed) {
    CHECK_HANDLE(h);
    API_BEGIN
    setup(h, nullptr, seed);
    API_END
}
ddamg_status ddamg_setup_random_count(ddamg_t* h, int64_t* n) {
    CHECK_HANDLE(h);
    API_BEGIN
    *n = setup_random_count(h);
    API_END
}
ddamg_status ddamg_setup_with_vectors(ddamg_t* h, const double* rnd, int64_t n) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!rnd || n < setup_random_count(h)) throw ParamFailure{"random stream too short"};
    setup(h, reinterpret_cast<const double2*>(rnd), 0);
    API_END
}
ddamg_status ddamg_get_test_vectors(ddamg_t* h, int level, double* out) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    LevelData& D = h->lv[level];
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, D.d.tv, sizeof(double2) * D.g.ntest * D.g.size(), cudaMemcpyDeviceToHost, h->s));
    sync(h);
    API_END
}
ddamg_status ddamg_set_test_vectors(ddamg_t* h, int level, const double* in) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    LevelData& D = h->lv[level];
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.tv, in, sizeof(double2) * D.g.ntest * D.g.size(), cudaMemcpyHostToDevice, h->s));
    if (D.fp32) launch_convert<double2, float2>(h->s, D.d.tv, D.f.tv, (long)D.g.ntest * D.g.size());
    sync(h);
    API_END
}
ddamg_status ddamg_orthonormalize(ddamg_t* h, int level) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    LevelData& D = h->lv[level];
    launch_orthonormalize(h->s, D.g, D.d.tv);
    if (D.fp32) launch_convert<double2, float2>(h->s, D.d.tv, D.f.tv, (long)D.g.ntest * D.g.size());
    sync(h);
    API_END
}
ddamg_status ddamg_build_coarse_links(ddamg_t* h, int level) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_level(h, level, false);
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    LevelData& D = h->lv[level];
    LevelData& N = h->lv[level + 1];
    launch_build_coarse_links(h->s, D.g, D.d.U, D.d.links, D.d.tv, N.d.links);
    if (N.fp32) launch_convert<double2, float2>(h->s, N.d.links, N.f.links, (long)N.g.sites * 5 * N.g.dof * N.g.dof);
    if (N.tc) launch_pack_tc_links(h->s, N.g, N.f.links, N.tcw.tiles);
    sync(h);
    API_END
}
ddamg_status ddamg_get_coarse_links(ddamg_t* h, int level, int which, double* out) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (level < 1 || level >= h->L) throw ParamFailure{"coarse links exist on levels >= 1"};
    if (which < 1 || which > 3) throw ParamFailure{"which must be 1, 2 or 3"};
    LevelData& D = h->lv[level];
    const int dof = D.g.dof, C = D.g.colors;
    std::vector<double2> M((size_t)D.g.sites * 5 * dof * dof);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(M.data(), D.d.links, sizeof(double2) * M.size(), cudaMemcpyDeviceToHost, h->s));
    sync(h);
    double2* o = reinterpret_cast<double2*>(out);
    for (int n = 0; n < D.g.sites; n++)
        for (int alf = 0; alf < 2; alf++)
            for (int bet = 0; bet < 2; bet++)
                for (int c = 0; c < C; c++)
                    for (int b = 0; b < C; b++) {
                        const int i = c * 2 + alf, j = b * 2 + bet;
                        auto get = [&](int d) { return M[(((size_t)n * 5 + d) * dof + j) * dof + i]; };
                        const size_t base = ((((size_t)n * 2 + alf) * 2 + bet) * C + c) * C + b;
                        if (which == 1) o[base] = get(0);
                        else
                            for (int mu = 0; mu < 2; mu++) o[base * 2 + mu] = get(which == 2 ? 1 + mu : 3 + mu);
                    }
    API_END
}

ddamg_status ddamg_coarse_solve(ddamg_t* h, const double* b, double* x, int* iters) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_setup(h);
    LevelData& D = h->lv[h->L - 1];
    const long n = D.g.size();
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, b, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    coarse_solve(h, D.d.eta, D.d.psi);
    int it = 0;
    check_coarse_status(h, &it);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    if (iters) *iters = it;
    API_END
}

static ddamg_status run_cycle(ddamg_t* h, const double* eta, double* psi, int kind) {
    need_setup(h);
    const long n = h->lv[0].g.size();
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ow, eta, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    const int saved = h->p.cycle;
    h->p.cycle = kind;
    try {
        outer_prec(h, h->ow, h->orr, 1);
    } catch (...) {
        h->p.cycle = saved;
        throw;
    }
    h->p.cycle = saved;
    check_coarse_status(h, nullptr);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(psi, h->orr, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    return DDAMG_OK;
}
ddamg_status ddamg_vcycle(ddamg_t* h, const double* eta, double* psi) {
    CHECK_HANDLE(h);
    API_BEGIN
    return run_cycle(h, eta, psi, DDAMG_CYCLE_V);
    API_END
}
ddamg_status ddamg_kcycle(ddamg_t* h, const double* eta, double* psi) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (h->p.cycle != DDAMG_CYCLE_K) throw ParamFailure{"the K-cycle needs a handle created with cycle = DDAMG_CYCLE_K"};
    return run_cycle(h, eta, psi, DDAMG_CYCLE_K);
    API_END
}

ddamg_status ddamg_solve_device(ddamg_t* h, const void* b, void* x, int nrhs, ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (nrhs < 1 || nrhs > h->p.max_rhs) throw ParamFailure{"nrhs must be in [1, max_rhs]"};
    return solve_device(h, static_cast<const double2*>(b), static_cast<double2*>(x), nrhs, info);
    API_END
}
ddamg_status ddamg_solve(ddamg_t* h, const double* b, double* x, int nrhs, ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (nrhs < 1 || nrhs > h->p.max_rhs) throw ParamFailure{"nrhs must be in [1, max_rhs]"};
    const long n = h->lv[0].g.size() * nrhs;
    for (long i = 0; i < 2 * n; i++)
        if (!std::isfinite(b[i])) {
            set_error("non-finite value in the right-hand side");
            return DDAMG_ERR_NAN;
        }
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ob, b, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    ddamg_status st = solve_device(h, h->ob, h->ox, nrhs, info);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, h->ox, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    return st;
    API_END
}

ddamg_status ddamg_gmres_plain(ddamg_t* h, const double* b, double* x, int m, int restarts, double tol,
                               ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (m < 1 || restarts < 1) throw ParamFailure{"m and restarts must be >= 1"};
    const Geom& g0 = h->lv[0].g;
    const long n = g0.size();
    double2* Vb = dalloc_t<double2>(h, (size_t)(m + 1) * n);
    double2* Z = dalloc_t<double2>(h, (size_t)m * n);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ob, b, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    std::function<void(const double2*, double2*, int)> A = [h, &g0](const double2* in, double2* out, int R) {
        launch_wilson<double2>(h->s, h->lv[0].d.U, in, out, nullptr, g0.Nx, g0.Nt, h->p.m0, 0, R);
    };
    Krylov<double2> K{Vb, Z, h->ow, h->orr};
    double rel = 0;
    int it = 0;
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev0, h->s));
    fgmres_host<double2>(h, n, 1, m, restarts, tol, A, nullptr, h->ob, nullptr, true, h->ox, K, &it, &rel);
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, h->ox, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    float ms = 0;
    DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    // release the temporary basis
    for (void* q : {(void*)Vb, (void*)Z}) {
        cudaFree(q);
        h->allocs.erase(std::find(h->allocs.begin(), h->allocs.end(), q));
    }
    h->counts[DDAMG_COUNT_GMRES] = it;
    if (info) {
        info->iterations = it;
        info->converged = rel < tol;
        info->rel_residual = rel;
        info->setup_seconds = 0;
        info->solve_seconds = ms * 1e-3;
    }
    if (!(rel < tol)) return DDAMG_NOT_CONVERGED;
    API_END
}

// ------------------------------------------------------------------ stand-alone multigrid, FGMRES_SAP
namespace ddamg {
static void check_finite(const double* a, long count, const char* what) {
    for (long i = 0; i < count; i++)
        if (!std::isfinite(a[i])) throw NanFailure{std::string("non-finite value in ") + what};
}

// the fine-level Schwarz layout of sap_x x sap_t blocks (counts), made on first use
static const SapLayout& fine_layout(ddamg_handle* h, int sx, int st) {
    const auto key = std::make_pair(sx, st);
    auto it = h->fine_sap.find(key);
    if (it != h->fine_sap.end()) return it->second;
    const Geom& g0 = h->lv[0].g;
    if (sx < 1 || st < 1 || g0.Nx % sx || g0.Nt % st) bad("SAP block counts must divide the lattice");
    const int nb = sx * st;
    // the reference fills RedBlocks[block/2] (src/sap.cpp:30-37): an odd count > 1 overruns it
    if (nb > 1 && nb % 2) bad("the number of SAP blocks must be even (or 1)");
    SapLayout L;
    L.g = g0;
    L.g.sap_x = sx;
    L.g.sap_t = st;
    L.g.sel_x = g0.Nx / sx;
    L.g.sel_t = g0.Nt / st;
    const int S = L.g.sel_x * L.g.sel_t, NE = 2 * S;
    // blocks of up to 256 sites run one per warp; larger ones one per CTA with the Krylov basis in
    // shared memory
    if (S > 256 && (NE > 4096 || sap_smem_bytes(h->p.sap_gmres_restart_length, NE, true) > 227 * 1024))
        bad("SAP block of " + std::to_string(S) + " sites too large (its Krylov basis does not fit in shared memory)");
    std::vector<int> red, black;
    for (int b = 0; b < nb; b++) {  // red iff (bx + bt) even (src/sap.cpp:27-38); one block is both
        const int bx = b / st, bt = b % st;
        if (nb == 1) {
            red.push_back(b);
            black.push_back(b);
        } else if ((bx + bt) % 2 == 0) red.push_back(b);
        else black.push_back(b);
    }
    L.red = dalloc_t<int>(h, red.size());
    L.black = dalloc_t<int>(h, black.size());
    DDAMG_CUDA_TRY(cudaMemcpyAsync(L.red, red.data(), red.size() * sizeof(int), cudaMemcpyHostToDevice, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(L.black, black.data(), black.size() * sizeof(int), cudaMemcpyHostToDevice, h->s));
    L.nred = (int)red.size();
    L.nblack = (int)black.size();
    sync(h);
    return h->fine_sap[key] = L;
}

// FGMRES_SAP::preconditioner (include/sap.h:269-280): out = 0, one SAP iteration over the layout's
// blocks in the level-0 working precision (one iteration ends before SAP's convergence test matters)
static void fine_sap_prec(ddamg_handle* h, const SapLayout& lay, const double2* in, double2* out, int R) {
    LevelData& D = h->lv[0];
    const long n = D.g.size() * R;
    if (D.fp32) {
        launch_convert<double2, float2>(h->s, in, D.f.eta, n);
        DDAMG_CUDA_TRY(cudaMemsetAsync(D.f.psi, 0, sizeof(float2) * n, h->s));
        sap_t<float2>(h, 0, D.f.eta, D.f.psi, 1, 0.0, true, R, false, &lay);
        launch_convert<float2, double2>(h->s, D.f.psi, out, n);
    } else {
        DDAMG_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double2) * n, h->s));
        sap_t<double2>(h, 0, in, out, 1, 0.0, true, R, false, &lay);
    }
}
}  // namespace ddamg

ddamg_status ddamg_set_coarse_barrier_polls(ddamg_t* h, int polls) {
    CHECK_HANDLE(h);
    API_BEGIN
    h->p.coarse_barrier_polls = polls;
    h->cg.spin_limit = polls;
    for (auto& w : h->cg_lane) w.spin_limit = polls;
    // captured V-cycle graphs hold the old limit in their kernel parameters: capture again
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second.exec);
    h->graphs.clear();
    h->graph_warm.clear();
    for (auto& kv : h->solve_graphs) cudaGraphExecDestroy(kv.second.exec);
    h->solve_graphs.clear();
    h->solve_warm.clear();
    API_END
}

// ------------------------------------------------------------------ run metadata
namespace ddamg {
// writeMetadata (src/io.cpp:72-145): the same lines, widths and number formats
static void write_metadata(const ddamg_params& p, const long long* c, int cycle, double tol, const char* path) {
    if (cycle != DDAMG_CYCLE_V && cycle != DDAMG_CYCLE_K) throw ParamFailure{"cycle must be 0 (V) or 1 (K)"};
    if (p.levels < 2 || p.levels > DDAMG_MAX_LEVELS) throw ParamFailure{"levels out of range"};
    std::string file;
    if (path) {
        file = path;
    } else {
        std::ostringstream fn;
        fn << "metadata_" << p.Nx << "x" << p.Nt << "_Levels" << p.levels << (cycle == 0 ? "_Vcycle" : "_Kcycle")
           << ".dat";
        file = fn.str();
    }
    std::string host;
    if (const char* e = std::getenv("HOSTNAME")) {
        host = e;
    } else {
        char buf[256] = {};
        if (gethostname(buf, sizeof(buf) - 1) == 0) host = buf;
    }
    const std::time_t now = std::time(nullptr);
    std::tm tmv{};
    localtime_r(&now, &tmv);
    std::ostringstream o;
    o << "Host: " << host << "\n";
    o << "Date: " << std::put_time(&tmv, "%Y-%m-%d %H:%M:%S") << "\n";
    o << "x ranks: " << 1 << "  t_ranks: " << 1 << "\n";
    o << "m0: " << std::setprecision(7) << p.m0 << "\n";
    o << "solvers tolerance: " << std::setprecision(4) << tol << "\n";
    o << "#level, blocks_x (global), blocks_t (global), Ntest, SAP_blocks_x (local), SAP_blocks_t (local)\n";
    for (int l = 0; l < p.levels - 1; l++) {
        o << l;
        for (int k = 1; k <= 5; k++) o << std::setw(5) << p.rows[l][k];
        o << "\n";
    }
    auto triple = [&](int a, int b, double t) {
        o << a << std::setw(5) << b << std::setw(15) << std::scientific << std::setprecision(7) << t << "\n";
    };
    o << "#SAP_test_vectors_iterations\n" << p.sap_test_vectors_iterations << "\n";
    o << "#cycle (0 = V, 1 = K)\n" << cycle << "\n";
    o << "#Pre-smoothing nu1, Post-smoothing nu2\n" << p.nu1 << std::setw(5) << p.nu2 << "\n";
    o << "#sap gmres restart length, sap gmres restarts, sap gmres tolerance\n";
    triple(p.sap_gmres_restart_length, p.sap_gmres_restarts, p.sap_gmres_tolerance);
    o << "#GMRES restart length coarse level, GMRES restarts coarse level, GMRES tolerance coarse level\n";
    triple(p.coarse_gmres_restart_length, p.coarse_gmres_restarts, p.coarse_gmres_tolerance);
    o << "#FGMRES restart length, FGMRES restarts, FGMRES tolerance\n";
    triple(p.fgmres_restart_length, p.fgmres_restarts, p.fgmres_tolerance);
    const long long none = -1;  // FLOP counters are not kept
    auto pair = [&](const char* head, long long it) { o << head << "\n" << it << std::setw(30) << none << "\n"; };
    pair("#CG iterations,   FLOPS", c[DDAMG_COUNT_CG]);
    pair("#BiCGStab iterations,   FLOPS", c[DDAMG_COUNT_BICG]);
    pair("#GMRES iterations,   FLOPS", c[DDAMG_COUNT_GMRES]);
    pair("#SAP iterations,   FLOPS", c[DDAMG_COUNT_SAP]);
    pair("#FGMRES_SAP iterations,   FLOPS", c[DDAMG_COUNT_FGMRES_SAP]);
    o << (cycle == 0 ? "#V cycle fgmres iterations,  Setup phase FLOPS, Total FLOPS\n"
                     : "#K cycle fgmres iterations,  Setup phase FLOPS, Total FLOPS\n");
    o << c[cycle == 0 ? DDAMG_COUNT_VCYCLE : DDAMG_COUNT_KCYCLE] << std::setw(30) << none << std::setw(30) << none
      << "\n";
    std::ofstream f(file);
    if (!f) throw IoFailure{"cannot open " + file + " for writing"};
    f << o.str();
    if (!f) throw IoFailure{"write failed: " + file};
}
}  // namespace ddamg

ddamg_status ddamg_set_stencil_kernel(int kind) {
    API_BEGIN
    if (kind < 0 || kind > 2) throw ParamFailure{"stencil kernel must be 0 (default), 1 (register) or 2 (staged)"};
    set_stencil_variant(kind);
    API_END
}
ddamg_status ddamg_get_stencil_kernel(int* kind) {
    if (!kind) {
        set_error("null argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    *kind = stencil_variant();
    return DDAMG_OK;
}

ddamg_status ddamg_get_counters(ddamg_t* h, long long counts[DDAMG_COUNT_KINDS]) {
    if (!h || !counts) {
        set_error("null argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    std::copy(h->counts, h->counts + DDAMG_COUNT_KINDS, counts);
    return DDAMG_OK;
}
ddamg_status ddamg_write_metadata(ddamg_t* h, const char* path, int cycle, double tol) {
    if (!h) {
        set_error("null handle");
        return DDAMG_ERR_BAD_PARAM;
    }
    return ddamg_write_metadata_params(&h->p, h->counts, cycle, tol, path);
}
ddamg_status ddamg_write_metadata_params(const ddamg_params* p, const long long counts[DDAMG_COUNT_KINDS], int cycle,
                                         double tol, const char* path) {
    API_BEGIN
    if (!p || !counts) throw ParamFailure{"null argument"};
    write_metadata(*p, counts, cycle, tol, path);
    API_END
}

ddamg_status ddamg_apply_multilevel(ddamg_t* h, const double* rhs, double* x, int max_cycles, double tol,
                                    int* cycles, double* rel_residual) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_setup(h);
    if (!rhs || !x || max_cycles < 0 || !(tol > 0)) throw ParamFailure{"ddamg_apply_multilevel: bad argument"};
    LevelData& D = h->lv[0];
    const Geom& g0 = D.g;
    const long n = g0.size();
    check_finite(rhs, 2 * n, "the right-hand side");
    check_finite(x, 2 * n, "the initial guess");
    cudaStream_t s = h->s;
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ob, rhs, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ox, x, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
    double* hn = reinterpret_cast<double*>(h->hpin);
    launch_norm2<double2>(s, h->ob, n, n, 1, h->dpart, h->dn);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(hn, h->dn, sizeof(double), cudaMemcpyDeviceToHost, s));
    sync(h);
    const double norm = std::sqrt(hn[0]);
    int ran = 0;
    double err = 0.0;
    bool conv = false;
    if (norm == 0.0) {  // the zero right-hand side: x = 0 (the reference would run max_cycles cycles)
        DDAMG_CUDA_TRY(cudaMemsetAsync(h->ox, 0, sizeof(double2) * n, s));
        conv = true;
    }
    for (int i = 0; i < max_cycles && !conv; i++) {
        if (!D.fp32) {
            cycle(h, 0, h->ob, h->ox, false, h->p.cycle, 1);  // v_cycle / k_cycle(0, rhs, out): out is the iterate
        } else {
            // the FP32 cycle acts on the FP64 residual from zero; its result corrects the FP64 iterate
            launch_wilson<double2>(s, D.d.U, h->ox, h->orr, h->ob, g0.Nx, g0.Nt, h->p.m0, 0, 1);
            outer_prec(h, h->orr, h->ow, 1);
            launch_add<double2>(s, h->ow, h->ox, n);
        }
        // r = rhs - D out with the level-0 operator, ||r|| (src/amg.cpp:186-199)
        launch_wilson<double2>(s, D.d.U, h->ox, h->orr, h->ob, g0.Nx, g0.Nt, h->p.m0, 0, 1);
        launch_norm2<double2>(s, h->orr, n, n, 1, h->dpart, h->dn);
        DDAMG_CUDA_TRY(cudaMemcpyAsync(hn, h->dn, sizeof(double), cudaMemcpyDeviceToHost, s));
        sync(h);
        err = std::sqrt(hn[0]);
        ran = i + 1;
        if (!std::isfinite(err)) throw NanFailure{"non-finite residual in the multigrid iteration"};
        if (err < tol * norm) conv = true;
    }
    check_coarse_status(h, nullptr);
    check_tc_status(h);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, h->ox, sizeof(double2) * n, cudaMemcpyDeviceToHost, s));
    sync(h);
    if (cycles) *cycles = ran;
    if (rel_residual) *rel_residual = norm > 0 ? err / norm : 0.0;
    if (!conv) {
        set_error("no convergence within max_cycles cycles");
        return DDAMG_NOT_CONVERGED;
    }
    API_END
}

ddamg_status ddamg_fgmres_sap(ddamg_t* h, const double* b, double* x, int blocks_x, int blocks_t, int m,
                              int restarts, double tol, ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (!b || !x || m < 1 || restarts < 1 || !(tol > 0)) throw ParamFailure{"ddamg_fgmres_sap: bad argument"};
    const Geom& g0 = h->lv[0].g;
    const long n = g0.size();
    check_finite(b, 2 * n, "the right-hand side");
    const SapLayout& lay = fine_layout(h, blocks_x, blocks_t);
    // the outer FGMRES basis: the handle's when it is long enough, else a temporary one
    const bool own = m <= h->p.fgmres_restart_length;
    double2* Vb = own ? h->oV : dalloc_t<double2>(h, (size_t)(m + 1) * n);
    double2* Z = own ? h->oZ : dalloc_t<double2>(h, (size_t)m * n);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ob, b, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    std::function<void(const double2*, double2*, int)> A = [h, &g0](const double2* in, double2* out, int R) {
        launch_wilson<double2>(h->s, h->lv[0].d.U, in, out, nullptr, g0.Nx, g0.Nt, h->p.m0, 0, R);
    };
    std::function<void(const double2*, double2*, int, int)> M = [h, &lay](const double2* in, double2* out, int R,
                                                                          int) { fine_sap_prec(h, lay, in, out, R); };
    Krylov<double2> K{Vb, Z, h->ow, h->orr};
    double rel = 0;
    int it = 0;
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev0, h->s));
    fgmres_host<double2>(h, n, 1, m, restarts, tol, A, &M, h->ob, nullptr, true, h->ox, K, &it, &rel);
    DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, h->ox, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    float ms = 0;
    DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (!own)
        for (void* q : {(void*)Vb, (void*)Z}) {
            cudaFree(q);
            h->allocs.erase(std::find(h->allocs.begin(), h->allocs.end(), q));
        }
    h->counts[DDAMG_COUNT_FGMRES_SAP] = it;
    if (info) {
        info->iterations = it;
        info->converged = rel < tol;
        info->rel_residual = rel;
        info->setup_seconds = 0;
        info->solve_seconds = ms * 1e-3;
    }
    if (!(rel < tol)) return DDAMG_NOT_CONVERGED;
    API_END
}

ddamg_status ddamg_sap_fine(ddamg_t* h, const double* v, double* x, int blocks_x, int blocks_t, int nu, double tol,
                            int* iters) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (!v || !x || nu < 0) throw ParamFailure{"ddamg_sap_fine: bad argument"};
    LevelData& D = h->lv[0];
    const long n = D.g.size();
    const SapLayout& lay = fine_layout(h, blocks_x, blocks_t);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, v, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.psi, x, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    const int it = sap_t<double2>(h, 0, D.d.eta, D.d.psi, nu, tol, false, 1, true, &lay);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(x, D.d.psi, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    h->counts[DDAMG_COUNT_SAP] = it;
    if (iters) *iters = it;
    API_END
}

// ------------------------------------------------------------------ comparison solvers
namespace ddamg {
static void krylov_alloc(ddamg_handle* h) {
    KrylovWork& w = h->kry;
    if (w.x) return;
    const long n = h->lv[0].g.size();
    for (double2** p : {&w.b, &w.rt, &w.x, &w.r, &w.s, &w.t, &w.y, &w.d[0], &w.d[1], &w.Ad[0], &w.Ad[1]})
        *p = dalloc_t<double2>(h, n);
    w.part = dalloc_t<double2>(h, 3 * (size_t)krylov_grid(h->lv[0].g.sites));
    w.st = static_cast<KrylovState*>(dalloc(h, sizeof(KrylovState)));
}

// bi_cgstab (solver 0) or conjugate_gradient on D^dagger D (solver 1), src/conjugate_gradient.cpp.
// With cuda_graphs set the whole iteration runs on the device: one graph whose while node repeats a
// body of kKrylovBody iterations and a one-thread kernel that keeps the loop going while the done
// word is clear (the device sets it at convergence or at max_iter, so the loop is bounded).
// Otherwise (or if the graph cannot be built) iterations are queued in batches of kKrylovBatch and
// the next batch is queued before the done word of the current one is read.  info->iterations
// follows the reference's count; the true residual is recomputed for the system the solver
// iterates on.
constexpr int kKrylovBatch = 16;
constexpr int kKrylovBody = 4;

// the device-driven solve graph; nullptr if this driver or runtime cannot build it
static cudaGraphExec_t krylov_while_graph(ddamg_handle* h, int solver, const KrylovWork& w, const Geom& g,
                                          double tol, int max_iter) {
    cudaStream_t s = h->s;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const long long l0 = g_launches;
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle hc{};
    ok = ok && cudaGraphConditionalHandleCreate(&hc, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hc;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    ok = ok && cudaGraphAddNode(&node, graph, nullptr, 0, &np) == cudaSuccess;
    if (ok && cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        try {
            launch_krylov_iterations(s, solver, w, h->lv[0].d.U, g.Nx, g.Nt, h->p.m0, tol, max_iter, kKrylovBody);
            launch_krylov_continue(s, hc, w);
        } catch (...) {
            ok = false;
        }
        cudaGraph_t body = nullptr;
        if (cudaStreamEndCapture(s, &body) != cudaSuccess) ok = false;
    } else {
        ok = false;
    }
    ok = ok && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    g_launches = l0;  // recorded, not run; counted after the solve
    if (!ok) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return nullptr;
    }
    return exec;
}
static ddamg_status krylov_run(ddamg_handle* h, int solver, const double* b, const double* x0, double* x,
                               int max_iter, double tol, ddamg_solve_info* info) {
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    if (max_iter < 1 || !(tol > 0)) throw ParamFailure{"max_iter must be >= 1 and tol > 0"};
    const Geom& g = h->lv[0].g;
    const long n = g.size();
    double bb = 0.0;
    for (long i = 0; i < 2 * n; i++) {
        if (!std::isfinite(b[i]) || (x0 && !std::isfinite(x0[i]))) {
            set_error("non-finite value in the right-hand side or the initial guess");
            return DDAMG_ERR_NAN;
        }
        bb += b[i] * b[i];
    }
    if (bb == 0.0) {  // the zero right-hand side has the zero solution (the reference divides by zero)
        std::fill(x, x + 2 * n, 0.0);
        if (info) *info = ddamg_solve_info{};
        if (info) info->converged = 1;
        return DDAMG_OK;
    }
    krylov_alloc(h);
    KrylovWork& w = h->kry;
    const double2* U = h->lv[0].d.U;
    cudaStream_t s = h->s;
    DDAMG_CUDA_TRY(cudaMemcpyAsync(w.b, b, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
    if (solver == 0) {
        if (x0) DDAMG_CUDA_TRY(cudaMemcpyAsync(w.x, x0, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
        else DDAMG_CUDA_TRY(cudaMemsetAsync(w.x, 0, sizeof(double2) * n, s));
    }
    cudaGraphExec_t wexec = (h->p.cuda_graphs && !h->prof) ? krylov_while_graph(h, solver, w, g, tol, max_iter)
                                                          : nullptr;
    {
        const std::string note = std::string(solver == 0 ? "bicgstab" : "cg_normal") +
                                 (wexec ? ": device loop (graph while node, " + std::to_string(kKrylovBody) +
                                              " iterations per body)\n"
                                        : ": host-queued batches of " + std::to_string(kKrylovBatch) + " iterations\n");
        if (h->tune_log.find(note) == std::string::npos) h->tune_log += note;
    }
    cudaGraphExec_t exec = nullptr;
    long long graph_kernels = 0;
    if (!wexec && h->p.cuda_graphs && !h->prof) {  // one batch of iterations as a graph
        cudaGraph_t graph = nullptr;
        const long long l0 = g_launches;
        bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) == cudaSuccess;
        if (ok) {
            try {
                launch_krylov_iterations(s, solver, w, U, g.Nx, g.Nt, h->p.m0, tol, max_iter, kKrylovBatch);
            } catch (...) {
                ok = false;
            }
            if (cudaStreamEndCapture(s, &graph) != cudaSuccess || !graph) ok = false;
        }
        if (ok && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) ok = false;
        if (graph) cudaGraphDestroy(graph);
        graph_kernels = g_launches - l0;
        g_launches -= graph_kernels;
        if (!ok) {
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
    }
    cudaEvent_t evb[2] = {nullptr, nullptr};
    int* hd = reinterpret_cast<int*>(h->hpin);
    ddamg_status result = DDAMG_OK;
    try {
        for (cudaEvent_t& e : evb) DDAMG_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        DDAMG_CUDA_TRY(cudaEventRecord(h->ev0, s));
        launch_krylov_init(s, solver, w, U, g.Nx, g.Nt, h->p.m0, tol, max_iter);
        long launched = 0;
        if (wexec) {  // the whole iteration on the device
            DDAMG_CUDA_TRY(cudaGraphLaunch(wexec, s));
            launched = max_iter;
        }
        auto enqueue = [&](int slot) {
            if (exec) {
                DDAMG_CUDA_TRY(cudaGraphLaunch(exec, s));
                g_launches += graph_kernels;
            } else {
                launch_krylov_iterations(s, solver, w, U, g.Nx, g.Nt, h->p.m0, tol, max_iter, kKrylovBatch);
            }
            DDAMG_CUDA_TRY(cudaMemcpyAsync(hd + slot, &w.st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
            DDAMG_CUDA_TRY(cudaEventRecord(evb[slot], s));
            launched += kKrylovBatch;
        };
        if (!wexec) {
            enqueue(0);
            for (int i = 0;; i++) {
                if (launched < max_iter) enqueue((i + 1) & 1);
                DDAMG_CUDA_TRY(cudaEventSynchronize(evb[i & 1]));
                if (hd[i & 1] >= 2) break;
            }
        }
        DDAMG_CUDA_TRY(cudaEventRecord(h->ev1, s));
        // true residual of the iterated system: b - D x (BiCGstab), phi - D^dagger D x (CG)
        if (solver == 0) {
            launch_wilson<double2>(s, U, w.x, w.r, w.b, g.Nx, g.Nt, h->p.m0, 0, 1);
        } else {
            launch_wilson<double2>(s, U, w.x, w.y, nullptr, g.Nx, g.Nt, h->p.m0, 0, 1);
            launch_wilson<double2>(s, U, w.y, w.r, w.b, g.Nx, g.Nt, h->p.m0, 1, 1);
        }
        launch_norm2<double2>(s, w.r, n, n, 1, h->dpart, h->dn);
        launch_norm2<double2>(s, w.b, n, n, 1, h->dpart, h->dn + 1);
        KrylovState st;
        double nn[2];
        DDAMG_CUDA_TRY(cudaMemcpyAsync(&st, w.st, sizeof(st), cudaMemcpyDeviceToHost, s));
        DDAMG_CUDA_TRY(cudaMemcpyAsync(nn, h->dn, sizeof(nn), cudaMemcpyDeviceToHost, s));
        DDAMG_CUDA_TRY(cudaMemcpyAsync(x, w.x, sizeof(double2) * n, cudaMemcpyDeviceToHost, s));
        sync(h);
        if (wexec) g_launches += (long long)(st.k / kKrylovBody + 1) * (3 * kKrylovBody + 1);
        float ms = 0;
        DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        const double rel = nn[1] > 0 ? std::sqrt(nn[0] / nn[1]) : 0.0;
        h->counts[solver == 0 ? DDAMG_COUNT_BICG : DDAMG_COUNT_CG] = st.iters;
        if (info) {
            info->iterations = st.iters;
            info->converged = st.done == 2;
            info->rel_residual = rel;
            info->setup_seconds = 0;
            info->solve_seconds = ms * 1e-3;
        }
        if (!std::isfinite(rel)) {
            set_error("the Krylov iteration produced a non-finite value");
            result = DDAMG_ERR_NAN;
        } else if (st.done != 2) {
            set_error("no convergence within max_iter iterations");
            result = DDAMG_NOT_CONVERGED;
        }
    } catch (...) {
        for (cudaEvent_t e : evb)
            if (e) cudaEventDestroy(e);
        if (exec) cudaGraphExecDestroy(exec);
        if (wexec) cudaGraphExecDestroy(wexec);
        throw;
    }
    for (cudaEvent_t e : evb) cudaEventDestroy(e);
    if (exec) cudaGraphExecDestroy(exec);
    if (wexec) cudaGraphExecDestroy(wexec);
    return result;
}
}  // namespace ddamg

ddamg_status ddamg_bicgstab(ddamg_t* h, const double* b, const double* x0, double* x, int max_iter, double tol,
                            ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!b || !x) throw ParamFailure{"null vector"};
    return krylov_run(h, 0, b, x0, x, max_iter, tol, info);
    API_END
}

ddamg_status ddamg_cg_normal(ddamg_t* h, const double* phi, double* x, int max_iter, double tol,
                             ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!phi || !x) throw ParamFailure{"null vector"};
    return krylov_run(h, 1, phi, nullptr, x, max_iter, tol, info);
    API_END
}

// ------------------------------------------------------------------ HMC
namespace ddamg {
constexpr uint64_t kStreamHmc = 0x484D43ull;
static const double kPi = 3.14159265358979323846;

static double host_gauge_action(const std::vector<double>& th, int Nx, int Nt, double beta, double* plaq_mean) {
    double s = 0.0, c = 0.0;
    for (int x = 0; x < Nx; x++)
        for (int t = 0; t < Nt; t++) {
            const int n = x * Nt + t, ntp = x * Nt + (t + 1) % Nt, nxp = ((x + 1) % Nx) * Nt + t;
            const double P = th[2 * n] + th[2 * ntp + 1] - th[2 * nxp] - th[2 * n + 1];
            s += 1.0 - std::cos(P);
            c += std::cos(P);
        }
    if (plaq_mean) *plaq_mean = c / ((double)Nx * Nt);
    return beta * s;
}

// HMC state on the device for one call: angles, momenta, the two force fields, the CG solution and D X
struct HmcBuffers {
    double *th = nullptr, *p = nullptr, *Fg = nullptr, *Ff = nullptr;
    double2 *X = nullptr, *Y = nullptr, *tmp = nullptr;
};

// dS/dtheta at the angles in B.th for phi (host): U = exp(i theta) into the handle, X = (D^dagger D)^-1 phi by
// CG (X also returned on the host), Y = D X, Ff = link derivative(psi = X, lambda = Y), Fg = gauge force
static int hmc_force(ddamg_handle* h, HmcBuffers& B, const std::vector<double>& phi, std::vector<double>& X,
                     double beta, double cg_tol) {
    const Geom& g = h->lv[0].g;
    const long nl = 2L * g.sites;
    launch_theta_to_links(h->s, B.th, h->lv[0].d.U, nl);
    ddamg_solve_info info{};
    const ddamg_status st = krylov_run(h, 1, phi.data(), nullptr, X.data(), 100000, cg_tol, &info);
    if (st == DDAMG_NOT_CONVERGED)
        throw NotConvergedFailure{"HMC force: the CG solve did not converge (" + std::string(ddamg_last_error()) + ")"};
    if (st == DDAMG_ERR_NAN) throw NanFailure{"HMC force: " + std::string(ddamg_last_error())};
    if (st != DDAMG_OK) throw ParamFailure{"HMC force: the CG solve failed (" + std::string(ddamg_last_error()) + ")"};
    DDAMG_CUDA_TRY(cudaMemcpyAsync(B.X, X.data(), sizeof(double2) * g.size(), cudaMemcpyHostToDevice, h->s));
    launch_wilson<double2>(h->s, h->lv[0].d.U, B.X, B.Y, nullptr, g.Nx, g.Nt, h->p.m0, 0, 1);
    launch_link_derivative(h->s, h->lv[0].d.U, B.X, B.Y, B.Ff, g.Nx, g.Nt);
    launch_gauge_force(h->s, B.th, B.Fg, g.Nx, g.Nt, beta);
    return info.iterations;
}

// the buffers are filled in place, so after a failure part way through hmc_free releases what was allocated
static void hmc_alloc(ddamg_handle* h, HmcBuffers& B) {
    const Geom& g = h->lv[0].g;
    const long nl = 2L * g.sites, n = g.size();
    DDAMG_CUDA_TRY(cudaMalloc(&B.th, sizeof(double) * nl));
    DDAMG_CUDA_TRY(cudaMalloc(&B.p, sizeof(double) * nl));
    DDAMG_CUDA_TRY(cudaMalloc(&B.Fg, sizeof(double) * nl));
    DDAMG_CUDA_TRY(cudaMalloc(&B.Ff, sizeof(double) * nl));
    DDAMG_CUDA_TRY(cudaMalloc(&B.X, sizeof(double2) * n));
    DDAMG_CUDA_TRY(cudaMalloc(&B.Y, sizeof(double2) * n));
    DDAMG_CUDA_TRY(cudaMalloc(&B.tmp, sizeof(double2) * n));
}
static void hmc_free(HmcBuffers& B) {
    for (void* q : {(void*)B.th, (void*)B.p, (void*)B.Fg, (void*)B.Ff, (void*)B.X, (void*)B.Y, (void*)B.tmp})
        if (q) cudaFree(q);
    B = HmcBuffers{};
}

// after a failed trajectory: the handle's links back to the caller's starting angles (best effort), the
// device buffers freed; the multigrid setup no longer matches the links the trajectory left behind
static void hmc_restore(ddamg_handle* h, HmcBuffers& B, const std::vector<double>& theta0) {
    if (B.th && !theta0.empty()) {
        const long nl = 2L * h->lv[0].g.sites;
        if (cudaMemcpyAsync(B.th, theta0.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, h->s) == cudaSuccess) {
            try {
                launch_theta_to_links(h->s, B.th, h->lv[0].d.U, nl);
            } catch (...) {
            }
        }
        cudaStreamSynchronize(h->s);
    }
    h->setup_done = false;
    hmc_free(B);
}

// the HMC entry points map their failures to status codes themselves, because the device buffers and
// the handle's links must be put right on every path
static ddamg_status hmc_guard(const std::function<ddamg_status()>& body, const std::function<void()>& cleanup) {
    try {
        return body();
    } catch (const ParamFailure& e) {
        cleanup();
        set_error(e.msg);
        return DDAMG_ERR_BAD_PARAM;
    } catch (const NotConvergedFailure& e) {
        cleanup();
        set_error(e.msg);
        return DDAMG_NOT_CONVERGED;
    } catch (const NanFailure& e) {
        cleanup();
        set_error(e.msg);
        return DDAMG_ERR_NAN;
    } catch (const CudaFailure&) {
        cleanup();
        return DDAMG_ERR_CUDA;
    } catch (const std::exception& e) {
        cleanup();
        set_error(e.what());
        return DDAMG_ERR_STATE;
    }
}
}  // namespace ddamg

ddamg_status ddamg_hmc_force(ddamg_t* h, const double* theta, const double* phi, double beta, double cg_tol,
                             double* force) {
    CHECK_HANDLE(h);
    if (!theta || !phi || !force || !(cg_tol > 0)) {
        set_error("ddamg_hmc_force: bad argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    HmcBuffers B;
    bool saved = false;
    // the force needs the links of theta in the handle for the CG: the handle's own links are kept in
    // B.tmp (2 complex per site, the size of a fine vector) and put back on every path, so the handle's
    // gauge field and multigrid setup are unchanged afterwards
    auto restore_links = [&]() {
        if (saved)
            cudaMemcpyAsync(h->lv[0].d.U, B.tmp, sizeof(double2) * 2 * h->lv[0].g.sites, cudaMemcpyDeviceToDevice, h->s);
        cudaStreamSynchronize(h->s);
        hmc_free(B);
    };
    return hmc_guard(
        [&]() -> ddamg_status {
            if (!h->gauge) throw ParamFailure{"load a gauge field first (it sets up the fine-level storage)"};
            const Geom& g = h->lv[0].g;
            const long nl = 2L * g.sites, n = g.size();
            hmc_alloc(h, B);
            DDAMG_CUDA_TRY(cudaMemcpyAsync(B.tmp, h->lv[0].d.U, sizeof(double2) * nl, cudaMemcpyDeviceToDevice, h->s));
            saved = true;
            DDAMG_CUDA_TRY(cudaMemcpyAsync(B.th, theta, sizeof(double) * nl, cudaMemcpyHostToDevice, h->s));
            std::vector<double> ph(phi, phi + 2 * n), X(2 * n);
            hmc_force(h, B, ph, X, beta, cg_tol);
            DDAMG_CUDA_TRY(cudaMemsetAsync(B.p, 0, sizeof(double) * nl, h->s));
            launch_hmc_momentum(h->s, B.p, B.Fg, B.Ff, -1.0, nl);  // p = Fg + 2 Ff
            DDAMG_CUDA_TRY(cudaMemcpyAsync(force, B.p, sizeof(double) * nl, cudaMemcpyDeviceToHost, h->s));
            DDAMG_CUDA_TRY(cudaMemcpyAsync(h->lv[0].d.U, B.tmp, sizeof(double2) * nl, cudaMemcpyDeviceToDevice, h->s));
            saved = false;
            sync(h);
            hmc_free(B);
            return DDAMG_OK;
        },
        restore_links);
}

ddamg_status ddamg_hmc_trajectory(ddamg_t* h, double* theta, double beta, int md_steps, double tau, uint64_t seed,
                                  double cg_tol, ddamg_hmc_info* info) {
    CHECK_HANDLE(h);
    if (!theta || md_steps < 1 || !(tau > 0) || !(cg_tol > 0)) {
        set_error("ddamg_hmc_trajectory: bad argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    HmcBuffers B;
    std::vector<double> th0;  // the caller's angles: theta is written only once the trajectory has succeeded
    return hmc_guard(
        [&]() -> ddamg_status {
            if (!h->gauge) throw ParamFailure{"load a gauge field first (it sets up the fine-level storage)"};
            const auto t0 = std::chrono::steady_clock::now();
            const Geom& g = h->lv[0].g;
            const long V = g.sites, nl = 2L * V, n = g.size();
            th0.assign(theta, theta + nl);
            hmc_alloc(h, B);
            std::vector<double> p(nl), eta(2 * n), phi(2 * n), X(2 * n), th1(nl), p1(nl), thw(nl);
            // momenta ~ N(0, 1) per link and eta complex Gaussian with E|eta|^2 = 1, from the counter RNG
            ddamg_gaussian_field(V, rng64(seed, kStreamHmc, 1), p.data());
            for (double& v : p) v *= std::sqrt(2.0);
            ddamg_gaussian_field(n, rng64(seed, kStreamHmc, 2), eta.data());
            double pp = 0.0, ee = 0.0;
            for (double v : p) pp += v * v;
            for (double v : eta) ee += v * v;
            DDAMG_CUDA_TRY(cudaMemcpyAsync(B.th, th0.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, h->s));
            DDAMG_CUDA_TRY(cudaMemcpyAsync(B.p, p.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, h->s));
            // phi = D^dagger eta at the starting field; then S_f(start) = phi^dagger (D^dagger D)^-1 phi = |eta|^2
            launch_theta_to_links(h->s, B.th, h->lv[0].d.U, nl);
            DDAMG_CUDA_TRY(cudaMemcpyAsync(B.tmp, eta.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
            launch_wilson<double2>(h->s, h->lv[0].d.U, B.tmp, B.Y, nullptr, g.Nx, g.Nt, h->p.m0, 1, 1);
            DDAMG_CUDA_TRY(cudaMemcpyAsync(phi.data(), B.Y, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->s));
            sync(h);
            const double H0 = 0.5 * pp + host_gauge_action(th0, g.Nx, g.Nt, beta, nullptr) + ee;
            // leapfrog: half step in p, md_steps full steps in theta, half step at the end
            const double eps = tau / md_steps;
            int cg = hmc_force(h, B, phi, X, beta, cg_tol);
            launch_hmc_momentum(h->s, B.p, B.Fg, B.Ff, 0.5 * eps, nl);
            for (int k = 1; k <= md_steps; k++) {
                launch_hmc_theta(h->s, B.th, B.p, eps, nl);
                cg += hmc_force(h, B, phi, X, beta, cg_tol);
                launch_hmc_momentum(h->s, B.p, B.Fg, B.Ff, k < md_steps ? eps : 0.5 * eps, nl);
            }
            DDAMG_CUDA_TRY(cudaMemcpyAsync(th1.data(), B.th, sizeof(double) * nl, cudaMemcpyDeviceToHost, h->s));
            DDAMG_CUDA_TRY(cudaMemcpyAsync(p1.data(), B.p, sizeof(double) * nl, cudaMemcpyDeviceToHost, h->s));
            sync(h);
            double pp1 = 0.0, sf1 = 0.0;
            for (double v : p1) pp1 += v * v;
            for (long i = 0; i < 2 * n; i++) sf1 += phi[i] * X[i];  // Re(phi^dagger X), X solved at the end field
            const double H1 = 0.5 * pp1 + host_gauge_action(th1, g.Nx, g.Nt, beta, nullptr) + sf1;
            const double dH = H1 - H0;
            const double u = u01(rng64(seed, kStreamHmc, 3));
            const bool acc = std::isfinite(dH) && (dH <= 0.0 || u < std::exp(-dH));
            const std::vector<double>& out = acc ? th1 : th0;
            for (long i = 0; i < nl; i++) thw[i] = out[i] - 2.0 * kPi * std::floor((out[i] + kPi) / (2.0 * kPi));
            // the handle's gauge field becomes the returned one
            DDAMG_CUDA_TRY(cudaMemcpyAsync(B.th, thw.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, h->s));
            launch_theta_to_links(h->s, B.th, h->lv[0].d.U, nl);
            sync(h);
            h->setup_done = false;
            std::copy(thw.begin(), thw.end(), theta);  // every step has succeeded
            if (info) {
                info->accepted = acc ? 1 : 0;
                info->dH = dH;
                host_gauge_action(thw, g.Nx, g.Nt, beta, &info->plaquette);
                info->cg_iterations = cg;
                info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            }
            hmc_free(B);
            return DDAMG_OK;
        },
        [&]() { hmc_restore(h, B, th0); });
}

ddamg_status ddamg_link_derivative(ddamg_t* h, const double* psi, const double* lambda, double* out) {
    CHECK_HANDLE(h);
    API_BEGIN
    if (!h->gauge) throw ParamFailure{"no gauge field loaded"};
    LevelData& D = h->lv[0];
    const long n = D.g.size();
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.eta, psi, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(D.d.psi, lambda, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    double* g = reinterpret_cast<double*>(D.d.r);
    launch_link_derivative(h->s, D.d.U, D.d.eta, D.d.psi, g, D.g.Nx, D.g.Nt);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, g, sizeof(double) * 2 * D.g.sites, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    API_END
}

ddamg_status ddamg_gradient(ddamg_t* h, const double* eta, const double* b, double* out, ddamg_solve_info* info) {
    CHECK_HANDLE(h);
    API_BEGIN
    need_setup(h);
    LevelData& D = h->lv[0];
    const long n = D.g.size();
    const long sites = D.g.sites;
    ddamg_solve_info inf[2];
    if (!h->grad) h->grad = dalloc_t<double2>(h, 3 * (size_t)n);
    double2 *gpsi = h->grad, *glam = h->grad + n, *gtmp = h->grad + 2 * n;
    // psi = D^-1 b and lambda = D^-dagger eta = sigma_3 D^-1 sigma_3 eta (gamma_5-hermiticity):
    // one lockstep solve of both when the handle batches, else two solves
    DDAMG_CUDA_TRY(cudaMemcpyAsync(h->ob, b, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    DDAMG_CUDA_TRY(cudaMemcpyAsync(gtmp, eta, sizeof(double2) * n, cudaMemcpyHostToDevice, h->s));
    ddamg_status s1, s2;
    if (h->p.max_rhs >= 2) {
        launch_sigma3(h->s, gtmp, h->ob + n, sites);
        s1 = s2 = solve_device(h, h->ob, gpsi, 2, inf);  // psi then sigma_3 lambda, back to back
        DDAMG_CUDA_TRY(cudaMemcpyAsync(gtmp, glam, sizeof(double2) * n, cudaMemcpyDeviceToDevice, h->s));
    } else {
        s1 = solve_device(h, h->ob, gpsi, 1, &inf[0]);
        launch_sigma3(h->s, gtmp, h->ob, sites);
        s2 = solve_device(h, h->ob, gtmp, 1, &inf[1]);
    }
    launch_sigma3(h->s, gtmp, glam, sites);
    double* g = reinterpret_cast<double*>(gtmp);
    launch_link_derivative(h->s, D.d.U, gpsi, glam, g, D.g.Nx, D.g.Nt);
    DDAMG_CUDA_TRY(cudaMemcpyAsync(out, g, sizeof(double) * 2 * sites, cudaMemcpyDeviceToHost, h->s));
    sync(h);
    if (info) {
        info[0] = inf[0];
        info[1] = inf[1];
    }
    if (s1 != DDAMG_OK) return s1;
    if (s2 != DDAMG_OK) return s2;
    API_END
}

ddamg_status ddamg_gauge_metropolis(int Nx, int Nt, double beta, int sweeps, uint64_t seed, double delta,
                                    double* theta, double* acceptance, int device) {
    if (!theta || Nx < 2 || Nt < 2 || (Nx & 1) || (Nt & 1) || sweeps < 0) return DDAMG_ERR_BAD_PARAM;
    try {
        DDAMG_CUDA_TRY(cudaSetDevice(device));
        cudaStream_t s;
        DDAMG_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        double* th = nullptr;
        unsigned long long* acc = nullptr;
        DDAMG_CUDA_TRY(cudaMalloc(&th, sizeof(double) * 2 * Nx * Nt));
        DDAMG_CUDA_TRY(cudaMalloc(&acc, sizeof(unsigned long long)));
        launch_metropolis_init(s, th, Nx, Nt, seed);
        for (int sw = 0; sw < sweeps; sw++) {
            if (sw == sweeps - 1) DDAMG_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), s));
            for (int sub = 0; sub < 4; sub++) launch_metropolis_sub(s, th, Nx, Nt, beta, delta, seed, sw, sub, acc);
        }
        unsigned long long a = 0;
        DDAMG_CUDA_TRY(cudaMemcpyAsync(theta, th, sizeof(double) * 2 * Nx * Nt, cudaMemcpyDeviceToHost, s));
        DDAMG_CUDA_TRY(cudaMemcpyAsync(&a, acc, sizeof(a), cudaMemcpyDeviceToHost, s));
        DDAMG_CUDA_TRY(cudaStreamSynchronize(s));
        cudaFree(th);
        cudaFree(acc);
        cudaStreamDestroy(s);
        if (acceptance) *acceptance = sweeps > 0 ? (double)a / (2.0 * Nx * Nt) : 0.0;
    } catch (const CudaFailure&) {
        return DDAMG_ERR_CUDA;
    }
    return DDAMG_OK;
}

ddamg_status ddamg_gaussian_field(int64_t n, uint64_t seed, double* out) {
    if (!out || n < 0) return DDAMG_ERR_BAD_PARAM;
    const double pi = 3.14159265358979323846;
    for (int64_t i = 0; i < n; i++) {
        double u1 = u01(rng64(seed, kStreamGauss, (uint64_t)(2 * i)));
        double u2 = u01(rng64(seed, kStreamGauss, (uint64_t)(2 * i + 1)));
        double r = std::sqrt(-std::log(1.0 - u1));
        out[2 * i] = r * std::cos(2.0 * pi * u2);
        out[2 * i + 1] = r * std::sin(2.0 * pi * u2);
    }
    return DDAMG_OK;
}

}  // extern "C"
