// SAP colour sweep (SAP_C::SAP inner loops, src/sap.cpp:48-77 and 104-139): for every Schwarz
// block of one colour solve D_B e = r_B with GMRES(m) x restarts (FGMRES::fgmres with the identity
// preconditioner, src/fgmres.cpp:5-97, x0 = r_B as src/sap.cpp:65) and add e to x on the block.
// One CTA per (block, rhs); the block's Krylov basis lives in shared memory, the block-local
// operator (Level::SAP_level_l::D_local, src/level.cpp:607-653: neighbours outside the block
// read as zero, no boundary sign) streams the level's links.
#include "internal.h"

namespace ddamg {

__device__ __forceinline__ double2 level0_hop(const double2* __restrict__ U, int Nx, int Nt, int n, int h, int alf,
                                              int bet) {
    const int x = n / Nt, t = n - x * Nt;
    double2 u, coef;
    if (h == 1 || h == 3) {
        const double sgn = (h == 1) ? -1.0 : 1.0;
        coef = (alf == bet) ? make_double2(1.0, 0.0) : make_double2(sgn, 0.0);
        u = (h == 1) ? __ldg(U + 2 * n) : conjc(__ldg(U + 2 * (x * Nt + ((t == 0) ? Nt - 1 : t - 1))));
    } else {
        const double sgn = (h == 2) ? -1.0 : 1.0;
        if (alf == bet) coef = make_double2(1.0, 0.0);
        else coef = make_double2(0.0, (alf == 0 ? -1.0 : 1.0) * sgn);
        const int nxm = ((x == 0) ? Nx - 1 : x - 1) * Nt + t;
        u = (h == 2) ? __ldg(U + 2 * n + 1) : conjc(__ldg(U + 2 * nxm + 1));
    }
    return 0.5 * cmul(coef, u);
}
__device__ __forceinline__ float2 level0_hop(const float2* __restrict__ U, int Nx, int Nt, int n, int h, int alf,
                                             int bet) {
    const int x = n / Nt, t = n - x * Nt;
    float2 u, coef;
    if (h == 1 || h == 3) {
        const float sgn = (h == 1) ? -1.f : 1.f;
        coef = (alf == bet) ? make_float2(1.f, 0.f) : make_float2(sgn, 0.f);
        u = (h == 1) ? __ldg(U + 2 * n) : conjc(__ldg(U + 2 * (x * Nt + ((t == 0) ? Nt - 1 : t - 1))));
    } else {
        const float sgn = (h == 2) ? -1.f : 1.f;
        if (alf == bet) coef = make_float2(1.f, 0.f);
        else coef = make_float2(0.f, (alf == 0 ? -1.f : 1.f) * sgn);
        const int nxm = ((x == 0) ? Nx - 1 : x - 1) * Nt + t;
        u = (h == 2) ? __ldg(U + 2 * n + 1) : conjc(__ldg(U + 2 * nxm + 1));
    }
    return 0.5f * cmul(coef, u);
}

struct SapKParams {
    int m, restarts;
    double tol, m0;
    const int* blocks;
    int nblocks;
    const int* done;
};

// Shared-memory layout of one block solve
template <typename V> struct SapSmem {
    V* basis;      // (m+1) x NE
    V* op;         // NE: operand of D_B
    double2* red;  // 33
    double2* H;    // (m+1) x m, H[i*m + j]
    double2* gm;   // m+1
    double2* cn;   // m
    double2* sn;   // m
    double2* eta;  // m
    int* flag;     // [0] = maxIt
    __device__ SapSmem(unsigned char* raw, int m, int NE) {
        double2* d = reinterpret_cast<double2*>(raw);
        red = d;
        H = red + 33;
        gm = H + (m + 1) * m;
        cn = gm + (m + 1);
        sn = cn + m;
        eta = sn + m;
        flag = reinterpret_cast<int*>(eta + m);
        basis = reinterpret_cast<V*>(flag + 4);
        op = basis + (long)(m + 1) * NE;
    }
    static size_t bytes(int m, int NE) {
        return sizeof(double2) * (33 + (m + 1) * m + (m + 1) + 3 * m) + 4 * sizeof(int) +
               sizeof(V) * (size_t)(m + 2) * NE;
    }
};

template <typename V, bool DENSE, int EPT>
__global__ void __launch_bounds__(1024) sap_block_kernel(Geom g, const V* __restrict__ L, const V* __restrict__ rg,
                                                         V* __restrict__ xg, SapKParams p) {
    typedef typename RealOf<V>::R R;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int S = g.sel_x * g.sel_t, dof = g.dof, NE = S * dof;
    const int rhs = blockIdx.x / p.nblocks, kb = blockIdx.x - rhs * p.nblocks;
    if (p.done && p.done[rhs]) return;
    SapSmem<V> sm(smraw, p.m, NE);
    const int blk = p.blocks[kb];
    const int bx = blk / g.sap_t, bt = blk - bx * g.sap_t;
    const long ro = (long)rhs * g.size();
    const R mm = R(p.m0) + R(2);

    // element ownership: e = tid + q * blockDim
    int ek[EPT], ei[EPT], en[EPT], nbk[EPT][5];
    bool ev[EPT];
    V b[EPT], x[EPT], w[EPT];
#pragma unroll
    for (int q = 0; q < EPT; q++) {
        const int e = threadIdx.x + q * blockDim.x;
        ev[q] = e < NE;
        const int k = ev[q] ? e / dof : 0, i = ev[q] ? e - k * dof : 0;
        const int kx = k / g.sel_t, kt = k - kx * g.sel_t;
        ek[q] = k;
        ei[q] = i;
        en[q] = (bx * g.sel_x + kx) * g.Nt + bt * g.sel_t + kt;
        nbk[q][0] = k;
        nbk[q][1] = (kt + 1 < g.sel_t) ? k + 1 : -1;
        nbk[q][2] = (kx + 1 < g.sel_x) ? k + g.sel_t : -1;
        nbk[q][3] = (kt > 0) ? k - 1 : -1;
        nbk[q][4] = (kx > 0) ? k - g.sel_t : -1;
        b[q] = ev[q] ? rg[ro + (long)en[q] * dof + i] : czero<V>();
        x[q] = b[q];
    }

    // w = D_B op   (op in shared memory, fully written before the call)
    auto apply = [&](const V* op) {
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            if (!ev[q]) {
                w[q] = czero<V>();
                continue;
            }
            const int k = ek[q], i = ei[q], n = en[q];
            V acc = czero<V>();
            if (DENSE) {
#pragma unroll
                for (int d = 0; d < 5; d++) {
                    const int kk = nbk[q][d];
                    if (kk < 0) continue;
                    const V* M = L + ((long)n * 5 + d) * dof * dof + i;
                    const V* o = op + kk * dof;
                    for (int j = 0; j < dof; j++) acc = cfma(__ldg(M + (long)j * dof), o[j], acc);
                }
            } else {
#pragma unroll
                for (int d = 1; d < 5; d++) {
                    const int kk = nbk[q][d];
                    if (kk < 0) continue;
                    acc = cfma(level0_hop(L, g.Nx, g.Nt, n, d, i, 0), op[kk * 2], acc);
                    acc = cfma(level0_hop(L, g.Nx, g.Nt, n, d, i, 1), op[kk * 2 + 1], acc);
                }
            }
            w[q] = mm * op[k * dof + i] - acc;
        }
    };
    auto dot_own = [&](const V* a_sm) -> double2 {  // sum_own w * conj(a)
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < EPT; q++)
            if (ev[q]) s = cfmac(to_d(a_sm[threadIdx.x + q * blockDim.x]), to_d(w[q]), s);
        return block_sum(s, sm.red);
    };
    auto norm_of = [&](const V* v) -> double {  // over own registers v[EPT]
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < EPT; q++)
            if (ev[q]) s += (double)cnorm2(v[q]);
        return sqrt(block_sum(make_double2(s, 0.0), sm.red).x);
    };

    const int m = p.m;
    // x = x0 = b; r = b - D_B x
#pragma unroll
    for (int q = 0; q < EPT; q++)
        if (ev[q]) sm.op[threadIdx.x + q * blockDim.x] = x[q];
    __syncthreads();
    apply(sm.op);
#pragma unroll
    for (int q = 0; q < EPT; q++) w[q] = b[q] - w[q];  // w holds r
    const double norm_b = norm_of(b);
    double err = norm_of(w);
    int maxIt = m;
    // a zero block right-hand side has the zero solution (the reference would divide by zero)
    if (norm_b == 0.0) return;
    for (int k = 0; k < p.restarts; k++) {
        // V_0 = r / beta
        {
            const R inv = R(1.0 / err);
#pragma unroll
            for (int q = 0; q < EPT; q++)
                if (ev[q]) sm.basis[threadIdx.x + q * blockDim.x] = inv * w[q];
            if (threadIdx.x == 0) sm.gm[0] = make_double2(err, 0.0);
        }
        bool brk = false;
        for (int j = 0; j < m; j++) {
            __syncthreads();
            apply(sm.basis + (long)j * NE);  // w = D_B V_j
            for (int i = 0; i <= j; i++) {   // modified Gram-Schmidt (src/fgmres.cpp:28-40)
                const V* vi = sm.basis + (long)i * NE;
                const double2 h = dot_own(vi);
                if (threadIdx.x == 0) sm.H[i * m + j] = h;
                const V hv = from_d<V>(h);
#pragma unroll
                for (int q = 0; q < EPT; q++)
                    if (ev[q]) w[q] = w[q] - cmul(hv, vi[threadIdx.x + q * blockDim.x]);
            }
            const double hn = norm_of(w);
            if (hn > 0) {
                const R inv = R(1.0 / hn);
#pragma unroll
                for (int q = 0; q < EPT; q++)
                    if (ev[q]) sm.basis[(long)(j + 1) * NE + threadIdx.x + q * blockDim.x] = inv * w[q];
            }
            if (threadIdx.x == 0) {
                double2* H = sm.H;
                H[(j + 1) * m + j] = make_double2(hn, 0.0);
                for (int i = 0; i < j; i++) {  // FGMRES::rotation (src/fgmres.cpp:99-115)
                    double2 hij = H[i * m + j], hi1 = H[(i + 1) * m + j];
                    double2 tmp = cmulc(sm.cn[i], hij) + cmulc(sm.sn[i], hi1);
                    H[(i + 1) * m + j] = cmul(sm.cn[i], hi1) - cmul(sm.sn[i], hij);
                    H[i * m + j] = tmp;
                }
                double2 hjj = H[j * m + j], hj1 = H[(j + 1) * m + j];
                double den = sqrt(cnorm2(hjj) + cnorm2(hj1));
                sm.sn[j] = make_double2(hj1.x / den, hj1.y / den);
                sm.cn[j] = make_double2(hjj.x / den, hjj.y / den);
                H[j * m + j] = cmulc(sm.cn[j], hjj) + cmulc(sm.sn[j], hj1);
                H[(j + 1) * m + j] = make_double2(0.0, 0.0);
                sm.gm[j + 1] = -cmul(sm.sn[j], sm.gm[j]);
                sm.gm[j] = cmulc(sm.cn[j], sm.gm[j]);
                sm.flag[0] = (sqrt(cnorm2(sm.gm[j + 1])) < p.tol * norm_b) ? 1 : 0;
            }
            __syncthreads();
            if (sm.flag[0]) {
                maxIt = j + 1;
                brk = true;
                break;
            }
        }
        (void)brk;
        // solve_upper_triangular (src/fgmres.cpp:118-128)
        if (threadIdx.x == 0) {
            for (int i = maxIt - 1; i >= 0; i--) {
                double2 e = sm.gm[i];
                for (int jj = i + 1; jj < maxIt; jj++) e = e - cmul(sm.H[i * m + jj], sm.eta[jj]);
                sm.eta[i] = cdiv(e, sm.H[i * m + i]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            if (!ev[q]) continue;
            V acc = x[q];
            for (int jj = 0; jj < maxIt; jj++)
                acc = cfma(from_d<V>(sm.eta[jj]), sm.basis[(long)jj * NE + threadIdx.x + q * blockDim.x], acc);
            x[q] = acc;
            sm.op[threadIdx.x + q * blockDim.x] = acc;
        }
        __syncthreads();
        apply(sm.op);
#pragma unroll
        for (int q = 0; q < EPT; q++) w[q] = b[q] - w[q];
        err = norm_of(w);
        if (err < p.tol * norm_b) break;
    }
    // x_B += e  (src/sap.cpp:106-113)
#pragma unroll
    for (int q = 0; q < EPT; q++)
        if (ev[q]) {
            V* o = xg + ro + (long)en[q] * dof + ei[q];
            *o = *o + x[q];
        }
}

template <typename V, bool DENSE>
static void launch_sap(cudaStream_t s, const Geom& g, const V* L, const V* r, V* x, const SapArgs& a, int nrhs) {
    const int NE = g.sel_x * g.sel_t * g.dof;
    int threads = std::min(1024, ((NE + 31) / 32) * 32);
    int ept = (NE + threads - 1) / threads;
    size_t smem = SapSmem<V>::bytes(a.m, NE);
    SapKParams p{a.m, a.restarts, a.tol, a.m0, a.blocks, a.nblocks, a.done};
    dim3 grid(a.nblocks * nrhs);
    if (ept == 1) {
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(sap_block_kernel<V, DENSE, 1>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DDAMG_LAUNCH((sap_block_kernel<V, DENSE, 1>), grid, threads, smem, s, g, L, r, x, p);
    } else if (ept == 2) {
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(sap_block_kernel<V, DENSE, 2>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DDAMG_LAUNCH((sap_block_kernel<V, DENSE, 2>), grid, threads, smem, s, g, L, r, x, p);
    } else if (ept <= 4) {
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(sap_block_kernel<V, DENSE, 4>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DDAMG_LAUNCH((sap_block_kernel<V, DENSE, 4>), grid, threads, smem, s, g, L, r, x, p);
    } else {
        throw ParamFailure{"SAP block too large (more than 4096 unknowns per block)"};
    }
}
size_t sap_smem_bytes(int m, int NE, bool fp64) {
    return fp64 ? SapSmem<double2>::bytes(m, NE) : SapSmem<float2>::bytes(m, NE);
}

template <typename V>
void launch_sap_sweep_fine(cudaStream_t s, const Geom& g, const V* U, const V* r, V* x, const SapArgs& a, int nrhs) {
    launch_sap<V, false>(s, g, U, r, x, a, nrhs);
}
template <typename V>
void launch_sap_sweep_coarse(cudaStream_t s, const Geom& g, const V* links, const V* r, V* x, const SapArgs& a,
                             int nrhs) {
    launch_sap<V, true>(s, g, links, r, x, a, nrhs);
}
template void launch_sap_sweep_fine<double2>(cudaStream_t, const Geom&, const double2*, const double2*, double2*,
                                             const SapArgs&, int);
template void launch_sap_sweep_fine<float2>(cudaStream_t, const Geom&, const float2*, const float2*, float2*,
                                            const SapArgs&, int);
template void launch_sap_sweep_coarse<double2>(cudaStream_t, const Geom&, const double2*, const double2*, double2*,
                                               const SapArgs&, int);
template void launch_sap_sweep_coarse<float2>(cudaStream_t, const Geom&, const float2*, const float2*, float2*,
                                              const SapArgs&, int);

}  // namespace ddamg
