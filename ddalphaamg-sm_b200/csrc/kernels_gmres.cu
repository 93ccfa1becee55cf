// Coarsest-level solve (Level::GMRES_level_l, include/level.h:70-140: GMRES(m) x restarts with
// the identity preconditioner, x0 = b) as ONE persistent cooperative kernel: every CTA owns a
// slice of coarse sites, applies the level operator to it, and the CTAs meet at a bounded grid
// barrier between phases.  Orthogonalisation is classical Gram-Schmidt with one
// re-orthogonalisation pass (CGS2); the Hessenberg/Givens work is repeated by every CTA on
// identical data so control flow stays uniform without broadcasts.
#include "internal.h"

#include <mutex>

namespace ddamg {

constexpr long long kSpinLimit = 1LL << 24;  // default: ~1-2 s of polling before a barrier gives up

// Bounded grid barrier: arrive on bar[0], wait for the generation bar[1] to move.  On timeout
// (or when another CTA already failed) it sets status[0] and returns false; callers return.
// Every CTA of the cooperative grid is resident, so a CTA that gives up only makes the others
// leave at their next wait: the kernel always ends.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, unsigned nblocks, long long limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = bar + 1;
        volatile int* vst = status;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        int good = 1;
        if (arrived == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*vgen == gen) {
                if (*vst != 0) {
                    good = 0;
                    break;
                }
                if (++spins > limit) {
                    atomicExch(status, 1);
                    good = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = good && (*vst == 0);
    }
    __syncthreads();
    return ok != 0;
}

struct GmresK {
    const double2* links;
    const double2* b;
    double2* x;
    double2* V;
    double2* w;
    double2* partial;  // 3 buffers of grid x P
    double2* H;        // column j at H + j*(m+1)
    unsigned* bar;
    int* status;
    int Nx, Nt, dof, m, restarts, P;
    double m0, tol;
    long long spin_limit;
};

// out = [b -] D in on this CTA's sites.  The CTA's (site, direction) pairs are spread over its
// warps (lane = output dof, NI = dof/32 rounded up); each pair leaves its partial product in
// shared memory and the five partials of a site are summed in a fixed order.
template <int NI>
__device__ void apply_own(const GmresK& k, const double2* __restrict__ in, double2* __restrict__ out,
                          const double2* __restrict__ bsub, int s0, int s1, double2* __restrict__ part,
                          double scale = 1.0) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int dof = k.dof, Nt = k.Nt, Nx = k.Nx;
    const int ntask = (s1 - s0) * 5;
    constexpr int CB = NI == 1 ? 16 : 4;  // column loads in flight per lane
    for (int task = wid; task < ntask; task += nw) {
        const int sl = task / 5, d = task - sl * 5;
        const int n = s0 + sl;
        const int x = n / Nt, t = n - x * Nt;
        int nb;
        double sg = 1.0;
        switch (d) {
            case 0: nb = n; break;
            case 1: nb = x * Nt + ((t + 1 == Nt) ? 0 : t + 1); sg = (t == Nt - 1) ? -1.0 : 1.0; break;
            case 2: nb = ((x + 1 == Nx) ? 0 : x + 1) * Nt + t; break;
            case 3: nb = x * Nt + ((t == 0) ? Nt - 1 : t - 1); sg = (t == 0) ? -1.0 : 1.0; break;
            default: nb = ((x == 0) ? Nx - 1 : x - 1) * Nt + t; break;
        }
        double2 vd[NI], acc[NI];
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const int i = lane + 32 * q;
            vd[q] = (i < dof) ? sg * in[(long)nb * dof + i] : make_double2(0.0, 0.0);
            acc[q] = make_double2(0.0, 0.0);
        }
        const double2* M = k.links + ((long)n * 5 + d) * dof * dof;
#pragma unroll
        for (int jq = 0; jq < NI; jq++) {
            const int jn = min(32, dof - 32 * jq);
            for (int j0 = 0; j0 < jn; j0 += CB) {
                double2 mv[CB][NI];
#pragma unroll
                for (int u = 0; u < CB; u++)
#pragma unroll
                    for (int q = 0; q < NI; q++) {
                        const int i = lane + 32 * q;
                        mv[u][q] = (j0 + u < jn && i < dof) ? __ldg(M + (long)(32 * jq + j0 + u) * dof + i)
                                                            : make_double2(0.0, 0.0);
                    }
#pragma unroll
                for (int u = 0; u < CB; u++) {
                    if (j0 + u >= jn) break;
                    const double2 vj = make_double2(__shfl_sync(0xffffffffu, vd[jq].x, j0 + u),
                                                    __shfl_sync(0xffffffffu, vd[jq].y, j0 + u));
#pragma unroll
                    for (int q = 0; q < NI; q++) acc[q] = cfma(mv[u][q], vj, acc[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const int i = lane + 32 * q;
            if (i < dof) part[(sl * 5 + d) * dof + i] = (d == 0) ? (k.m0 + 2.0) * vd[q] - acc[q] : acc[q];
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < (s1 - s0) * dof; e += blockDim.x) {
        const int sl = e / dof, i = e - sl * dof;
        const double2* pp = part + sl * 5 * dof + i;
        double2 o = scale * (pp[0] - pp[dof] - pp[2 * dof] - pp[3 * dof] - pp[4 * dof]);
        const long ge = (long)(s0 + sl) * dof + i;
        if (bsub) o = bsub[ge] - o;
        out[ge] = o;
    }
}

// partial[blk*P + i] = sum_own w * conj(V_i), i < cnt (warp per i)
__device__ void partial_dots(const GmresK& k, const double2* __restrict__ w, int cnt, double2* __restrict__ part,
                             long e0, long e1, long n) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = wid; i < cnt; i += nw) {
        const double2* vi = k.V + (long)i * n;
        double2 s = make_double2(0.0, 0.0);
        for (long e = e0 + lane; e < e1; e += 32) s = cfmac(vi[e], w[e], s);
        s = warp_sum(s);
        if (lane == 0) part[(long)blockIdx.x * k.P + i] = s;
    }
}
// the same with slot cnt = ||w||^2: the Gram-Schmidt coefficients and the norm in one reduction
__device__ void partial_dots_norm(const GmresK& k, const double2* __restrict__ w, int cnt, double2* __restrict__ part,
                                  long e0, long e1, long n) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = wid; i <= cnt; i += nw) {
        const double2* vi = i < cnt ? k.V + (long)i * n : w;
        double2 s = make_double2(0.0, 0.0);
        for (long e = e0 + lane; e < e1; e += 32) s = cfmac(vi[e], w[e], s);
        s = warp_sum(s);
        if (lane == 0) part[(long)blockIdx.x * k.P + i] = s;
    }
}
// h[i] = sum_blk partial[blk*P + i]: one warp per coefficient, lanes stride over the CTAs' partials,
// a shuffle tree finishes; every CTA runs the identical order, so all CTAs hold identical sums
__device__ void reduce_partials(const GmresK& k, const double2* __restrict__ part, int cnt, double2* h) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = wid; i < cnt; i += nw) {
        double2 s = make_double2(0.0, 0.0);
        for (int bk = lane; bk < (int)gridDim.x; bk += 32) s += part[(long)bk * k.P + i];
        s = warp_sum(s);
        if (lane == 0) h[i] = s;
    }
    __syncthreads();
}
// sum over the CTAs of the first slot of pC (norms), same order in every CTA
__device__ double2 reduce_slot0(const GmresK& k, const double2* __restrict__ part, double2* tmp) {
    if (threadIdx.x < 32) {
        double2 s = make_double2(0.0, 0.0);
        for (int bk = threadIdx.x; bk < (int)gridDim.x; bk += 32) s += part[(long)bk * k.P];
        s = warp_sum(s);
        if (threadIdx.x == 0) *tmp = s;
    }
    __syncthreads();
    return *tmp;
}

constexpr int kHs = 48;
// threads per CTA: 16 warps, so the (site, direction) matrix products of a CTA's two sites stream at once
constexpr int kCoarseThreads = 512;  // Hessenberg columns every CTA keeps for its own triangular solve

// The Krylov basis is stored unnormalised: slot i of V holds u_i with v_i = sc[i] u_i (sc in shared
// memory, identical in every CTA).  An Arnoldi step reduces the Gram-Schmidt coefficients and ||w||^2
// together (one grid barrier), forms ||w - V h||^2 = ||w||^2 - sum |h_i|^2, writes u_{j+1} and
// publishes it with a second barrier; only where that difference cancels below 1e-4 of ||w||^2 (so that
// it would lose digits) does it run a second Gram-Schmidt pass (classical Gram-Schmidt twice, whose norm
// barrier publishes u_{j+1}), as the SAP block solvers do.  Every CTA keeps the rotated Hessenberg triangle of the first kHs columns, so the
// triangular solve at a restart end needs no barrier.
template <int NI>
__global__ void __launch_bounds__(kCoarseThreads) coarse_gmres_kernel(GmresK k) {
    extern __shared__ double2 sh[];
    const int m = k.m;
    double2* h = sh;              // m+1
    double2* h2 = h + (m + 1);    // m+1
    double2* gm = h2 + (m + 1);   // m+1
    double2* cn = gm + (m + 1);   // m
    double2* sn = cn + m;         // m
    double2* eta = sn + m;        // m
    double* sc = reinterpret_cast<double*>(eta + m);  // m+1 scale factors (m+1 double2 reserved)
    double2* hs = eta + m + (m + 1);    // kHs (kHs + 1) / 2: the rotated Hessenberg triangle of the first kHs columns
    double2* part = hs + kHs * (kHs + 1) / 2;  // sites per CTA x 5 x dof: per-direction partial products
    __shared__ int s_flag;
    __shared__ double2 s_sum;
    const unsigned G = gridDim.x;
    const int sites = k.Nx * k.Nt;
    const long n = (long)sites * k.dof;
    const int spc = (sites + G - 1) / G;
    const int s0 = min(sites, (int)blockIdx.x * spc), s1 = min(sites, s0 + spc);
    const long e0 = (long)s0 * k.dof, e1 = (long)s1 * k.dof;
    double2* pA = k.partial;
    double2* pB = pA + (long)G * k.P;
    double2* pC = pB + (long)G * k.P;
    double2* u0 = k.V;  // the residual lands in slot 0

    // x = x0 = b
    for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) k.x[e] = k.b[e];
    if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
    apply_own<NI>(k, k.x, u0, k.b, s0, s1, part);  // u_0 = r = b - D x
    __syncthreads();
    {
        double rr = 0.0, bb = 0.0;
        for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            rr += cnorm2(u0[e]);
            bb += cnorm2(k.b[e]);
        }
        __shared__ double2 red[33];
        double2 t = block_sum(make_double2(rr, bb), red);
        if (threadIdx.x == 0) pC[(long)blockIdx.x * k.P] = t;
    }
    if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
    double err, norm_b;
    {
        const double2 t = reduce_slot0(k, pC, &s_sum);
        err = sqrt(t.x);
        norm_b = sqrt(t.y);
    }
    int maxIt = m, iters = k.restarts * m;
    bool converged = false;
    if (norm_b == 0.0) {  // zero right-hand side: x = 0 (the reference would divide by zero)
        for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) k.x[e] = make_double2(0.0, 0.0);
        iters = 0;
        converged = true;
    }
    for (int kk = 0; kk < k.restarts && !converged; kk++) {
        if (threadIdx.x == 0) {
            gm[0] = make_double2(err, 0.0);
            sc[0] = 1.0 / err;  // v_0 = r / ||r||
        }
        __syncthreads();
        for (int j = 0; j < m; j++) {
            // w = D v_j = sc_j D u_j (u_j of the neighbours was published by the last barrier)
            apply_own<NI>(k, k.V + (long)j * n, k.w, nullptr, s0, s1, part, sc[j]);
            __syncthreads();
            // (u_i, w) for i <= j and ||w||^2 in one reduction
            partial_dots_norm(k, k.w, j + 1, pA, e0, e1, n);
            if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
            reduce_partials(k, pA, j + 2, h);
            for (int i = threadIdx.x; i <= j; i += blockDim.x) h[i] = sc[i] * h[i];  // h_i = (v_i, w)
            __syncthreads();
            // ||w - V h||^2 = ||w||^2 - sum |h_i|^2; a second Gram-Schmidt pass only where that difference
            // cancels below 1e-4 of ||w||^2 (identical in every CTA)
            double hh = 0.0;
            for (int i = 0; i <= j; i++) hh += cnorm2(h[i]);
            const double w2 = h[j + 1].x, d2 = w2 - hh;
            const bool reorth = !(d2 > 1e-4 * w2);
            double2* un = k.V + (long)(j + 1) * n;  // u_{j+1}, unnormalised
            double hn;
            if (!reorth) {
                for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                    double2 a = k.w[e];
                    for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h[i], k.V[(long)i * n + e]);
                    un[e] = a;
                }
                hn = sqrt(d2);
                if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;  // publishes u_{j+1}
            } else {
                // w -= V h ; reorthogonalise
                for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                    double2 a = k.w[e];
                    for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h[i], k.V[(long)i * n + e]);
                    k.w[e] = a;
                }
                __syncthreads();
                partial_dots(k, k.w, j + 1, pB, e0, e1, n);
                if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
                reduce_partials(k, pB, j + 1, h2);
                for (int i = threadIdx.x; i <= j; i += blockDim.x) h2[i] = sc[i] * h2[i];
                __syncthreads();
                {
                    double ss = 0.0;
                    for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                        double2 a = k.w[e];
                        for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h2[i], k.V[(long)i * n + e]);
                        un[e] = a;
                        ss += cnorm2(a);
                    }
                    __shared__ double2 red2[33];
                    double2 t = block_sum(make_double2(ss, 0.0), red2);
                    if (threadIdx.x == 0) pC[(long)blockIdx.x * k.P] = t;
                }
                for (int i = threadIdx.x; i <= j; i += blockDim.x) h[i] = h[i] + h2[i];
                if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;  // also publishes u_{j+1}
                hn = sqrt(reduce_slot0(k, pC, &s_sum).x);
            }
            if (threadIdx.x == 0) {  // FGMRES::rotation (src/fgmres.cpp:99-115) on column j
                sc[j + 1] = hn > 0 ? 1.0 / hn : 0.0;
                h[j + 1] = make_double2(hn, 0.0);
                for (int i = 0; i < j; i++) {
                    double2 tmp = cmulc(cn[i], h[i]) + cmulc(sn[i], h[i + 1]);
                    h[i + 1] = cmul(cn[i], h[i + 1]) - cmul(sn[i], h[i]);
                    h[i] = tmp;
                }
                const double den = sqrt(cnorm2(h[j]) + cnorm2(h[j + 1]));
                sn[j] = make_double2(h[j + 1].x / den, h[j + 1].y / den);
                cn[j] = make_double2(h[j].x / den, h[j].y / den);
                h[j] = cmulc(cn[j], h[j]) + cmulc(sn[j], h[j + 1]);
                h[j + 1] = make_double2(0.0, 0.0);
                gm[j + 1] = -cmul(sn[j], gm[j]);
                gm[j] = cmulc(cn[j], gm[j]);
                s_flag = (sqrt(cnorm2(gm[j + 1])) < k.tol * norm_b) ? 1 : 0;
            }
            __syncthreads();
            if (j < kHs)  // this CTA's own copy of the rotated column (identical in every CTA)
                for (int i = threadIdx.x; i <= j; i += blockDim.x) hs[j * (j + 1) / 2 + i] = h[i];
            if (blockIdx.x == 0)
                for (int i = threadIdx.x; i <= j; i += blockDim.x) k.H[(long)j * (m + 1) + i] = h[i];
            if (s_flag) {  // identical in every CTA
                maxIt = j + 1;
                break;
            }
        }
        // solve_upper_triangular (src/fgmres.cpp:118-128)
        if (maxIt <= kHs) {  // from this CTA's own triangle, by one thread, in the reference's row order
            __syncthreads();
            if (threadIdx.x == 0)
                for (int i = maxIt - 1; i >= 0; i--) {
                    double2 e = gm[i];
                    for (int q = i + 1; q < maxIt; q++) e = e - cmul(hs[q * (q + 1) / 2 + i], eta[q]);
                    eta[i] = cdiv(e, hs[i * (i + 1) / 2 + i]);
                }
        } else {  // column-oriented from block 0's columns in global memory
            if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;  // the Hessenberg columns visible
            for (int i = threadIdx.x; i < maxIt; i += blockDim.x) eta[i] = gm[i];
            __syncthreads();
            for (int i = maxIt - 1; i >= 0; i--) {
                if (threadIdx.x == 0) eta[i] = cdiv(eta[i], k.H[(long)i * (m + 1) + i]);
                __syncthreads();
                for (int q = threadIdx.x; q < i; q += blockDim.x) eta[q] = eta[q] - cmul(k.H[(long)i * (m + 1) + q], eta[i]);
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < maxIt; i += blockDim.x) eta[i] = sc[i] * eta[i];  // x += sum eta_i v_i
        __syncthreads();
        for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            double2 a = k.x[e];
            for (int jj = 0; jj < maxIt; jj++) a = cfma(eta[jj], k.V[(long)jj * n + e], a);
            k.x[e] = a;
        }
        if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
        apply_own<NI>(k, k.x, u0, k.b, s0, s1, part);  // new residual into slot 0
        __syncthreads();
        {
            double rr = 0.0;
            for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) rr += cnorm2(u0[e]);
            __shared__ double2 red3[33];
            double2 t = block_sum(make_double2(rr, 0.0), red3);
            if (threadIdx.x == 0) pC[(long)blockIdx.x * k.P] = t;
        }
        if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
        err = sqrt(reduce_slot0(k, pC, &s_sum).x);
        if (err < k.tol * norm_b) {
            iters = kk * m + maxIt;
            converged = true;
        }
        // pC is rewritten only after the next barrier, so no CTA can still be reading it then
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) k.status[1] = iters;
}

// CTAs of the coarsest solve: about two coarse sites per CTA, at most one CTA per SM
int coarse_gmres_grid(long sites, int sms) { return (int)std::min<long>(sms, std::max<long>(1, (sites + 1) / 2)); }
static size_t coarse_gmres_smem(long sites, int grid, int m, int dof) {
    const long spc = (sites + grid - 1) / grid;
    return sizeof(double2) * ((size_t)7 * (m + 1) + (size_t)kHs * (kHs + 1) / 2 + (size_t)spc * 5 * dof);
}

void coarse_gmres_prepare(CoarseGmresWork& w, int n, int m, int dof, int device) {
    int sms = 0;
    DDAMG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = coarse_gmres_grid(n / dof, sms);
    size_t smem = coarse_gmres_smem(n / dof, grid, m, dof);
    if (smem > 227 * 1024) throw ParamFailure{"coarsest GMRES restart length too large for shared memory"};
    int per_sm = 0;
    if (dof <= 32) {
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(coarse_gmres_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
        DDAMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, coarse_gmres_kernel<1>, kCoarseThreads, smem));
    } else {
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(coarse_gmres_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
        DDAMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, coarse_gmres_kernel<2>, kCoarseThreads, smem));
    }
    if (per_sm < 1) throw ParamFailure{"coarsest GMRES kernel cannot be resident"};
    w.grid = grid;
    w.block = kCoarseThreads;
}

void launch_coarse_gmres(cudaStream_t s, const CoarseGmresWork& w, const double2* links, const double2* b,
                         double2* x, int Nx, int Nt, int dof, double m0, int m, int restarts, double tol) {
    GmresK k;
    k.links = links;
    k.b = b;
    k.x = x;
    k.V = w.V;
    k.w = w.w;
    k.partial = w.partial;
    k.H = w.H;
    k.bar = w.bar;
    k.status = w.status;
    k.Nx = Nx;
    k.Nt = Nt;
    k.dof = dof;
    k.m = m;
    k.restarts = restarts;
    k.P = m + 2;
    k.m0 = m0;
    k.tol = tol;
    k.spin_limit = w.spin_limit > 0 ? w.spin_limit : kSpinLimit;
    DDAMG_CUDA_TRY(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned), s));
    DDAMG_CUDA_TRY(cudaMemsetAsync(w.status, 0, 2 * sizeof(int), s));
    size_t smem = coarse_gmres_smem((long)Nx * Nt, w.grid, m, dof);
    void* args[] = {&k};
    if (dof <= 32)
        DDAMG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)coarse_gmres_kernel<1>, dim3(w.grid), dim3(w.block),
                                                   args, smem, s));
    else
        DDAMG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)coarse_gmres_kernel<2>, dim3(w.grid), dim3(w.block),
                                                   args, smem, s));
    ++g_launches;
}

// ---------------------------------------------------------------- allocation-free coarsest solve
// Some callers cannot allocate device memory when they solve: a host framework that owns every
// device allocation through its own memory pool and forbids others, or a time-critical loop that
// cannot pay for the implicit device synchronisation of cudaMalloc / cudaFree.  For them the
// coarsest-level GMRES runs out of one fixed scratch array compiled into the library instead of a
// handle's workspace.  The array is device memory of every GPU on which this code is loaded and
// stays allocated until the process exits.
constexpr size_t kNoAllocScratch = (size_t)1 << 21;  // complex FP64 values: 32 MiB
static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratch];
constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static double2* g_noalloc_base[kNoAllocMaxDevices] = {};

}  // namespace ddamg

extern "C" ddamg_status ddamg_coarse_gmres_noalloc(const void* links, const void* b, void* x, int Nx, int Nt, int dof,
                                                   double m0, int m, int restarts, double tol, void* stream,
                                                   int* iterations) {
    using namespace ddamg;
    if (!links || !b || !x || Nx < 1 || Nt < 1 || dof < 2 || dof > 64 || (dof & 1) || m < 1 || restarts < 1) {
        set_error("ddamg_coarse_gmres_noalloc: bad argument");
        return DDAMG_ERR_BAD_PARAM;
    }
    try {
        int dev = 0, sms = 0;
        DDAMG_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kNoAllocMaxDevices) {
            set_error("ddamg_coarse_gmres_noalloc: device ordinal out of range");
            return DDAMG_ERR_BAD_PARAM;
        }
        DDAMG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const long sites = (long)Nx * Nt, n = sites * dof;
        const long grid = coarse_gmres_grid(sites, sms);
        // scratch: Krylov basis (m+1) n, w n, 3 partial-sum buffers, Hessenberg (m+1) m, 2 control words
        const long need = (long)(m + 1) * n + n + 3 * grid * (m + 2) + (long)(m + 1) * m + 2;
        if (need > (long)kNoAllocScratch || coarse_gmres_smem(sites, (int)grid, m, dof) > 227 * 1024) {
            set_error("ddamg_coarse_gmres_noalloc: the solve needs " + std::to_string(need) +
                      " complex values of scratch; the fixed array holds " + std::to_string(kNoAllocScratch) +
                      " ((m+2)*n + (m+1)*m + 3*G*(m+2) + 2 must fit, G = min(SMs, sites/2))");
            return DDAMG_ERR_BAD_PARAM;
        }
        double2* base;
        {
            std::lock_guard<std::mutex> lk(g_noalloc_mutex);
            if (!g_noalloc_base[dev]) {  // once per device, with that device current
                void* p = nullptr;
                DDAMG_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
                g_noalloc_base[dev] = static_cast<double2*>(p);
            }
            base = g_noalloc_base[dev];
        }
        CoarseGmresWork w;
        coarse_gmres_prepare(w, (int)n, m, dof, dev);
        if (w.grid != grid) {
            set_error("ddamg_coarse_gmres_noalloc: unexpected grid size");
            return DDAMG_ERR_STATE;
        }
        w.V = base;
        w.w = w.V + (long)(m + 1) * n;
        w.r = nullptr;
        w.partial = w.w + n;
        w.H = w.partial + 3 * grid * (m + 2);
        w.bar = reinterpret_cast<unsigned*>(w.H + (long)(m + 1) * m);
        w.status = reinterpret_cast<int*>(w.bar + 2);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // the barrier words and status are zeroed inside; the rest is written before it is read
        launch_coarse_gmres(s, w, static_cast<const double2*>(links), static_cast<const double2*>(b),
                            static_cast<double2*>(x), Nx, Nt, dof, m0, m, restarts, tol);
        int st[2] = {0, 0};
        DDAMG_CUDA_TRY(cudaMemcpyAsync(st, w.status, sizeof(st), cudaMemcpyDeviceToHost, s));
        DDAMG_CUDA_TRY(cudaStreamSynchronize(s));
        if (st[0] != 0) {
            set_error("ddamg_coarse_gmres_noalloc: a bounded grid barrier gave up");
            return DDAMG_ERR_DEVICE_TIMEOUT;
        }
        if (iterations) *iterations = st[1];
    } catch (const CudaFailure&) {
        return DDAMG_ERR_CUDA;
    } catch (const ParamFailure& e) {
        set_error(e.msg);
        return DDAMG_ERR_BAD_PARAM;
    }
    return DDAMG_OK;
}
