// Coarsest-level solve (Level::GMRES_level_l, include/level.h:70-140: GMRES(m) x restarts with
// the identity preconditioner, x0 = b) as ONE persistent cooperative kernel: every CTA owns a
// slice of coarse sites, applies the level operator to it, and the CTAs meet at a bounded grid
// barrier between phases.  Orthogonalisation is classical Gram-Schmidt with one
// re-orthogonalisation pass (CGS2); the Hessenberg/Givens work is repeated by every CTA on
// identical data so control flow stays uniform without broadcasts.
#include "internal.h"

#include <cooperative_groups.h>
#include <mutex>

namespace ddamg {

constexpr long long kSpinLimit = 1LL << 24;  // default: ~1-2 s of polling before a barrier gives up

// Bounded grid barrier on a counter that only grows (zeroed per launch): a CTA arrives with one atomic
// add and waits until the counter reaches the next multiple of the grid size, so the last arrival itself
// releases the others (no reset and no separate generation word: two L2 round trips fewer than a
// generation barrier).  On timeout (or when another CTA already failed) it sets status[0] and returns
// false; callers return.  Every CTA of the cooperative grid is resident, so a CTA that gives up only makes
// the others leave at their next wait: the kernel always ends.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, unsigned nblocks, long long limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vb = bar;
        volatile int* vst = status;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        const unsigned target = (arrived / nblocks + 1) * nblocks;
        int good = 1;
        long long spins = 0;
        while ((int)(*vb - target) < 0) {
            if (*vst != 0) {
                good = 0;
                break;
            }
            if (++spins > limit) {
                atomicExch(status, 1);
                good = 0;
                break;
            }
            __nanosleep(32);
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
    int ncache;  // link matrices of the CTA's (site, direction) pairs kept in shared memory, in task order
    int nbs;     // basis slots whose slice of this CTA's sites is kept in shared memory
};

// out = [b -] D in on this CTA's sites.  The CTA's (site, direction) pairs are spread over its
// warps (lane = output dof, NI = dof/32 rounded up); each pair leaves its partial product in
// shared memory and the five partials of a site are summed in a fixed order.
template <int NI>
__device__ void apply_own(const GmresK& k, const double2* __restrict__ in, double2* __restrict__ out,
                          const double2* __restrict__ bsub, int s0, int s1, double2* __restrict__ part,
                          double scale = 1.0, const double2* lcache = nullptr, long obase = 0) {
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
        const bool incache = lcache && task < k.ncache;
        const double2* M = incache ? lcache + (long)task * dof * dof : k.links + ((long)n * 5 + d) * dof * dof;
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
                        const long o = (long)(32 * jq + j0 + u) * dof + i;
                        mv[u][q] = (j0 + u < jn && i < dof) ? (incache ? M[o] : __ldg(M + o)) : make_double2(0.0, 0.0);
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
        out[ge - obase] = o;
    }
}

// This CTA's slice of the Krylov basis: slots below nbs in shared memory (vc, ls values per slot,
// indexed from e0), the others in global memory; w lives in shared memory (wl, indexed from e0).
struct BasisSlice {
    const GmresK* k;
    double2* vc;
    long ls, e0, n;
    __device__ double2 get(int i, long e) const {
        return i < k->nbs ? vc[(long)i * ls + (e - e0)] : k->V[(long)i * n + e];
    }
    __device__ void put(int i, long e, double2 a) const {  // the global copy is what the neighbours read
        k->V[(long)i * n + e] = a;
        if (i < k->nbs) vc[(long)i * ls + (e - e0)] = a;
    }
};

// partial[blk*P + i] = sum_own w * conj(V_i), i < cnt (warp per i)
__device__ void partial_dots(const GmresK& k, const BasisSlice& V, const double2* __restrict__ wl, int cnt,
                             double2* __restrict__ part, long e0, long e1) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = wid; i < cnt; i += nw) {
        double2 s = make_double2(0.0, 0.0);
        for (long e = e0 + lane; e < e1; e += 32) s = cfmac(V.get(i, e), wl[e - e0], s);
        s = warp_sum(s);
        if (lane == 0) part[(long)blockIdx.x * k.P + i] = s;
    }
}
// the same with slot cnt = ||w||^2: the Gram-Schmidt coefficients and the norm in one reduction
__device__ void partial_dots_norm(const GmresK& k, const BasisSlice& V, const double2* __restrict__ wl, int cnt,
                                  double2* __restrict__ part, long e0, long e1) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = wid; i <= cnt; i += nw) {
        double2 s = make_double2(0.0, 0.0);
        for (long e = e0 + lane; e < e1; e += 32) s = cfmac(i < cnt ? V.get(i, e) : wl[e - e0], wl[e - e0], s);
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

// FGMRES::rotation (src/fgmres.cpp:99-115) on column j of h (h[0..j] the Gram-Schmidt coefficients,
// hn2 = ||u_{j+1}||^2), with one reciprocal square root per norm (1 ulp) instead of a square root and
// divisions: the previous rotations, the new one, the residual estimate g and the scale of v_{j+1}; *flag
// says whether |g_{j+1}| < tol ||b|| (compared squared, tol2 = (tol ||b||)^2).  One thread.
__device__ __forceinline__ void coarse_rotation(double2* h, double2* gm, double2* cn, double2* sn, double* sc, int j,
                                                double hn2, double tol2, int* flag) {
    const double ihn = hn2 > 0 ? rsqrt(hn2) : 0.0;
    sc[j + 1] = ihn;
    h[j + 1] = make_double2(hn2 * ihn, 0.0);
    for (int i = 0; i < j; i++) {
        double2 tmp = cmulc(cn[i], h[i]) + cmulc(sn[i], h[i + 1]);
        h[i + 1] = cmul(cn[i], h[i + 1]) - cmul(sn[i], h[i]);
        h[i] = tmp;
    }
    const double iden = rsqrt(cnorm2(h[j]) + cnorm2(h[j + 1]));
    sn[j] = make_double2(h[j + 1].x * iden, h[j + 1].y * iden);
    cn[j] = make_double2(h[j].x * iden, h[j].y * iden);
    h[j] = cmulc(cn[j], h[j]) + cmulc(sn[j], h[j + 1]);
    h[j + 1] = make_double2(0.0, 0.0);
    gm[j + 1] = -cmul(sn[j], gm[j]);
    gm[j] = cmulc(cn[j], gm[j]);
    *flag = cnorm2(gm[j + 1]) < tol2 ? 1 : 0;
}

constexpr int kHs = 48;
// dynamic shared memory a CTA of these kernels may take: the 227 KB opt-in limit less room for their
// static shared variables
constexpr size_t kDynSmemCap = 227 * 1024 - 4096;
// threads per CTA: 16 warps, so the (site, direction) matrix products of a CTA's two sites stream at once
constexpr int kCoarseThreads = 512;  // Hessenberg columns every CTA keeps for its own triangular solve

// The Krylov basis is stored unnormalised: slot i of V holds u_i with v_i = sc[i] u_i (sc in shared
// memory, identical in every CTA).  An Arnoldi step reduces the Gram-Schmidt coefficients and ||w||^2
// together (one grid barrier), forms ||w - V h||^2 = ||w||^2 - sum |h_i|^2, writes u_{j+1} and
// publishes it with a second barrier; only where that difference cancels below 1e-4 of ||w||^2 (so that
// it would lose digits) does it run a second Gram-Schmidt pass (classical Gram-Schmidt twice, whose norm
// barrier publishes u_{j+1}), as the SAP block solvers do.  Every CTA keeps the rotated Hessenberg
// triangle of the first kHs columns, so the triangular solve at a restart end needs no barrier.
// Phase timing (clock64 marks, 256x256 bench workload, cycles per Arnoldi step) showed the operator
// application streaming the CTA's link matrices from L2 (7.0 K), two grid barriers (5.3 K each), the
// partial-sum reduction (3.0 K), the update (2.6 K) and the rotation on one thread (3.3 K).  So the CTA
// keeps its own link matrices (they do not change during a solve), its slice of the first basis
// vectors and w in shared memory, and the rotation uses one reciprocal square root instead of a
// square root and divisions.
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
    const unsigned G = gridDim.x;
    const int sites = k.Nx * k.Nt;
    const long n = (long)sites * k.dof;
    const int spc = (sites + G - 1) / G;
    double2* part = hs + kHs * (kHs + 1) / 2;  // spc x 5 x dof: per-direction partial products
    double2* wl = part + (long)spc * 5 * k.dof;        // spc x dof: this CTA's slice of w
    double2* lcache = wl + (long)spc * k.dof;           // ncache link matrices
    double2* vc = lcache + (long)k.ncache * k.dof * k.dof;  // nbs slots of spc x dof
    __shared__ int s_flag;
    __shared__ double2 s_sum;
    const int s0 = min(sites, (int)blockIdx.x * spc), s1 = min(sites, s0 + spc);
    const long e0 = (long)s0 * k.dof, e1 = (long)s1 * k.dof;
    const BasisSlice V{&k, vc, (long)spc * k.dof, e0, n};
    double2* pA = k.partial;
    double2* pB = pA + (long)G * k.P;
    double2* pC = pB + (long)G * k.P;
    double2* u0 = k.V;  // the residual lands in slot 0
    {  // the CTA's link matrices, task order (site, direction)
        const long dd = (long)k.dof * k.dof;
        const int nc = min(k.ncache, (s1 - s0) * 5);
        for (long q = threadIdx.x; q < nc * dd; q += blockDim.x) {
            const long task = q / dd;
            lcache[q] = k.links[((long)(s0 + task / 5) * 5 + task % 5) * dd + (q - task * dd)];
        }
    }

    // x = x0 = b
    for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) k.x[e] = k.b[e];
    if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
    apply_own<NI>(k, k.x, u0, k.b, s0, s1, part, 1.0, lcache);  // u_0 = r = b - D x
    __syncthreads();
    {
        double rr = 0.0, bb = 0.0;
        for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            rr += cnorm2(u0[e]);
            bb += cnorm2(k.b[e]);
            if (k.nbs > 0) vc[e - e0] = u0[e];
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
    const double tol2 = (k.tol * norm_b) * (k.tol * norm_b);
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
            apply_own<NI>(k, k.V + (long)j * n, wl, nullptr, s0, s1, part, sc[j], lcache, e0);
            __syncthreads();
            // (u_i, w) for i <= j and ||w||^2 in one reduction
            partial_dots_norm(k, V, wl, j + 1, pA, e0, e1);
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
            double hn2;  // ||u_{j+1}||^2
            if (!reorth) {
                for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                    double2 a = wl[e - e0];
                    for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h[i], V.get(i, e));
                    V.put(j + 1, e, a);
                }
                hn2 = d2;
                if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;  // publishes u_{j+1}
            } else {
                // w -= V h ; reorthogonalise
                for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                    double2 a = wl[e - e0];
                    for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h[i], V.get(i, e));
                    wl[e - e0] = a;
                }
                __syncthreads();
                partial_dots(k, V, wl, j + 1, pB, e0, e1);
                if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
                reduce_partials(k, pB, j + 1, h2);
                for (int i = threadIdx.x; i <= j; i += blockDim.x) h2[i] = sc[i] * h2[i];
                __syncthreads();
                {
                    double ss = 0.0;
                    for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                        double2 a = wl[e - e0];
                        for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h2[i], V.get(i, e));
                        V.put(j + 1, e, a);
                        ss += cnorm2(a);
                    }
                    __shared__ double2 red2[33];
                    double2 t = block_sum(make_double2(ss, 0.0), red2);
                    if (threadIdx.x == 0) pC[(long)blockIdx.x * k.P] = t;
                }
                for (int i = threadIdx.x; i <= j; i += blockDim.x) h[i] = h[i] + h2[i];
                if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;  // also publishes u_{j+1}
                hn2 = reduce_slot0(k, pC, &s_sum).x;
            }
            if (threadIdx.x == 0) coarse_rotation(h, gm, cn, sn, sc, j, hn2, tol2, &s_flag);
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
            for (int jj = 0; jj < maxIt; jj++) a = cfma(eta[jj], V.get(jj, e), a);
            k.x[e] = a;
        }
        if (!grid_barrier(k.bar, k.status, G, k.spin_limit)) return;
        apply_own<NI>(k, k.x, u0, k.b, s0, s1, part, 1.0, lcache);  // new residual into slot 0
        __syncthreads();
        {
            double rr = 0.0;
            for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                rr += cnorm2(u0[e]);
                if (k.nbs > 0) vc[e - e0] = u0[e];
            }
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

// ---------------------------------------------------------------- the same solve on one thread-block cluster
// The cooperative kernel above spreads the coarsest solve over ~128 CTAs and pays two grid barriers per
// Arnoldi step (atomics and polling through L2, about 2.5 us each).  Here one cluster of C CTAs (16 where
// the device schedules such clusters) runs the whole solve: the cluster barrier is a hardware barrier, the
// vector being applied lives in the CTAs' shared memory and neighbouring CTAs read it through distributed
// shared memory, and the partial sums of every reduction are read from the other CTAs' shared memory in
// rank order (identical totals in every CTA).  The link matrices still stream from L2, now through C SMs
// instead of ~128, which bounds the operator application.  With several right-hand sides the grid holds
// several clusters, each looping over its share of them with its own workspace.  The arithmetic per
// element (operator, Gram-Schmidt, rotations) is that of coarse_gmres_kernel; only the reduction trees
// differ.  No wait in this kernel can outlast the cluster: its CTAs are co-scheduled by construction.
namespace cgrp = cooperative_groups;
constexpr int kClusterThreads = 512;

struct GmresC {
    const double2* links;
    const double2* b;  // R right-hand sides, n apart
    double2* x;
    double2* ws;       // per cluster: basis (m+1) n, w n, Hessenberg (m+1) m
    long wstride;
    int* status;       // [1]: iterations of the last right-hand side of cluster 0
    int Nx, Nt, dof, m, restarts, R;
    double m0, tol;
};

// out = [b -] scale * D in on this CTA's sites, `cur` holding every CTA's slice of `in` (spc sites each);
// neighbours come from the owning CTA's shared memory.  Same per-element arithmetic as apply_own.
__device__ void apply_cluster(const GmresC& k, cgrp::cluster_group& cl, double2* cur, double2* __restrict__ out,
                              const double2* __restrict__ bsub, int s0, int s1, int spc, double2* __restrict__ part,
                              double scale) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int dof = k.dof, Nt = k.Nt, Nx = k.Nx;
    const int ntask = (s1 - s0) * 5;
    constexpr int CB = 16;  // column loads in flight per lane
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
        const int owner = nb / spc;
        const double2* src = cl.map_shared_rank(cur, owner) + (long)(nb - owner * spc) * dof;
        const double2 vd = (lane < dof) ? sg * src[lane] : make_double2(0.0, 0.0);
        double2 acc = make_double2(0.0, 0.0);
        const double2* M = k.links + ((long)n * 5 + d) * dof * dof;
        for (int j0 = 0; j0 < dof; j0 += CB) {
            double2 mv[CB];
#pragma unroll
            for (int u = 0; u < CB; u++)
                mv[u] = (j0 + u < dof && lane < dof) ? __ldg(M + (long)(j0 + u) * dof + lane) : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < CB; u++) {
                if (j0 + u >= dof) break;
                const double2 vj = make_double2(__shfl_sync(0xffffffffu, vd.x, j0 + u),
                                                __shfl_sync(0xffffffffu, vd.y, j0 + u));
                acc = cfma(mv[u], vj, acc);
            }
        }
        if (lane < dof) part[(sl * 5 + d) * dof + lane] = (d == 0) ? (k.m0 + 2.0) * vd - acc : acc;
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
// own partial sums of (V_i, w), i < cnt (and ||w||^2 in slot cnt when with_norm), into part[i]
__device__ void cl_partial_dots(const double2* __restrict__ V, const double2* __restrict__ w, int cnt, bool with_norm,
                                double2* part, long e0, long e1, long n) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int last = with_norm ? cnt : cnt - 1;
    for (int i = wid; i <= last; i += nw) {
        const double2* vi = i < cnt ? V + (long)i * n : w;
        double2 s = make_double2(0.0, 0.0);
        for (long e = e0 + lane; e < e1; e += 32) s = cfmac(vi[e], w[e], s);
        s = warp_sum(s);
        if (lane == 0) part[i] = s;
    }
}
// out[i] = sum over the cluster's CTAs of their part[i], rank order, the same in every CTA
__device__ void cl_reduce(cgrp::cluster_group& cl, double2* part, int cnt, double2* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int C = (int)cl.num_blocks();
    for (int i = wid; i < cnt; i += nw) {
        double2 s = make_double2(0.0, 0.0);
        for (int q = lane; q < C; q += 32) s += cl.map_shared_rank(part, q)[i];
        s = warp_sum(s);
        if (lane == 0) out[i] = s;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kClusterThreads) coarse_gmres_cluster_kernel(GmresC k) {
    cgrp::cluster_group cl = cgrp::this_cluster();
    extern __shared__ double2 sh[];
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int cid = blockIdx.x / C, ncl = gridDim.x / C;
    const int m = k.m, dof = k.dof;
    const int sites = k.Nx * k.Nt;
    const long n = (long)sites * dof;
    const int spc = (sites + C - 1) / C;
    const int s0 = min(sites, rank * spc), s1 = min(sites, s0 + spc);
    const long e0 = (long)s0 * dof, e1 = (long)s1 * dof;
    double2* h = sh;
    double2* h2 = h + (m + 1);
    double2* gm = h2 + (m + 1);
    double2* cn = gm + (m + 1);
    double2* sn = cn + m;
    double2* eta = sn + m;
    double* sc = reinterpret_cast<double*>(eta + m);
    double2* hs = eta + m + (m + 1);
    double2* pA = hs + kHs * (kHs + 1) / 2;
    double2* pB = pA + (m + 2);
    double2* pC = pB + (m + 2);
    double2* cur = pC + (m + 2);       // spc x dof: this CTA's slice of the vector being applied
    double2* part = cur + spc * dof;   // spc x 5 x dof
    __shared__ int s_flag;
    __shared__ double2 red[33];
    double2* V = k.ws + cid * k.wstride;
    double2* w = V + (long)(m + 1) * n;
    double2* Hg = w + n;
    for (int rhs = cid; rhs < k.R; rhs += ncl) {
        const double2* b = k.b + rhs * n;
        double2* x = k.x + rhs * n;
        for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {  // x = x0 = b
            x[e] = b[e];
            cur[e - e0] = b[e];
        }
        cl.sync();
        apply_cluster(k, cl, cur, V, b, s0, s1, spc, part, 1.0);  // u_0 = r = b - D x
        __syncthreads();
        {
            double rr = 0.0, bb = 0.0;
            for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                rr += cnorm2(V[e]);
                bb += cnorm2(b[e]);
            }
            const double2 t = block_sum(make_double2(rr, bb), red);
            if (threadIdx.x == 0) pC[0] = t;
        }
        cl.sync();
        cl_reduce(cl, pC, 1, h2);
        double err = sqrt(h2[0].x);
        const double norm_b = sqrt(h2[0].y);
        const double tol2 = (k.tol * norm_b) * (k.tol * norm_b);
        int maxIt = m, iters = k.restarts * m;
        bool converged = false;
        if (norm_b == 0.0) {  // zero right-hand side: x = 0
            for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) x[e] = make_double2(0.0, 0.0);
            iters = 0;
            converged = true;
        }
        for (int kk = 0; kk < k.restarts && !converged; kk++) {
            __syncthreads();
            if (threadIdx.x == 0) {
                gm[0] = make_double2(err, 0.0);
                sc[0] = 1.0 / err;
            }
            for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) cur[e - e0] = V[e];  // u_0
            cl.sync();
            for (int j = 0; j < m; j++) {
                apply_cluster(k, cl, cur, w, nullptr, s0, s1, spc, part, sc[j]);  // w = D v_j
                __syncthreads();
                cl_partial_dots(V, w, j + 1, true, pA, e0, e1, n);
                cl.sync();
                cl_reduce(cl, pA, j + 2, h);
                for (int i = threadIdx.x; i <= j; i += blockDim.x) h[i] = sc[i] * h[i];
                __syncthreads();
                double hh = 0.0;
                for (int i = 0; i <= j; i++) hh += cnorm2(h[i]);
                const double w2 = h[j + 1].x, d2 = w2 - hh;
                const bool reorth = !(d2 > 1e-4 * w2);
                double2* un = V + (long)(j + 1) * n;
                double hn2;
                if (!reorth) {
                    for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                        double2 a = w[e];
                        for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h[i], V[(long)i * n + e]);
                        un[e] = a;
                        cur[e - e0] = a;
                    }
                    hn2 = d2;
                    cl.sync();  // publishes u_{j+1}
                } else {
                    for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                        double2 a = w[e];
                        for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h[i], V[(long)i * n + e]);
                        w[e] = a;
                    }
                    __syncthreads();
                    cl_partial_dots(V, w, j + 1, false, pB, e0, e1, n);
                    cl.sync();
                    cl_reduce(cl, pB, j + 1, h2);
                    for (int i = threadIdx.x; i <= j; i += blockDim.x) h2[i] = sc[i] * h2[i];
                    __syncthreads();
                    {
                        double ss = 0.0;
                        for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                            double2 a = w[e];
                            for (int i = 0; i <= j; i++) a = a - cmul(sc[i] * h2[i], V[(long)i * n + e]);
                            un[e] = a;
                            cur[e - e0] = a;
                            ss += cnorm2(a);
                        }
                        const double2 t = block_sum(make_double2(ss, 0.0), red);
                        if (threadIdx.x == 0) pC[0] = t;
                    }
                    for (int i = threadIdx.x; i <= j; i += blockDim.x) h[i] = h[i] + h2[i];
                    cl.sync();  // also publishes u_{j+1}
                    cl_reduce(cl, pC, 1, h2 + j + 1);
                    hn2 = h2[j + 1].x;
                }
                if (threadIdx.x == 0) coarse_rotation(h, gm, cn, sn, sc, j, hn2, tol2, &s_flag);
                __syncthreads();
                if (j < kHs)
                    for (int i = threadIdx.x; i <= j; i += blockDim.x) hs[j * (j + 1) / 2 + i] = h[i];
                if (rank == 0)
                    for (int i = threadIdx.x; i <= j; i += blockDim.x) Hg[(long)j * (m + 1) + i] = h[i];
                if (s_flag) {  // identical in every CTA
                    maxIt = j + 1;
                    break;
                }
            }
            if (maxIt <= kHs) {
                __syncthreads();
                if (threadIdx.x == 0)
                    for (int i = maxIt - 1; i >= 0; i--) {
                        double2 e = gm[i];
                        for (int q = i + 1; q < maxIt; q++) e = e - cmul(hs[q * (q + 1) / 2 + i], eta[q]);
                        eta[i] = cdiv(e, hs[i * (i + 1) / 2 + i]);
                    }
            } else {  // from rank 0's columns in global memory
                __threadfence();
                cl.sync();
                for (int i = threadIdx.x; i < maxIt; i += blockDim.x) eta[i] = gm[i];
                __syncthreads();
                for (int i = maxIt - 1; i >= 0; i--) {
                    if (threadIdx.x == 0) eta[i] = cdiv(eta[i], __ldcg(Hg + (long)i * (m + 1) + i));
                    __syncthreads();
                    for (int q = threadIdx.x; q < i; q += blockDim.x)
                        eta[q] = eta[q] - cmul(__ldcg(Hg + (long)i * (m + 1) + q), eta[i]);
                    __syncthreads();
                }
            }
            for (int i = threadIdx.x; i < maxIt; i += blockDim.x) eta[i] = sc[i] * eta[i];
            __syncthreads();
            for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                double2 a = x[e];
                for (int jj = 0; jj < maxIt; jj++) a = cfma(eta[jj], V[(long)jj * n + e], a);
                x[e] = a;
                cur[e - e0] = a;
            }
            cl.sync();
            apply_cluster(k, cl, cur, V, b, s0, s1, spc, part, 1.0);  // new residual into slot 0
            __syncthreads();
            {
                double rr = 0.0;
                for (long e = e0 + threadIdx.x; e < e1; e += blockDim.x) rr += cnorm2(V[e]);
                const double2 t = block_sum(make_double2(rr, 0.0), red);
                if (threadIdx.x == 0) pC[0] = t;
            }
            cl.sync();
            cl_reduce(cl, pC, 1, h2);
            err = sqrt(h2[0].x);
            if (err < k.tol * norm_b) {
                iters = kk * m + maxIt;
                converged = true;
            }
        }
        if (cid == 0 && rank == 0 && threadIdx.x == 0) k.status[1] = iters;
        cl.sync();  // no CTA leaves, or starts the next right-hand side, while another reads its shared memory
    }
}

static size_t cluster_smem(int spc, int m, int dof) {
    return sizeof(double2) * ((size_t)7 * (m + 1) + (size_t)kHs * (kHs + 1) / 2 + 3 * (size_t)(m + 2) +
                              (size_t)spc * dof + (size_t)spc * 5 * dof);
}

bool coarse_cluster_prepare(CoarseClusterWork& w, int n, int m, int dof, int max_rhs) {
    w = CoarseClusterWork{};
    if (dof > 32) return false;
    const int sites = n / dof;
    for (int C : {16, 8}) {
        const int spc = (sites + C - 1) / C;
        const size_t smem = cluster_smem(spc, m, dof);
        if (smem > kDynSmemCap) continue;
        if (C > 8 && cudaFuncSetAttribute(coarse_gmres_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed,
                                          1) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(coarse_gmres_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = C;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, coarse_gmres_cluster_kernel, &cfg) != cudaSuccess || nc < 1) {
            cudaGetLastError();
            continue;
        }
        w.C = C;
        w.clusters = std::max(1, std::min(nc, max_rhs));
        w.smem = smem;
        w.wstride = (long)(m + 2) * n + (long)(m + 1) * m;
        return true;
    }
    return false;
}

void launch_coarse_gmres_cluster(cudaStream_t s, const CoarseClusterWork& w, const double2* links, const double2* b,
                                 double2* x, int R, int Nx, int Nt, int dof, double m0, int m, int restarts,
                                 double tol) {
    GmresC k;
    k.links = links;
    k.b = b;
    k.x = x;
    k.ws = w.ws;
    k.wstride = w.wstride;
    k.status = w.status;
    k.Nx = Nx;
    k.Nt = Nt;
    k.dof = dof;
    k.m = m;
    k.restarts = restarts;
    k.R = R;
    k.m0 = m0;
    k.tol = tol;
    DDAMG_CUDA_TRY(cudaMemsetAsync(w.status, 0, 2 * sizeof(int), s));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(w.C * std::min(R, w.clusters));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = w.smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = w.C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    DDAMG_CUDA_TRY(cudaLaunchKernelEx(&cfg, coarse_gmres_cluster_kernel, k));
    ++g_launches;
}

// CTAs of the coarsest solve: about two coarse sites per CTA, at most one CTA per SM
int coarse_gmres_grid(long sites, int sms) { return (int)std::min<long>(sms, std::max<long>(1, (sites + 1) / 2)); }
// shared memory of the cooperative kernel without the caches, and with ncache link matrices and nbs
// basis slots of the CTA's slice
static size_t coarse_gmres_smem(long sites, int grid, int m, int dof, int ncache = 0, int nbs = 0) {
    const long spc = (sites + grid - 1) / grid;
    return sizeof(double2) * ((size_t)7 * (m + 1) + (size_t)kHs * (kHs + 1) / 2 + (size_t)spc * 5 * dof +
                              (size_t)spc * dof + (size_t)ncache * dof * dof + (size_t)nbs * spc * dof);
}
// the caches that fit beside the rest in 227 KB: the link matrices first (read every step), then basis
// slots (up to kHs: restarts rarely go further)
static void coarse_gmres_caches(long sites, int grid, int m, int dof, int* ncache, int* nbs) {
    const long spc = (sites + grid - 1) / grid;
    const size_t cap = kDynSmemCap, base = coarse_gmres_smem(sites, grid, m, dof);
    const size_t mat = sizeof(double2) * (size_t)dof * dof, slot = sizeof(double2) * (size_t)spc * dof;
    *ncache = base >= cap ? 0 : (int)std::min<size_t>((size_t)spc * 5, (cap - base) / mat);
    const size_t used = base + (size_t)*ncache * mat;
    *nbs = used >= cap ? 0 : (int)std::min<size_t>((size_t)std::min(m + 1, kHs), (cap - used) / slot);
}

void coarse_gmres_prepare(CoarseGmresWork& w, int n, int m, int dof, int device) {
    int sms = 0;
    DDAMG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = coarse_gmres_grid(n / dof, sms);
    if (coarse_gmres_smem(n / dof, grid, m, dof) > kDynSmemCap)
        throw ParamFailure{"coarsest GMRES restart length too large for shared memory"};
    coarse_gmres_caches(n / dof, grid, m, dof, &w.ncache, &w.nbs);
    const size_t smem = coarse_gmres_smem(n / dof, grid, m, dof, w.ncache, w.nbs);
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
    k.ncache = w.ncache;
    k.nbs = w.nbs;
    DDAMG_CUDA_TRY(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned), s));
    DDAMG_CUDA_TRY(cudaMemsetAsync(w.status, 0, 2 * sizeof(int), s));
    size_t smem = coarse_gmres_smem((long)Nx * Nt, w.grid, m, dof, w.ncache, w.nbs);
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
        if (need > (long)kNoAllocScratch || coarse_gmres_smem(sites, (int)grid, m, dof) > kDynSmemCap) {
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
