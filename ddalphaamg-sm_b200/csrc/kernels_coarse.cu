// Coarse-level kernels: generic level operator, transfers P / P^dagger, local
// orthonormalisation of the test vectors and the Galerkin coarse-link construction.
#include "internal.h"

namespace ddamg {

__device__ __forceinline__ double shfl(double v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ float shfl(float v, int l) { return __shfl_sync(0xffffffffu, v, l); }
template <typename V> __device__ __forceinline__ V shflc(V v, int l) { return mkc(shfl(v.x, l), shfl(v.y, l)); }

// Level::D_operator (src/level.cpp:394-426) for a level >= 1:
//   out = (m0+2) v - sum_d s_d M_d(n) v(nbr_d(n))       [or b - that when b != null]
// One warp per site; lane i owns output dof i (and i+32 when dof > 32). Neighbour vectors
// are held one dof per lane and broadcast with shuffles; M_d is read column by column.
template <typename V, int NI>
__global__ void __launch_bounds__(128) coarse_op_kernel(const V* __restrict__ links, const V* __restrict__ in,
                                                        V* __restrict__ out, const V* __restrict__ b, int Nx, int Nt,
                                                        int dof, typename RealOf<V>::R m0, long stride) {
    typedef typename RealOf<V>::R R;
    const int lane = threadIdx.x & 31;
    const int n = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (n >= Nx * Nt) return;
    const long ro = (long)blockIdx.y * stride;
    in += ro;
    out += ro;
    const int x = n / Nt, t = n - x * Nt;
    int nb[5];
    R sg[5];
    nb[0] = n;
    nb[1] = x * Nt + ((t + 1 == Nt) ? 0 : t + 1);
    nb[2] = ((x + 1 == Nx) ? 0 : x + 1) * Nt + t;
    nb[3] = x * Nt + ((t == 0) ? Nt - 1 : t - 1);
    nb[4] = ((x == 0) ? Nx - 1 : x - 1) * Nt + t;
    sg[0] = R(1);
    sg[1] = (t == Nt - 1) ? R(-1) : R(1);
    sg[2] = R(1);
    sg[3] = (t == 0) ? R(-1) : R(1);
    sg[4] = R(1);
    V acc[NI];
#pragma unroll
    for (int q = 0; q < NI; q++) acc[q] = czero<V>();
    V self[NI];
#pragma unroll
    for (int d = 0; d < 5; d++) {
        V vd[NI];
#pragma unroll
        for (int q = 0; q < NI; q++) {
            int i = lane + 32 * q;
            vd[q] = (i < dof) ? sg[d] * in[(long)nb[d] * dof + i] : czero<V>();
            if (d == 0) self[q] = vd[q];
        }
        const V* M = links + ((long)n * 5 + d) * dof * dof;
#pragma unroll
        for (int jq = 0; jq < NI; jq++) {
            const int jn = min(32, dof - 32 * jq);
            for (int j0 = 0; j0 < jn; j0 += 8) {  // 8 column loads in flight per lane
                V mv[8][NI];
#pragma unroll
                for (int u = 0; u < 8; u++)
#pragma unroll
                    for (int q = 0; q < NI; q++) {
                        const int i = lane + 32 * q;
                        mv[u][q] = (j0 + u < jn && i < dof) ? __ldg(M + (long)(32 * jq + j0 + u) * dof + i) : czero<V>();
                    }
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    if (j0 + u >= jn) break;
                    const V vj = shflc(vd[jq], j0 + u);
#pragma unroll
                    for (int q = 0; q < NI; q++) acc[q] = cfma(mv[u][q], vj, acc[q]);
                }
            }
        }
    }
    const R mm = m0 + R(2);
#pragma unroll
    for (int q = 0; q < NI; q++) {
        int i = lane + 32 * q;
        if (i < dof) {
            V o = mm * self[q] - acc[q];
            if (b) o = b[ro + (long)n * dof + i] - o;
            out[(long)n * dof + i] = o;
        }
    }
}
// The same operator for several vectors at once: one warp per (site, chunk of RC vectors), lane =
// output dof (dof <= 32).  Each link element is loaded once and applied to all RC vectors; the
// neighbour vectors of the chunk are staged in per-warp shared memory and read as broadcasts.
// Tasks run site-major, so the chunks of one site are neighbours in the grid and share its links
// through L2.
template <typename V, int RC>
__global__ void __launch_bounds__(128) coarse_op_multi_kernel(const V* __restrict__ links, const V* __restrict__ in,
                                                              V* __restrict__ out, const V* __restrict__ b, int Nx,
                                                              int Nt, int dof, typename RealOf<V>::R m0, long stride,
                                                              int nrhs) {
    typedef typename RealOf<V>::R R;
    __shared__ V sv[4][RC][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nchunk = (nrhs + RC - 1) / RC;
    const long task = (long)blockIdx.x * 4 + wib;
    const int sites = Nx * Nt;
    if (task >= (long)sites * nchunk) return;
    const int n = (int)(task / nchunk), r0 = (int)(task - (long)n * nchunk) * RC;
    const int rc = min(RC, nrhs - r0);
    const int x = n / Nt, t = n - x * Nt;
    int nb[5];
    R sg[5];
    nb[0] = n;
    nb[1] = x * Nt + ((t + 1 == Nt) ? 0 : t + 1);
    nb[2] = ((x + 1 == Nx) ? 0 : x + 1) * Nt + t;
    nb[3] = x * Nt + ((t == 0) ? Nt - 1 : t - 1);
    nb[4] = ((x == 0) ? Nx - 1 : x - 1) * Nt + t;
    sg[0] = R(1);
    sg[1] = (t == Nt - 1) ? R(-1) : R(1);
    sg[2] = R(1);
    sg[3] = (t == 0) ? R(-1) : R(1);
    sg[4] = R(1);
    V acc[RC], self[RC];
#pragma unroll
    for (int r = 0; r < RC; r++) acc[r] = self[r] = czero<V>();
    const bool li = lane < dof;
    for (int d = 0; d < 5; d++) {
        __syncwarp();
#pragma unroll
        for (int r = 0; r < RC; r++) {
            V v = (li && r < rc) ? sg[d] * in[(long)(r0 + r) * stride + (long)nb[d] * dof + lane] : czero<V>();
            sv[wib][r][lane] = v;
            if (d == 0) self[r] = v;
        }
        __syncwarp();
        const V* M = links + ((long)n * 5 + d) * dof * dof;
        for (int j0 = 0; j0 < dof; j0 += 8) {  // 8 column loads in flight
            V mv[8];
#pragma unroll
            for (int u = 0; u < 8; u++) mv[u] = (j0 + u < dof && li) ? __ldg(M + (long)(j0 + u) * dof + lane) : czero<V>();
#pragma unroll
            for (int u = 0; u < 8; u++) {
                if (j0 + u >= dof) break;
#pragma unroll
                for (int r = 0; r < RC; r++) acc[r] = cfma(mv[u], sv[wib][r][j0 + u], acc[r]);
            }
        }
    }
    if (!li) return;
    const R mm = m0 + R(2);
#pragma unroll
    for (int r = 0; r < RC; r++) {
        if (r >= rc) break;
        V o = mm * self[r] - acc[r];
        const long idx = (long)(r0 + r) * stride + (long)n * dof + lane;
        if (b) o = b[idx] - o;
        out[idx] = o;
    }
}

template <typename V>
void launch_coarse_op(cudaStream_t s, const V* links, const V* in, V* out, const V* b, int Nx, int Nt, int dof,
                      double m0, int nrhs) {
    typedef typename RealOf<V>::R R;
    long stride = (long)Nx * Nt * dof;
    if (nrhs > 1 && dof <= 32) {
        const long tasks = (long)Nx * Nt * ((nrhs + 7) / 8);
        DDAMG_LAUNCH((coarse_op_multi_kernel<V, 8>), ceil_div(tasks, 4), 128, 0, s, links, in, out, b, Nx, Nt, dof,
                     (R)m0, stride, nrhs);
        return;
    }
    dim3 grid(ceil_div((long)Nx * Nt, 4), nrhs);
    if (dof <= 32)
        DDAMG_LAUNCH((coarse_op_kernel<V, 1>), grid, 128, 0, s, links, in, out, b, Nx, Nt, dof, (R)m0, stride);
    else
        DDAMG_LAUNCH((coarse_op_kernel<V, 2>), grid, 128, 0, s, links, in, out, b, Nx, Nt, dof, (R)m0, stride);
}

// Level::Pdagg_v (src/level.cpp:145-189): out[b][cc][s] = sum_{n in b, c} conj(w_cc[n][c][s]) v[n][c][s].
// One CTA per (aggregate, rhs); one warp per test vector cc; lanes stride over (site, colour).
template <typename V>
__global__ void __launch_bounds__(128) restrict_kernel(Geom g, const V* __restrict__ tv, const V* __restrict__ in,
                                                       V* __restrict__ out) {
    const int b = blockIdx.x, r = blockIdx.y;
    const int bx = b / g.agg_t, bt = b - bx * g.agg_t;
    const int C = g.colors, dof = g.dof, E = g.el_x * g.el_t * C;
    const V* v = in + (long)r * g.size();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int cc = wid; cc < g.ntest; cc += nw) {
        const V* w = tv + (long)cc * g.size();
        double2 a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
        for (int e = lane; e < E; e += 32) {
            const int k = e / C, c = e - k * C;
            const int kx = k / g.el_t, kt = k - kx * g.el_t;
            const long n = (long)(bx * g.el_x + kx) * g.Nt + bt * g.el_t + kt;
            const long idx = n * dof + c * 2;
            a0 = cfmac(to_d(w[idx]), to_d(v[idx]), a0);
            a1 = cfmac(to_d(w[idx + 1]), to_d(v[idx + 1]), a1);
        }
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        if (lane == 0) {
            V* o = out + (long)r * g.agg_x * g.agg_t * 2 * g.ntest + ((long)b * g.ntest + cc) * 2;
            o[0] = from_d<V>(a0);
            o[1] = from_d<V>(a1);
        }
    }
}
template <typename V>
void launch_restrict(cudaStream_t s, const Geom& g, const V* tv, const V* in, V* out, int nrhs) {
    DDAMG_LAUNCH(restrict_kernel<V>, dim3(g.agg_x * g.agg_t, nrhs), 128, 0, s, g, tv, in, out);
}

// Level::P_vc (src/level.cpp:92-141): out[n][c][s] (+)= sum_cc w_cc[n][c][s] vc[block(n)][cc][s]
template <typename V>
__global__ void __launch_bounds__(256) prolong_kernel(Geom g, const V* __restrict__ tv, const V* __restrict__ vc,
                                                      V* __restrict__ out, int add) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= g.size()) return;
    const int r = blockIdx.y;
    const int n = (int)(e / g.dof), k = (int)(e - (long)n * g.dof), s = k & 1;
    const int x = n / g.Nt, t = n - x * g.Nt;
    const int b = (x / g.el_x) * g.agg_t + t / g.el_t;
    const V* v = vc + (long)r * g.agg_x * g.agg_t * 2 * g.ntest + (long)b * 2 * g.ntest + s;
    double2 acc = make_double2(0.0, 0.0);
    for (int cc = 0; cc < g.ntest; cc++) acc = cfma(to_d(tv[(long)cc * g.size() + e]), to_d(v[2 * cc]), acc);
    V* o = out + (long)r * g.size() + e;
    if (add) {
        double2 p = to_d(*o);
        acc.x += p.x;
        acc.y += p.y;
    }
    *o = from_d<V>(acc);
}
template <typename V>
void launch_prolong(cudaStream_t s, const Geom& g, const V* tv, const V* vc, V* out, int add, int nrhs) {
    DDAMG_LAUNCH(prolong_kernel<V>, dim3(ceil_div(g.size(), 256), nrhs), 256, 0, s, g, tv, vc, out, add);
}

// Level::orthonormalize (src/level.cpp:193-284): modified Gram-Schmidt of the ntest vectors
// restricted to one aggregate (block b, spin s); a vector is normalised only if its norm
// exceeds 1e-8.  One CTA per aggregate; the aggregate's vectors are staged in shared memory.
__global__ void __launch_bounds__(256) orthonormalize_kernel(Geom g, double2* __restrict__ tv) {
    extern __shared__ double2 sm[];
    __shared__ double2 red[33];
    const int b = blockIdx.x >> 1, s = blockIdx.x & 1;
    const int bx = b / g.agg_t, bt = b - bx * g.agg_t;
    const int C = g.colors, E = g.el_x * g.el_t * C, Nv = g.ntest;
    auto gidx = [&](int e) -> long {
        const int k = e / C, c = e - k * C;
        const int kx = k / g.el_t, kt = k - kx * g.el_t;
        return ((long)(bx * g.el_x + kx) * g.Nt + bt * g.el_t + kt) * g.dof + c * 2 + s;
    };
    for (int q = threadIdx.x; q < Nv * E; q += blockDim.x) {
        const int cc = q / E, e = q - cc * E;
        sm[q] = tv[(long)cc * g.size() + gidx(e)];
    }
    __syncthreads();
    for (int nt = 0; nt < Nv; nt++) {
        double2* w = sm + (long)nt * E;
        for (int ntt = 0; ntt < nt; ntt++) {
            const double2* u = sm + (long)ntt * E;
            double2 p = make_double2(0.0, 0.0);
            for (int e = threadIdx.x; e < E; e += blockDim.x) p = cfmac(u[e], w[e], p);  // w * conj(u)
            p = block_sum(p, red);
            for (int e = threadIdx.x; e < E; e += blockDim.x) w[e] = w[e] - cmul(p, u[e]);
            __syncthreads();
        }
        double nr = 0.0;
        for (int e = threadIdx.x; e < E; e += blockDim.x) nr += cnorm2(w[e]);
        double2 nr2 = block_sum(make_double2(nr, 0.0), red);
        const double nrm = sqrt(nr2.x);
        if (nrm > 1e-8)
            for (int e = threadIdx.x; e < E; e += blockDim.x) w[e] = make_double2(w[e].x / nrm, w[e].y / nrm);
        __syncthreads();
    }
    for (int q = threadIdx.x; q < Nv * E; q += blockDim.x) {
        const int cc = q / E, e = q - cc * E;
        tv[(long)cc * g.size() + gidx(e)] = sm[q];
    }
}
// The same for aggregates of at most 32 unknowns per spin (level 0: 16 sites of one colour): one warp per
// (aggregate, spin), one unknown per lane, the warp's vectors in its own slice of shared memory and warp
// sums instead of CTA barriers.  With one unknown per lane the CTA version's block_sum reduces to the same
// warp butterfly (the other warps add exact zeros), so the results are bit for bit those of
// orthonormalize_kernel.
constexpr int kOrthWarps = 8;
__global__ void __launch_bounds__(32 * kOrthWarps) orthonormalize_warp_kernel(Geom g, double2* __restrict__ tv) {
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int task = blockIdx.x * kOrthWarps + warp;
    if (task >= 2 * g.agg_x * g.agg_t) return;  // whole warps; no CTA barrier follows
    const int b = task >> 1, s = task & 1;
    const int bx = b / g.agg_t, bt = b - bx * g.agg_t;
    const int C = g.colors, E = g.el_x * g.el_t * C, Nv = g.ntest;
    const bool own = lane < E;
    long gi = 0;
    if (own) {
        const int k = lane / C, c = lane - k * C;
        const int kx = k / g.el_t, kt = k - kx * g.el_t;
        gi = ((long)(bx * g.el_x + kx) * g.Nt + bt * g.el_t + kt) * g.dof + c * 2 + s;
    }
    double2* v = sm + (size_t)warp * Nv * 32;  // v[cc * 32 + lane]: only this lane's column is touched
    for (int cc = 0; cc < Nv; cc++) v[cc * 32 + lane] = own ? tv[(long)cc * g.size() + gi] : make_double2(0.0, 0.0);
    for (int nt = 0; nt < Nv; nt++) {
        double2 w = v[nt * 32 + lane];
        for (int ntt = 0; ntt < nt; ntt++) {
            const double2 u = v[ntt * 32 + lane];
            double2 p = make_double2(0.0, 0.0);
            if (own) p = cfmac(u, w, p);  // w * conj(u)
            p = warp_sum(p);
            if (own) w = w - cmul(p, u);
        }
        double nr = 0.0;
        if (own) nr += cnorm2(w);
        const double nrm = sqrt(warp_sum(make_double2(nr, 0.0)).x);
        if (nrm > 1e-8 && own) w = make_double2(w.x / nrm, w.y / nrm);
        v[nt * 32 + lane] = w;
    }
    if (own)
        for (int cc = 0; cc < Nv; cc++) tv[(long)cc * g.size() + gi] = v[cc * 32 + lane];
}

void launch_orthonormalize(cudaStream_t s, const Geom& g, double2* tv) {
    const int E = g.el_x * g.el_t * g.colors;
    if (E <= 32) {
        const size_t smem = sizeof(double2) * (size_t)kOrthWarps * g.ntest * 32;
        DDAMG_CUDA_TRY(cudaFuncSetAttribute(orthonormalize_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
        const int tasks = 2 * g.agg_x * g.agg_t;
        DDAMG_LAUNCH(orthonormalize_warp_kernel, (tasks + kOrthWarps - 1) / kOrthWarps, 32 * kOrthWarps, smem, s, g, tv);
        return;
    }
    size_t smem = sizeof(double2) * (size_t)g.ntest * E;
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(orthonormalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DDAMG_LAUNCH(orthonormalize_kernel, 2 * g.agg_x * g.agg_t, 256, smem, s, g, tv);
}

// Level::makeCoarseLinks (src/level.cpp:431-542) as a triple product per fine site and hop:
//   Coarse[D] += W(n)^dagger F_h(n) W(nbr_h(n)),   W spin-block-diagonal (aggregates split spin),
// D = 0 (A) when the hop stays inside the aggregate, else the hop direction (B_mu / C_mu).
// F_h is the fine level's link matrix for hop h without the antiperiodic sign (the sign is
// applied by the operator on the coarse lattice, as the reference does).  Level 0's F_h is
// makeDirac's G2 / G3 (src/level.cpp:286-331) built from U on the fly.
__device__ __forceinline__ double2 level0_link(const double2* __restrict__ U, int Nx, int Nt, int n, int h, int alf,
                                               int bet) {
    const int x = n / Nt, t = n - x * Nt;
    double2 u;
    double2 coef;
    // (1 - sigma_mu) for forward hops, (1 + sigma_mu) for backward hops; sigma_0 = sigma_x, sigma_1 = sigma_y
    if (h == 1 || h == 3) {  // mu = 0
        const double sgn = (h == 1) ? -1.0 : 1.0;
        coef = (alf == bet) ? make_double2(1.0, 0.0) : make_double2(sgn, 0.0);
        u = (h == 1) ? U[2 * n] : conjc(U[2 * (x * Nt + ((t == 0) ? Nt - 1 : t - 1))]);
    } else {  // mu = 1, sigma_y = [[0,-i],[i,0]]
        const double sgn = (h == 2) ? -1.0 : 1.0;
        if (alf == bet) coef = make_double2(1.0, 0.0);
        else coef = make_double2(0.0, (alf == 0 ? -1.0 : 1.0) * sgn);
        u = (h == 2) ? U[2 * n + 1] : conjc(U[2 * (((x == 0) ? Nx - 1 : x - 1) * Nt + t) + 1]);
    }
    return 0.5 * cmul(coef, u);
}

__global__ void __launch_bounds__(256) build_links_kernel(Geom g, const double2* __restrict__ U,
                                                          const double2* __restrict__ links,
                                                          const double2* __restrict__ tv, double2* __restrict__ next) {
    extern __shared__ double2 sm[];
    const int C = g.colors, df = g.dof, Nv = g.ntest, dc = 2 * Nv;
    double2* acc = sm;                     // [5][dc][dc]  (i, j)
    double2* Wn = acc + 5 * dc * dc;       // [df][Nv]
    double2* Wm = Wn + df * Nv;            // [df][Nv]
    double2* T = Wm + df * Nv;             // [df][dc]
    double2* Fs = T + df * dc;             // [df][df]: the hop's link matrix (levels >= 1)
    const int b = blockIdx.x;
    const int bx = b / g.agg_t, bt = b - bx * g.agg_t;
    for (int q = threadIdx.x; q < 5 * dc * dc; q += blockDim.x) acc[q] = make_double2(0.0, 0.0);
    for (int k = 0; k < g.el_x * g.el_t; k++) {
        const int kx = k / g.el_t, kt = k - kx * g.el_t;
        const int x = bx * g.el_x + kx, t = bt * g.el_t + kt;
        const int n = x * g.Nt + t;
        __syncthreads();
        for (int q = threadIdx.x; q < df * Nv; q += blockDim.x) {
            const int rr = q / Nv, p = q - rr * Nv;
            Wn[q] = tv[(long)p * g.size() + (long)n * df + rr];
        }
        for (int h = (g.level == 0 ? 1 : 0); h < 5; h++) {
            int m, D;
            switch (h) {
                case 0: m = n; D = 0; break;
                case 1: m = x * g.Nt + ((t + 1 == g.Nt) ? 0 : t + 1); D = (kt + 1 < g.el_t) ? 0 : 1; break;
                case 2: m = ((x + 1 == g.Nx) ? 0 : x + 1) * g.Nt + t; D = (kx + 1 < g.el_x) ? 0 : 2; break;
                case 3: m = x * g.Nt + ((t == 0) ? g.Nt - 1 : t - 1); D = (kt - 1 >= 0) ? 0 : 3; break;
                default: m = ((x == 0) ? g.Nx - 1 : x - 1) * g.Nt + t; D = (kx - 1 >= 0) ? 0 : 4; break;
            }
            __syncthreads();
            for (int q = threadIdx.x; q < df * Nv; q += blockDim.x) {
                const int rr = q / Nv, s = q - rr * Nv;
                Wm[q] = tv[(long)s * g.size() + (long)m * df + rr];
            }
            if (g.level > 0) {  // every T entry reads C values of the link: stage it once
                const double2* F = links + ((long)n * 5 + h) * df * df;
                for (int q = threadIdx.x; q < df * df; q += blockDim.x) Fs[q] = F[q];
            }
            __syncthreads();
            // T[(c,alf)][(s,bet)] = sum_b' F_h(n)[(c,alf)][(b',bet)] w_s(m)[b'][bet]
            for (int q = threadIdx.x; q < df * dc; q += blockDim.x) {
                const int rr = q / dc, cs = q - rr * dc;
                const int s = cs >> 1, bet = cs & 1;
                double2 a = make_double2(0.0, 0.0);
                if (g.level == 0) {
                    a = cmul(level0_link(U, g.Nx, g.Nt, n, h, rr, bet), Wm[bet * Nv + s]);
                } else {
                    for (int bb = 0; bb < C; bb++) {
                        const int jj = bb * 2 + bet;
                        a = cfma(Fs[jj * df + rr], Wm[jj * Nv + s], a);
                    }
                }
                T[q] = a;
            }
            __syncthreads();
            // Coarse[D][(p,alf)][(s,bet)] += sum_c conj(w_p(n)[c][alf]) T[(c,alf)][(s,bet)]
            double2* A = acc + D * dc * dc;
            for (int q = threadIdx.x; q < dc * dc; q += blockDim.x) {
                const int i = q / dc, j = q - i * dc;
                const int p = i >> 1, alf = i & 1;
                double2 a = A[q];
                for (int c = 0; c < C; c++) a = cfmac(Wn[(c * 2 + alf) * Nv + p], T[(c * 2 + alf) * dc + j], a);
                A[q] = a;
            }
        }
    }
    __syncthreads();
    // store as [site][d][j][i]
    for (int q = threadIdx.x; q < 5 * dc * dc; q += blockDim.x) {
        const int d = q / (dc * dc), rem = q - d * dc * dc, j = rem / dc, i = rem - j * dc;
        next[(long)b * 5 * dc * dc + q] = acc[d * dc * dc + i * dc + j];
    }
}
// Level 0 (dof 2, one colour): the same sums with all operands staged once per aggregate.  The
// per-hop loop above is latency bound there (four tiny hops per fine site, three barriers and a global
// round trip each); here the aggregate's test vectors with a one-site halo and its hop matrices come
// into shared memory together, and every thread then forms whole entries of the coarse links, each
// summing its (site, hop) terms in the order of the loop above, so the result is bit for bit the same.
__global__ void __launch_bounds__(256) build_links_l0_kernel(Geom g, const double2* __restrict__ U,
                                                             const double2* __restrict__ tv,
                                                             double2* __restrict__ next) {
    extern __shared__ double2 sm[];
    const int Nv = g.ntest, dc = 2 * Nv, ex = g.el_x, et = g.el_t, K = ex * et;
    const int hx = ex + 2, ht = et + 2;  // halo box of the aggregate
    double2* Wh = sm;                    // [hx * ht][2][Nv]: w_p(site)[alf]
    double2* F = Wh + (size_t)hx * ht * 2 * Nv;  // [K][5][2][2]: F_h(n_k)[alf][bet]
    const int b = blockIdx.x;
    const int bx = b / g.agg_t, bt = b - bx * g.agg_t;
    for (int q = threadIdx.x; q < hx * ht * 2 * Nv; q += blockDim.x) {
        const int site = q / (2 * Nv), r = q - site * 2 * Nv, alf = r / Nv, p = r - alf * Nv;
        const int lx = site / ht - 1, lt = site % ht - 1;
        int x = bx * ex + lx, t = bt * et + lt;
        x = x < 0 ? x + g.Nx : (x >= g.Nx ? x - g.Nx : x);
        t = t < 0 ? t + g.Nt : (t >= g.Nt ? t - g.Nt : t);
        Wh[q] = tv[(long)p * g.size() + ((long)x * g.Nt + t) * 2 + alf];
    }
    for (int q = threadIdx.x; q < K * 16; q += blockDim.x) {
        const int k = q / 16, h = 1 + (q / 4) % 4, alf = (q / 2) % 2, bet = q % 2;
        const int kx = k / et, kt = k - kx * et;
        const int n = (bx * ex + kx) * g.Nt + bt * et + kt;
        F[((size_t)k * 5 + h) * 4 + alf * 2 + bet] = level0_link(U, g.Nx, g.Nt, n, h, alf, bet);
    }
    __syncthreads();
    const int dd = dc * dc;
    for (int q = threadIdx.x; q < 5 * dd; q += blockDim.x) {
        const int D = q / dd, rem = q - D * dd, i = rem / dc, j = rem - i * dc;  // entry (i, j) of D
        const int p = i >> 1, alf = i & 1, s = j >> 1, bet = j & 1;
        double2 a = make_double2(0.0, 0.0);
        // the (site, hop) pairs whose hop lands in D, in the loop order above (sites, then hops 1-4);
        // a hop leaves the aggregate only from its edge, so D > 0 visits one row or column of sites
        for (int kx = 0; kx < ex; kx++) {
            if ((D == 2 && kx != ex - 1) || (D == 4 && kx != 0)) continue;
            for (int kt = 0; kt < et; kt++) {
                if ((D == 1 && kt != et - 1) || (D == 3 && kt != 0)) continue;
                const int k = kx * et + kt;
                const double2 wn = Wh[((size_t)(kx + 1) * ht + (kt + 1)) * 2 * Nv + alf * Nv + p];
#pragma unroll
                for (int h = 1; h < 5; h++) {
                    const bool inside = h == 1 ? kt + 1 < et : h == 2 ? kx + 1 < ex : h == 3 ? kt > 0 : kx > 0;
                    if ((inside ? 0 : h) != D) continue;
                    const int mx = kx + (h == 2) - (h == 4), mt = kt + (h == 1) - (h == 3);
                    const double2 wm = Wh[((size_t)(mx + 1) * ht + (mt + 1)) * 2 * Nv + bet * Nv + s];
                    const double2 t = cmul(F[((size_t)k * 5 + h) * 4 + alf * 2 + bet], wm);
                    a = cfmac(wn, t, a);
                }
            }
        }
        next[(long)b * 5 * dd + D * dd + j * dc + i] = a;  // [site][d][j][i]
    }
}

void launch_build_coarse_links(cudaStream_t s, const Geom& g, const double2* U, const double2* links,
                               const double2* tv, double2* next_links) {
    const int df = g.dof, dc = 2 * g.ntest;
    if (g.level == 0 && g.dof == 2) {
        const int K = g.el_x * g.el_t;
        const size_t smem = sizeof(double2) * ((size_t)(g.el_x + 2) * (g.el_t + 2) * 2 * g.ntest + (size_t)K * 20);
        DDAMG_CUDA_TRY(
            cudaFuncSetAttribute(build_links_l0_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DDAMG_LAUNCH(build_links_l0_kernel, g.agg_x * g.agg_t, 256, smem, s, g, U, tv, next_links);
        return;
    }
    size_t smem = sizeof(double2) * ((size_t)5 * dc * dc + 2 * (size_t)df * g.ntest + (size_t)df * dc + (size_t)df * df);
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(build_links_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DDAMG_LAUNCH(build_links_kernel, g.agg_x * g.agg_t, 256, smem, s, g, U, links, tv, next_links);
}

#define DDAMG_INST_COARSE(V)                                                                                   \
    template void launch_coarse_op<V>(cudaStream_t, const V*, const V*, V*, const V*, int, int, int, double, int); \
    template void launch_restrict<V>(cudaStream_t, const Geom&, const V*, const V*, V*, int);                  \
    template void launch_prolong<V>(cudaStream_t, const Geom&, const V*, const V*, V*, int, int);
DDAMG_INST_COARSE(double2)
DDAMG_INST_COARSE(float2)

}  // namespace ddamg
