// Coarse-level SAP colour sweep with the block GMRES control trimmed for latency
// (SAP_C::SAP inner loops, src/sap.cpp:48-77 and 104-139; FGMRES::fgmres with the identity
// preconditioner, src/fgmres.cpp:5-128, x0 = r_B as src/sap.cpp:65; block operator
// Level::SAP_level_l::D_local, src/level.cpp:607-653).
#include "internal.h"
#include "sap_common.cuh"

namespace ddamg {

// ---------------------------------------------------------------- coarse levels, restart length M
// The block solve of sap_block_kernel (RB right-hand sides of one Schwarz block per CTA, one block
// element per thread) restructured around what its phase timing showed (cycles per Arnoldi step at
// 256x256 level 1, FP64, one right-hand side: block-operator application 9.1 K, Gram-Schmidt warp
// butterfly 2.6 K, totals and update 1.9 K, Givens 1.9 K, barrier waits 3.5 K):
//  * the multi-value warp sums halve the value set at each of the first levels (a double2 costs four
//    32-bit shuffles per level, so six coefficients cost 120 shuffles as a plain butterfly, 36 here);
//  * the coefficients of all RB right-hand sides share one packed warp reduction (groups of eight), and
//    every warp forms the CTA totals of all of them at once from the warps' partial sums (a lane per
//    slot, then a butterfly over the lane groups; the same order in every warp, so all threads hold
//    bit-identical totals): one CTA barrier per reduction;
//  * warp 0 forms Hessenberg column j, the Givens rotation and the break flag after its own update;
//    the flag is read after the next step's first barrier, where the reference reads it;
//  * norms and the rotation use one reciprocal square root (1/sqrt(x) with 1 ulp error) instead of a
//    square root and divisions, and the triangular solve at a restart end multiplies by reciprocal
//    diagonal entries formed with the rotation, so no FP64 division sits on the critical path;
//  * the shared memory the Krylov basis leaves free caches the first `ncache` in-block link matrices
//    (self terms first), filled by the first block-operator application: later applications stream
//    only the rest from L2.
// The arithmetic is the single-vector FGMRES::fgmres of the reference (src/fgmres.cpp:5-128) with
// classical Gram-Schmidt; rounding differs from the reference's order at the ulp level.

// sum over the warp of 8 double2 values by recursive halving: afterwards every lane l holds the warp
// total of value ((l >> 2) & 7).  The values are separate arguments, so the lane-dependent selections
// stay register selects.
__device__ __forceinline__ double2 xor_shfl2(double2 a, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, a.x, o), __shfl_xor_sync(0xffffffffu, a.y, o));
}
__device__ __forceinline__ double2 sel2(bool c, double2 a, double2 b) {
    return make_double2(c ? a.x : b.x, c ? a.y : b.y);
}
__device__ __forceinline__ double2 warp_sum8(double2 v0, double2 v1, double2 v2, double2 v3, double2 v4, double2 v5,
                                             double2 v6, double2 v7) {
    const int lane = threadIdx.x & 31;
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
    // level 16: lanes with bit 4 keep values 4-7, the others 0-3
    const double2 a0 = sel2(h16, v4, v0) + xor_shfl2(sel2(h16, v0, v4), 16);
    const double2 a1 = sel2(h16, v5, v1) + xor_shfl2(sel2(h16, v1, v5), 16);
    const double2 a2 = sel2(h16, v6, v2) + xor_shfl2(sel2(h16, v2, v6), 16);
    const double2 a3 = sel2(h16, v7, v3) + xor_shfl2(sel2(h16, v3, v7), 16);
    // level 8: bit 3 keeps the upper pair
    const double2 c0 = sel2(h8, a2, a0) + xor_shfl2(sel2(h8, a0, a2), 8);
    const double2 c1 = sel2(h8, a3, a1) + xor_shfl2(sel2(h8, a1, a3), 8);
    // level 4: bit 2 keeps the odd value
    double2 d = sel2(h4, c1, c0) + xor_shfl2(sel2(h4, c0, c1), 4);
    d = d + xor_shfl2(d, 2);
    d = d + xor_shfl2(d, 1);
    return d;
}

// the warp sums of the RB x NV values val(r, q) (all right-hand sides packed into groups of eight, each
// value formed when its group is reduced) into this warp's partial-sum slots row[r * KS + q]
template <int RB, int NV, int KS, typename F>
__device__ __forceinline__ void warp_partials(F&& val, double2* row) {
    const int lane = threadIdx.x & 31;
    constexpr int NF = RB * NV, NG = (NF + 7) / 8;
#pragma unroll
    for (int gi = 0; gi < NG; gi++) {
        double2 v[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int f = gi * 8 + t;
            v[t] = f < NF ? val(f / NV, f % NV) : make_double2(0.0, 0.0);
        }
        const double2 tot = warp_sum8(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]);
        const int f = gi * 8 + ((lane >> 2) & 7);
        if ((lane & 3) == 0 && f < NF) row[(f / NV) * KS + f % NV] = tot;
    }
}
// CTA totals of the RB x KS slots of the warps' partial sums (warp w's at col + w * stride; slot q of each
// rhs only for q < cnt), formed by the calling warp and broadcast through its scratch tw[RB * KS]: lane l
// sums slot l % (RB*KS) over every (32 / (RB*KS))-th warp in two chains, and a butterfly over the lane
// groups finishes; the same order in every warp, so all threads hold bit-identical totals
template <int RB, int KS>
__device__ __forceinline__ void cta_totals(const double2* col, int stride, int nwe, int cnt, double2* tw) {
    constexpr int ST = RB * KS, NGR = 32 / ST;
    const int lane = threadIdx.x & 31, slot = lane % ST, g = lane / ST;
    double2 v0 = make_double2(0.0, 0.0), v1 = v0;
    if (slot % KS < cnt) {
        int ww = g;
        for (; ww + NGR < nwe; ww += 2 * NGR) {
            v0 = v0 + col[(size_t)ww * stride + slot];
            v1 = v1 + col[(size_t)(ww + NGR) * stride + slot];
        }
        if (ww < nwe) v0 = v0 + col[(size_t)ww * stride + slot];
    }
    double2 v = v0 + v1;
#pragma unroll
    for (int o = ST; o < 32; o <<= 1) v = v + xor_shfl2(v, o);
    __syncwarp();  // this warp's previous reads of tw are done
    if (lane < ST) tw[lane] = v;
    __syncwarp();
}

template <typename V, int RB, int M> struct Sap2Smem {
    static constexpr int kSlots = 8;  // per rhs: the Gram-Schmidt coefficients and the new norm (M + 2 <= 8)
    V* basis;       // (M+1) x RB x NE
    V* op;          // RB x NE: operand of the residual applications
    double2* red;   // 2 buffers x nwe x RB*kSlots: warp partial sums
    double2* tw;    // nwe x RB*kSlots: per-warp broadcast of the totals
    double2* H;     // RB x (M+1) x M, H[r][i*M + j]
    double2* gm;    // RB x (M+1)
    double2* cn;    // RB x M
    double2* sn;    // RB x M
    double2* dinv;  // RB x M: 1 / H[q][q] once column q is rotated
    double2* ct;    // RB x kSlots: step j's totals of rhs r for warp 0's lanes (slot j+1: the new norm)
    int* flag;      // RB x M: break flag of step j
    V* cache;       // ncache x dof x dof link matrices
    __device__ Sap2Smem(unsigned char* raw, int NE, int nwe) {
        double2* d = reinterpret_cast<double2*>(raw);
        red = d;
        tw = red + (size_t)2 * nwe * RB * kSlots;
        H = tw + (size_t)nwe * RB * kSlots;
        gm = H + RB * (M + 1) * M;
        cn = gm + RB * (M + 1);
        sn = cn + RB * M;
        dinv = sn + RB * M;
        ct = dinv + RB * M;
        flag = reinterpret_cast<int*>(ct + RB * kSlots);
        basis = reinterpret_cast<V*>(reinterpret_cast<double2*>(flag) + (RB * M + 3) / 4);
        op = basis + (size_t)(M + 1) * NE * RB;
        cache = op + (size_t)NE * RB;
    }
    static size_t bytes(int NE, int nwe) {  // without the link cache
        return sizeof(double2) * ((size_t)2 * nwe * RB * kSlots + (size_t)nwe * RB * kSlots +
                                  (size_t)RB * ((M + 1) * M + (M + 1) + 3 * M + kSlots) + (RB * M + 3) / 4) +
               sizeof(V) * (size_t)(M + 2) * NE * RB;
    }
};

template <typename V, int RB, int M, int CH, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) sap_block2_kernel(Geom g, const V* __restrict__ L, const V* __restrict__ rg,
                                                           V* __restrict__ xg, SapKParams p, int ncache) {
    typedef typename RealOf<V>::R R;
    typedef Sap2Smem<V, RB, M> SM;
    constexpr int KS = SM::kSlots;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int et = g.sel_t, ex = g.sel_x, S = ex * et, dof = g.dof, NE = S * dof;
    const int nwe = (NE + 31) >> 5;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int kb = blockIdx.x / p.ngroups, r0 = (blockIdx.x - kb * p.ngroups) * RB;
    constexpr int SL = RB * KS;  // partial-sum slots per warp
    bool act[RB];
    bool any = false;
#pragma unroll
    for (int r = 0; r < RB; r++) {
        act[r] = (r0 + r < p.nrhs) && !(p.done && p.done[r0 + r]);
        any |= act[r];
    }
    if (!any) return;
    SM sm(smraw, NE, nwe);
    const int blk = p.blocks[kb];
    const int bx = blk / g.sap_t, bt = blk - bx * g.sap_t;
    const R mm = R(p.m0) + R(2);
    int rbuf = 0;

    const int e = threadIdx.x;
    const bool ev = e < NE;
    const int k = ev ? e / dof : 0, i = ev ? e - k * dof : 0;
    const int kx = k / et, kt = k - kx * et;
    const int n = (bx * ex + kx) * g.Nt + bt * et + kt;
    int nbk[5], cslot[5];
    nbk[0] = k;
    nbk[1] = (kt + 1 < et) ? k + 1 : -1;
    nbk[2] = (kx + 1 < ex) ? k + et : -1;
    nbk[3] = (kt > 0) ? k - 1 : -1;
    nbk[4] = (kx > 0) ? k - et : -1;
    {  // cache slots of the in-block matrices: self terms, then +t, +x, -t, -x hops
        const int b1 = S, b2 = b1 + ex * (et - 1), b3 = b2 + (ex - 1) * et, b4 = b3 + ex * (et - 1);
        cslot[0] = k;
        cslot[1] = b1 + kx * (et - 1) + kt;
        cslot[2] = b2 + kx * et + kt;
        cslot[3] = b3 + kx * (et - 1) + kt - 1;
        cslot[4] = b4 + (kx - 1) * et + kt;
    }
    const int dd2 = dof * dof;
    V b[RB], x[RB], w[RB];
    const V* __restrict__ vres = static_cast<const V*>(p.vres);
    if (!vres) {
#pragma unroll
        for (int r = 0; r < RB; r++) b[r] = (ev && act[r]) ? rg[(long)(r0 + r) * g.size() + (long)n * dof + i] : czero<V>();
    } else {
        // r_B = v - D x on this block's sites, all five hops, each link element loaded once for the CTA's
        // right-hand sides (the iterate of the other colour's blocks is final: the previous sweep has
        // finished); Level::D_operator (src/level.cpp:394-426) restricted to the block's sites.
        // The iterate at the five neighbours of every block site is staged first in the Krylov basis's
        // space (unused until the first restart; 5 <= M + 1 vectors per rhs), with independent coalesced
        // loads, so the link chains below wait on link loads only (several in flight), not on one operand
        // round trip per column pair.
        V* const stg = sm.basis;  // [d][r][NE]: x_{r0+r} at site nbr_d(k), entry j, at (d * RB + r) * NE + k * dof + j
        for (int q = threadIdx.x; q < 5 * RB * NE; q += blockDim.x) {
            const int d = q / (RB * NE), rem = q - d * RB * NE, r = rem / NE, el = rem - r * NE;
            const int kq = el / dof, jq = el - kq * dof, qkx = kq / et;
            const int qx = bx * ex + qkx, qt = bt * et + (kq - qkx * et);
            int nb = qx * g.Nt + qt;
            if (d == 1) nb = qx * g.Nt + (qt + 1 == g.Nt ? 0 : qt + 1);
            else if (d == 2) nb = (qx + 1 == g.Nx ? 0 : qx + 1) * g.Nt + qt;
            else if (d == 3) nb = qx * g.Nt + (qt == 0 ? g.Nt - 1 : qt - 1);
            else if (d == 4) nb = (qx == 0 ? g.Nx - 1 : qx - 1) * g.Nt + qt;
            stg[q] = (r0 + r < p.nrhs) ? xg[(long)(r0 + r) * g.size() + (long)nb * dof + jq] : czero<V>();
        }
        __syncthreads();
        V acc[RB];
#pragma unroll
        for (int r = 0; r < RB; r++) acc[r] = czero<V>();
        if (ev) {
            const int gt = bt * et + kt;
#pragma unroll 1
            for (int d = 0; d < 5; d++) {
                const R sg = ((d == 1 && gt == g.Nt - 1) || (d == 3 && gt == 0)) ? R(-1) : R(1);
                const V* Mt = L + ((long)n * 5 + d) * dd2 + i;
                const V* xs = stg + (size_t)d * RB * NE + (size_t)k * dof;
                // an in-block hop with a cache slot is kept on the way, so the first application reads it
                // from shared memory
                int nbd = nbk[0], csd = cslot[0];  // selects, not a dynamic index (which would put the
#pragma unroll                                     // arrays in local memory)
                for (int h = 1; h < 5; h++)
                    if (h == d) {
                        nbd = nbk[h];
                        csd = cslot[h];
                    }
                const bool keep = nbd >= 0 && csd < ncache;
                V* Mc = sm.cache + (size_t)csd * dd2 + i;
                V ae[RB], ao[RB];  // even and odd columns: two independent chains per right-hand side
#pragma unroll
                for (int r = 0; r < RB; r++) ae[r] = ao[r] = czero<V>();
                constexpr int RCH = CH;  // link loads in flight (even)
                int j = 0;
                for (; j + RCH <= dof; j += RCH) {
                    V mv[RCH];
#pragma unroll
                    for (int u = 0; u < RCH; u++) mv[u] = __ldg(Mt + (long)(j + u) * dof);
                    if (keep)
#pragma unroll
                        for (int u = 0; u < RCH; u++) Mc[(size_t)(j + u) * dof] = mv[u];
#pragma unroll
                    for (int u = 0; u < RCH; u += 2)
#pragma unroll
                        for (int r = 0; r < RB; r++) {
                            ae[r] = cfma(mv[u], xs[(size_t)r * NE + j + u], ae[r]);
                            ao[r] = cfma(mv[u + 1], xs[(size_t)r * NE + j + u + 1], ao[r]);
                        }
                }
                for (; j < dof; j += 2) {  // dof is even
                    const V m0 = __ldg(Mt + (long)j * dof), m1 = __ldg(Mt + (long)(j + 1) * dof);
                    if (keep) {
                        Mc[(size_t)j * dof] = m0;
                        Mc[(size_t)(j + 1) * dof] = m1;
                    }
#pragma unroll
                    for (int r = 0; r < RB; r++) {
                        ae[r] = cfma(m0, xs[(size_t)r * NE + j], ae[r]);
                        ao[r] = cfma(m1, xs[(size_t)r * NE + j + 1], ao[r]);
                    }
                }
#pragma unroll
                for (int r = 0; r < RB; r++) acc[r] = acc[r] + sg * (ae[r] + ao[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < RB; r++) {
            const long o = (long)(r0 + r) * g.size() + (long)n * dof + i;
            b[r] = (ev && act[r]) ? vres[o] - (mm * xg[o] - acc[r]) : czero<V>();
        }
    }
#pragma unroll
    for (int r = 0; r < RB; r++) x[r] = b[r];

    // w = D_B op for the RB vectors op[r * NE + .]; fill: keep the cached matrices while loading them
    auto apply = [&](const V* op, bool fill) {
        V acc[RB][2];
#pragma unroll
        for (int r = 0; r < RB; r++) acc[r][0] = acc[r][1] = czero<V>();
        if (!ev) {
#pragma unroll
            for (int r = 0; r < RB; r++) w[r] = czero<V>();
            return;
        }
#pragma unroll
        for (int d = 0; d < 5; d++) {
            const int kk = nbk[d];
            if (kk < 0) continue;
            const V* o = op + (size_t)kk * dof;
            const bool cached = cslot[d] < ncache;
            V* Mc = sm.cache + (size_t)cslot[d] * dd2 + i;
            if (cached && !fill) {
                for (int j = 0; j < dof; j += 2) {  // dof is even
                    const V m0 = Mc[(size_t)j * dof], m1 = Mc[(size_t)(j + 1) * dof];
#pragma unroll
                    for (int r = 0; r < RB; r++) {
                        acc[r][0] = cfma(m0, o[(size_t)r * NE + j], acc[r][0]);
                        acc[r][1] = cfma(m1, o[(size_t)r * NE + j + 1], acc[r][1]);
                    }
                }
                continue;
            }
            const V* Mt = L + ((long)n * 5 + d) * dd2 + i;
            int j = 0;
            for (; j + CH <= dof; j += CH) {  // CH link loads in flight
                V mv[CH];
#pragma unroll
                for (int u = 0; u < CH; u++) mv[u] = __ldg(Mt + (long)(j + u) * dof);
                if (cached)
#pragma unroll
                    for (int u = 0; u < CH; u++) Mc[(size_t)(j + u) * dof] = mv[u];
#pragma unroll
                for (int u = 0; u < CH; u++)
#pragma unroll
                    for (int r = 0; r < RB; r++) acc[r][u & 1] = cfma(mv[u], o[(size_t)r * NE + j + u], acc[r][u & 1]);
            }
            for (; j < dof; j++) {
                const V mv = __ldg(Mt + (long)j * dof);
                if (cached) Mc[(size_t)j * dof] = mv;
#pragma unroll
                for (int r = 0; r < RB; r++) acc[r][0] = cfma(mv, o[(size_t)r * NE + j], acc[r][0]);
            }
        }
#pragma unroll
        for (int r = 0; r < RB; r++) w[r] = mm * op[(size_t)r * NE + e] - (acc[r][0] + acc[r][1]);
    };
    constexpr int NV = M + 1;  // values per rhs in a reduction: the dots and the new norm
    // this warp's partial sums of values 0..nv-1 of all right-hand sides into buffer rbuf (the slots from
    // nv on keep older sums, which the totals below never read)
#define SAP2_PARTIAL(nv, val) warp_partials<RB, nv, KS>(val, sm.red + ((size_t)rbuf * nwe + wid) * SL)
    // CTA totals of slots 0..cnt of every rhs in buffer buf (every warp forms them itself); then
    // SAP2_TOT(r, q) is total q of rhs r
#define SAP2_TOTALS(buf, cnt) cta_totals<RB, KS>(sm.red + (size_t)(buf) * nwe * SL, SL, nwe, cnt, twp)
#define SAP2_TOT(r, q) twp[(r) * KS + (q)]
    double2* const twp = sm.tw + (size_t)wid * SL;  // this warp's copy of the totals

    // x = x0 = b; r = b - D_B x (this application fills the link cache, unless the fused residual did)
#pragma unroll
    for (int r = 0; r < RB; r++)
        if (ev) sm.op[(size_t)r * NE + e] = x[r];
    __syncthreads();
    apply(sm.op, vres == nullptr);
    double norm_b[RB], err[RB];
    bool fin[RB];  // converged, inactive, or a zero right-hand side
    int maxIt[RB];
#pragma unroll
    for (int r = 0; r < RB; r++) w[r] = b[r] - w[r];
    SAP2_PARTIAL(2, [&](int r, int q) {  // ||b||^2, ||r||^2
        return make_double2(ev ? (double)cnorm2(q == 0 ? b[r] : w[r]) : 0.0, 0.0);
    });
    __syncthreads();
    SAP2_TOTALS(rbuf, 2);
#pragma unroll
    for (int r = 0; r < RB; r++) {
        norm_b[r] = sqrt(SAP2_TOT(r, 0).x);
        err[r] = sqrt(SAP2_TOT(r, 1).x);
        // a zero block right-hand side has the zero solution (the reference would divide by zero)
        fin[r] = !act[r] || norm_b[r] == 0.0;
        maxIt[r] = M;
    }
    rbuf ^= 1;
    for (int kr = 0; kr < p.restarts; kr++) {
        bool arn[RB], anyarn = false;
#pragma unroll
        for (int r = 0; r < RB; r++) {
            arn[r] = !fin[r];
            anyarn |= arn[r];
        }
        if (!anyarn) break;
#pragma unroll
        for (int r = 0; r < RB; r++) {  // V_0 = r / beta
            if (!arn[r]) continue;
            const R inv = R(1.0 / err[r]);
            if (ev) sm.basis[(size_t)r * NE + e] = inv * w[r];
            if (wid == 0 && lane == 0) sm.gm[r * (M + 1)] = make_double2(err[r], 0.0);
        }
        // warp 0: column jr of every active rhs's Hessenberg matrix, its Givens rotation and break flag
        // (FGMRES::rotation, src/fgmres.cpp:99-115), from the totals of step jr in ct
        auto rotate = [&](int jr) {
            __syncwarp();
            bool a = false;
            double nbr = 0.0;
#pragma unroll
            for (int r = 0; r < RB; r++)
                if (r == lane) {
                    a = arn[r];
                    nbr = norm_b[r];
                }
            if (lane < RB && a) {  // lane r: Hessenberg column jr of rhs r
                const int r = lane;
                double2* H = sm.H + r * (M + 1) * M;
                double2* cn = sm.cn + r * M;
                double2* sn = sm.sn + r * M;
                double2* gm = sm.gm + r * (M + 1);
                const double2* ct = sm.ct + r * KS;
                double2 hc[M + 1];
#pragma unroll
                for (int q = 0; q <= M; q++) hc[q] = (q <= jr + 1) ? ct[q] : make_double2(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < M; q++) {  // FGMRES::rotation (src/fgmres.cpp:99-115)
                    if (q >= jr) break;
                    const double2 tmp = cmulc(cn[q], hc[q]) + cmulc(sn[q], hc[q + 1]);
                    hc[q + 1] = cmul(cn[q], hc[q + 1]) - cmul(sn[q], hc[q]);
                    hc[q] = tmp;
                }
                double2 hjj = make_double2(0.0, 0.0), hj1 = hjj;
#pragma unroll
                for (int q = 0; q < M; q++)
                    if (q == jr) {
                        hjj = hc[q];
                        hj1 = hc[q + 1];
                    }
                const double iden = rsqrt(cnorm2(hjj) + cnorm2(hj1));
                const double2 s_j = make_double2(hj1.x * iden, hj1.y * iden);
                const double2 c_j = make_double2(hjj.x * iden, hjj.y * iden);
                sn[jr] = s_j;
                cn[jr] = c_j;
                const double2 hd = cmulc(c_j, hjj) + cmulc(s_j, hj1);
#pragma unroll
                for (int q = 0; q < M; q++) {
                    if (q > jr) break;
                    H[q * M + jr] = (q == jr) ? hd : hc[q];
                }
                const double id2 = 1.0 / cnorm2(hd);
                sm.dinv[r * M + jr] = make_double2(hd.x * id2, -hd.y * id2);
                const double2 gj = gm[jr];
                const double2 g1 = -cmul(s_j, gj);
                gm[jr + 1] = g1;
                gm[jr] = cmulc(c_j, gj);
                const double thr = p.tol * nbr;
                sm.flag[r * M + jr] = (cnorm2(g1) < thr * thr) ? 1 : 0;
            }
        };
        // The rotation of step j - 1 runs on warp 0 after its share of step j's application (warp 0's sites
        // have fewer in-block hops than the busiest warps'), and its break flags are read after step j's
        // partial-sum barrier: a rhs that met the tolerance at step j - 1 drops out there, its step-j values
        // unused: the arithmetic of the step-by-step order.
        int jdone = 0;
        for (int j = 0; j < M; j++) {
            __syncthreads();  // v_j complete
            apply(sm.basis + (size_t)j * NE * RB, false);  // w = D_B V_j
            if (j > 0 && wid == 0) rotate(j - 1);
            // classical Gram-Schmidt coefficients <w, V_i>, i <= j, and ||w||^2 (slot j + 1)
            // (selects on j, not a store at index j + 1, which would put the values in local memory)
            {
                auto gs = [&](int r, int q) {
                    double2 v = make_double2(0.0, 0.0);
                    if (arn[r] && ev) {
                        if (q <= j) v = cfmac(to_d(sm.basis[((size_t)q * RB + r) * NE + e]), to_d(w[r]), v);
                        v.x += (q == j + 1) ? (double)cnorm2(w[r]) : 0.0;
                    }
                    return v;
                };
                // the j + 2 live values of each rhs packed densely: fewer warp-sum groups for early j (the
                // sum of a value does not depend on its place in the group)
                static_assert(M == 5, "the restart length of this kernel is 5");
                if (j == 0) SAP2_PARTIAL(2, gs);
                else if (j == 1) SAP2_PARTIAL(3, gs);
                else if (j == 2) SAP2_PARTIAL(4, gs);
                else if (j == 3) SAP2_PARTIAL(5, gs);
                else SAP2_PARTIAL(6, gs);
            }
            __syncthreads();  // partial sums visible; warp 0's step j - 1 (flags, Hessenberg) visible
            if (j > 0) {
                anyarn = false;
#pragma unroll
                for (int r = 0; r < RB; r++) {
                    if (arn[r] && sm.flag[r * M + j - 1]) {
                        maxIt[r] = j;  // not reset at the next restart (src/fgmres.cpp:14,56)
                        arn[r] = false;
                    }
                    anyarn |= arn[r];
                }
                if (!anyarn) break;
            }
            const int dbuf = rbuf;
            rbuf ^= 1;
            // ||w - V h||^2 = ||w||^2 - sum |h_i|^2 for orthonormal V: no second reduction, unless the
            // difference cancels below 1e-4 of ||w||^2 (1e-2 for an FP32 basis, whose orthogonality holds
            // to ~1e-6); then the norm of the updated w is reduced as is
            constexpr double kCancel = sizeof(R) == 8 ? 1e-4 : 1e-2;
            double hn[RB], ihn[RB];
            bool reduce_norm = false;
            SAP2_TOTALS(dbuf, j + 2);
#pragma unroll
            for (int r = 0; r < RB; r++) {
                hn[r] = 0.0;
                ihn[r] = 0.0;
                if (!arn[r]) continue;
                double2 t[NV];
#pragma unroll
                for (int q = 0; q < NV; q++) t[q] = q <= j + 1 ? SAP2_TOT(r, q) : make_double2(0.0, 0.0);
                double w2 = 0.0, hh = 0.0;
#pragma unroll
                for (int q = 0; q <= M; q++) {
                    if (q <= j) hh += cnorm2(t[q]);
                    else if (q == j + 1) w2 = t[q].x;
                }
                const double dd = w2 - hh;
                if (dd > kCancel * w2) {
                    ihn[r] = rsqrt(dd);
                    hn[r] = dd * ihn[r];
                } else {
                    reduce_norm = true;  // identical in every thread: the totals are
                }
                if (ev) {
#pragma unroll
                    for (int q = 0; q <= M; q++)
                        if (q <= j) w[r] = w[r] - cmul(from_d<V>(t[q]), sm.basis[((size_t)q * RB + r) * NE + e]);
                }
                if (wid == 0 && lane == 0)
#pragma unroll
                    for (int q = 0; q <= M; q++)
                        if (q <= j) sm.ct[r * KS + q] = t[q];
            }
            if (reduce_norm) {
                SAP2_PARTIAL(1, [&](int r, int q) {
                    return make_double2(arn[r] && ev ? (double)cnorm2(w[r]) : 0.0, 0.0);
                });
                __syncthreads();
                SAP2_TOTALS(rbuf, 1);
#pragma unroll
                for (int r = 0; r < RB; r++) {
                    const double t0 = SAP2_TOT(r, 0).x;
                    if (arn[r] && t0 > 0) {
                        ihn[r] = rsqrt(t0);
                        hn[r] = t0 * ihn[r];
                    }
                }
                rbuf ^= 1;
            }
#pragma unroll
            for (int r = 0; r < RB; r++) {
                if (arn[r] && hn[r] > 0 && ev) sm.basis[((size_t)(j + 1) * RB + r) * NE + e] = R(ihn[r]) * w[r];
                if (wid == 0 && lane == 0) sm.ct[r * KS + j + 1] = make_double2(hn[r], 0.0);
            }
            jdone = j + 1;
        }
        if (jdone == M && wid == 0) rotate(M - 1);  // the last step's column
        __syncthreads();  // the last step's Hessenberg column and rotations visible
        // solve_upper_triangular (src/fgmres.cpp:118-128), repeated by every thread; x += sum eta_j V_j
#pragma unroll
        for (int r = 0; r < RB; r++) {
            if (fin[r]) continue;
            const double2* H = sm.H + r * (M + 1) * M;
            const double2* gmr = sm.gm + r * (M + 1);
            const double2* di = sm.dinv + r * M;
            double2 eta[M];
#pragma unroll
            for (int q = M - 1; q >= 0; q--) {
                eta[q] = make_double2(0.0, 0.0);
                if (q >= maxIt[r]) continue;
                double2 t = gmr[q];
#pragma unroll
                for (int jj = q + 1; jj < M; jj++)
                    if (jj < maxIt[r]) t = t - cmul(H[q * M + jj], eta[jj]);
                eta[q] = cmul(t, di[q]);
            }
            if (ev) {
                V a = x[r];
#pragma unroll
                for (int jj = 0; jj < M; jj++)
                    if (jj < maxIt[r]) a = cfma(from_d<V>(eta[jj]), sm.basis[((size_t)jj * RB + r) * NE + e], a);
                x[r] = a;
            }
        }
#pragma unroll
        for (int r = 0; r < RB; r++)
            if (ev) sm.op[(size_t)r * NE + e] = x[r];
        __syncthreads();
        apply(sm.op, false);
#pragma unroll
        for (int r = 0; r < RB; r++) w[r] = b[r] - w[r];
        SAP2_PARTIAL(1, [&](int r, int q) { return make_double2(ev ? (double)cnorm2(w[r]) : 0.0, 0.0); });
        __syncthreads();
        SAP2_TOTALS(rbuf, 1);
#pragma unroll
        for (int r = 0; r < RB; r++) {
            err[r] = sqrt(SAP2_TOT(r, 0).x);
            if (!fin[r] && err[r] < p.tol * norm_b[r]) fin[r] = true;
        }
        rbuf ^= 1;
    }
    // x_B += e  (src/sap.cpp:106-113)
#pragma unroll
    for (int r = 0; r < RB; r++) {
        if (!act[r] || norm_b[r] == 0.0 || !ev) continue;
        V* o = xg + (long)(r0 + r) * g.size() + (long)n * dof + i;
        *o = *o + x[r];
    }
#undef SAP2_PARTIAL
#undef SAP2_TOTALS
#undef SAP2_TOT
}

// the kernel takes blocks of at most 512 unknowns at restart length 5 with 1, 2 or 4 right-hand sides
// per CTA, where its shared memory (without the link cache) fits
constexpr int kSap2M = 5;
template <typename V> static size_t sap2_base_bytes(int rb, int NE) {
    const int nwe = (NE + 31) / 32;
    return rb == 1 ? Sap2Smem<V, 1, kSap2M>::bytes(NE, nwe)
                   : rb == 2 ? Sap2Smem<V, 2, kSap2M>::bytes(NE, nwe) : Sap2Smem<V, 4, kSap2M>::bytes(NE, nwe);
}
bool sap2_fits(int rb, int m, int NE, size_t vbytes) {
    if (m != kSap2M || NE > 512 || !(rb == 1 || rb == 2 || rb == 4)) return false;
    const size_t smem = vbytes == 16 ? sap2_base_bytes<double2>(rb, NE) : sap2_base_bytes<float2>(rb, NE);
    return smem <= 227 * 1024;
}
template <typename V, int RB, int CH, int MAXT>
static void launch_sap2_k(cudaStream_t s, const Geom& g, const V* L, const V* r, V* x, SapKParams p) {
    const int ex = g.sel_x, et = g.sel_t, S = ex * et, NE = S * g.dof;
    const int nwe = (NE + 31) / 32;
    p.ngroups = (p.nrhs + RB - 1) / RB;
    const size_t base = Sap2Smem<V, RB, kSap2M>::bytes(NE, nwe);
    // link matrices in the rest of the 227 KB: at most the block's in-block (site, hop) pairs
    const int inblock = S + 2 * ex * (et - 1) + 2 * (ex - 1) * et;
    const size_t mat = sizeof(V) * (size_t)g.dof * g.dof;
    const int ncache = (int)std::min<size_t>(inblock, (227 * 1024 - base) / mat);
    const size_t smem = base + (size_t)ncache * mat;
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(sap_block2_kernel<V, RB, kSap2M, CH, MAXT>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DDAMG_LAUNCH((sap_block2_kernel<V, RB, kSap2M, CH, MAXT>), dim3(p.nblocks * p.ngroups), 32 * nwe, smem, s, g, L, r,
                 x, p, ncache);
}
template <typename V, int RB>
void launch_sap2(cudaStream_t s, const Geom& g, const V* L, const V* r, V* x, SapKParams p) {
    const int NE = g.sel_x * g.sel_t * g.dof;
    if (NE <= 384) launch_sap2_k<V, RB, 12, 384>(s, g, L, r, x, p);
    else launch_sap2_k<V, RB, 8, 512>(s, g, L, r, x, p);
}

template void launch_sap2<double2, 1>(cudaStream_t, const Geom&, const double2*, const double2*, double2*, SapKParams);
template void launch_sap2<double2, 2>(cudaStream_t, const Geom&, const double2*, const double2*, double2*, SapKParams);
template void launch_sap2<double2, 4>(cudaStream_t, const Geom&, const double2*, const double2*, double2*, SapKParams);
template void launch_sap2<float2, 1>(cudaStream_t, const Geom&, const float2*, const float2*, float2*, SapKParams);
template void launch_sap2<float2, 2>(cudaStream_t, const Geom&, const float2*, const float2*, float2*, SapKParams);
template void launch_sap2<float2, 4>(cudaStream_t, const Geom&, const float2*, const float2*, float2*, SapKParams);

}  // namespace ddamg
