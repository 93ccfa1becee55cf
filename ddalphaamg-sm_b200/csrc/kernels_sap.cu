// SAP colour sweep (SAP_C::SAP inner loops, src/sap.cpp:48-77 and 104-139): for every Schwarz
// block of one colour solve D_B e = r_B with GMRES(m) x restarts (FGMRES::fgmres with the identity
// preconditioner, src/fgmres.cpp:5-97, x0 = r_B as src/sap.cpp:65) and add e to x on the block.
// One CTA per (block, rhs); the block's Krylov basis lives in shared memory, the block-local
// operator (Level::SAP_level_l::D_local, src/level.cpp:607-653: neighbours outside the block
// read as zero, no boundary sign) streams the level's links.
#include "internal.h"
#include "sap_common.cuh"

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

constexpr int kGsBatch = 6;  // Gram-Schmidt coefficients per interleaved butterfly (restart length 5: all)

// Shared memory of one CTA: RB right-hand sides of one Schwarz block.  Vectors are stored
// [rhs][element], so a warp's Gram-Schmidt loads and stores of one right-hand side are
// contiguous (no bank conflicts); the operator's operand reads are broadcasts either way.
template <typename V, int RB> struct SapSmem {
    V* basis;      // (m+1) x RB x NE
    V* op;         // RB x NE: operand of D_B
    double2* red;  // 2 buffers x warps x RB*(kSapMaxM+1): reductions
    double2* H;    // RB x (m+1) x m, H[r][i*m + j]
    double2* gm;   // RB x (m+1)
    double2* cn;   // RB x m
    double2* sn;   // RB x m
    double2* eta;  // RB x m
    double2* tot;  // RB x (kSapMaxM+1): CTA totals of the Gram-Schmidt coefficients
    int* flag;     // RB: the Arnoldi estimate met tol
    __device__ SapSmem(unsigned char* raw, int m, int NE, int nw) {
        double2* d = reinterpret_cast<double2*>(raw);
        red = d;
        H = red + (size_t)2 * nw * RB * (kSapMaxM + 1);
        gm = H + RB * (m + 1) * m;
        cn = gm + RB * (m + 1);
        sn = cn + RB * m;
        eta = sn + RB * m;
        tot = eta + RB * m;
        flag = reinterpret_cast<int*>(tot + RB * (kSapMaxM + 1));
        basis = reinterpret_cast<V*>(flag + ((RB + 3) / 4) * 4);
        op = basis + (size_t)(m + 1) * NE * RB;
    }
    static size_t bytes(int m, int NE, int nw) {
        return sizeof(double2) * ((size_t)2 * nw * RB * (kSapMaxM + 1) +
                                  (size_t)RB * ((m + 1) * m + (m + 1) + 3 * m + kSapMaxM + 1)) +
               sizeof(int) * ((RB + 3) / 4) * 4 + sizeof(V) * (size_t)(m + 2) * NE * RB;
    }
};

// One SAP colour sweep for RB right-hand sides of one Schwarz block in lockstep: each link
// element is loaded once and applied to all RB vectors; every right-hand side keeps its own
// Hessenberg matrix, rotations, break point (maxIt) and convergence state, and freezes once it
// has finished, so each follows exactly the single-vector algorithm of FGMRES::fgmres.
template <typename V, bool DENSE, int EPT, int MAXT, int RB, int CH>
__global__ void __launch_bounds__(MAXT, 1) sap_block_kernel(Geom g, const V* __restrict__ L, const V* __restrict__ rg,
                                                         V* __restrict__ xg, SapKParams p) {
    typedef typename RealOf<V>::R R;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int S = g.sel_x * g.sel_t, dof = g.dof, NE = S * dof;
    const int nw = (blockDim.x + 31) >> 5, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // block-major order: the CTAs of one Schwarz block run side by side and share its links in L2
    const int kb = blockIdx.x / p.ngroups, r0 = (blockIdx.x - kb * p.ngroups) * RB;
    bool act[RB];
    bool any = false;
#pragma unroll
    for (int r = 0; r < RB; r++) {
        act[r] = (r0 + r < p.nrhs) && !(p.done && p.done[r0 + r]);
        any |= act[r];
    }
    if (!any) return;
    SapSmem<V, RB> sm(smraw, p.m, NE, nw);
    const int blk = p.blocks[kb];
    const int bx = blk / g.sap_t, bt = blk - bx * g.sap_t;
    const R mm = R(p.m0) + R(2);
    const int m = p.m;
    constexpr int SL = RB * (kSapMaxM + 1);  // reduction slots per warp
    int rbuf = 0;

    int ek[EPT], ei[EPT], en[EPT], nbk[EPT][5];
    bool ev[EPT];
    V b[EPT][RB], x[EPT][RB], w[EPT][RB];
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
#pragma unroll
        for (int r = 0; r < RB; r++) {
            b[q][r] = (ev[q] && act[r]) ? rg[(long)(r0 + r) * g.size() + (long)en[q] * dof + i] : czero<V>();
            x[q][r] = b[q][r];
        }
    }
    // level 0: the block operator's eight 2x2-hop coefficients of each owned element are
    // formed once from U (they do not change during the block solve)
    V hop[EPT][DENSE ? 1 : 8];
    if (!DENSE) {
#pragma unroll
        for (int q = 0; q < EPT; q++)
#pragma unroll
            for (int d = 1; d < 5; d++)
#pragma unroll
                for (int bet = 0; bet < 2; bet++)
                    hop[q][DENSE ? 0 : (d - 1) * 2 + bet] =
                        (ev[q] && nbk[q][d] >= 0) ? level0_hop(L, g.Nx, g.Nt, en[q], d, ei[q], bet) : czero<V>();
    }
    auto sidx = [&](int q) { return threadIdx.x + q * blockDim.x; };
    // warp partial of one reduction slot; totals are read after the next __syncthreads
    auto partial = [&](double2 v, int slot) {
        v = warp_sum(v);
        if (lane == 0) sm.red[((size_t)rbuf * nw + wid) * SL + slot] = v;
    };
    auto total = [&](int buf, int slot) {  // four independent load/add chains over the warps
        const double2* pr = sm.red + (size_t)buf * nw * SL + slot;
        double2 t0 = make_double2(0.0, 0.0), t1 = t0, t2 = t0, t3 = t0;
        int ww = 0;
        for (; ww + 4 <= nw; ww += 4) {
            t0 += pr[(ww + 0) * SL];
            t1 += pr[(ww + 1) * SL];
            t2 += pr[(ww + 2) * SL];
            t3 += pr[(ww + 3) * SL];
        }
        for (; ww < nw; ww++) t0 += pr[ww * SL];
        return (t0 + t1) + (t2 + t3);
    };

    // w = D_B op for all RB vectors (op in shared memory, fully written before the call)
    auto apply = [&](const V* op) {
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            V acc[RB][2];
#pragma unroll
            for (int r = 0; r < RB; r++) acc[r][0] = acc[r][1] = czero<V>();
            if (!ev[q]) {
#pragma unroll
                for (int r = 0; r < RB; r++) w[q][r] = czero<V>();
                continue;
            }
            const int k = ek[q], i = ei[q], n = en[q];
            if (DENSE) {
#pragma unroll
                for (int d = 0; d < 5; d++) {
                    const int kk = nbk[q][d];
                    if (kk < 0) continue;
                    const V* M = L + ((long)n * 5 + d) * dof * dof + i;
                    const V* o = op + (size_t)kk * dof;  // vector r at o[r * NE + j]
                    int j = 0;
                    for (; j + CH <= dof; j += CH) {  // CH link loads in flight
                        V mv[CH];
#pragma unroll
                        for (int u = 0; u < CH; u++) mv[u] = __ldg(M + (long)(j + u) * dof);
#pragma unroll
                        for (int u = 0; u < CH; u++)
#pragma unroll
                            for (int r = 0; r < RB; r++) acc[r][u & 1] = cfma(mv[u], o[(size_t)r * NE + j + u], acc[r][u & 1]);
                    }
                    for (; j + 8 <= dof; j += 8) {  // 8 link loads in flight
                        V mv[8];
#pragma unroll
                        for (int u = 0; u < 8; u++) mv[u] = __ldg(M + (long)(j + u) * dof);
#pragma unroll
                        for (int u = 0; u < 8; u++)
#pragma unroll
                            for (int r = 0; r < RB; r++) acc[r][u & 1] = cfma(mv[u], o[(size_t)r * NE + j + u], acc[r][u & 1]);
                    }
                    for (; j < dof; j++) {
                        const V mv = __ldg(M + (long)j * dof);
#pragma unroll
                        for (int r = 0; r < RB; r++) acc[r][0] = cfma(mv, o[(size_t)r * NE + j], acc[r][0]);
                    }
                }
            } else {
#pragma unroll
                for (int d = 1; d < 5; d++) {
                    const int kk = nbk[q][d];
                    if (kk < 0) continue;
                    const V h0 = hop[q][DENSE ? 0 : (d - 1) * 2], h1 = hop[q][DENSE ? 0 : (d - 1) * 2 + 1];
#pragma unroll
                    for (int r = 0; r < RB; r++) {
                        acc[r][0] = cfma(h0, op[(size_t)r * NE + kk * 2], acc[r][0]);
                        acc[r][1] = cfma(h1, op[(size_t)r * NE + kk * 2 + 1], acc[r][1]);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < RB; r++) w[q][r] = mm * op[(size_t)r * NE + k * dof + i] - (acc[r][0] + acc[r][1]);
        }
    };
    auto store_op = [&](V (&v)[EPT][RB]) {
#pragma unroll
        for (int q = 0; q < EPT; q++)
            if (ev[q])
#pragma unroll
                for (int r = 0; r < RB; r++) sm.op[(size_t)r * NE + sidx(q)] = v[q][r];
    };

    // x = x0 = b; r = b - D_B x
    store_op(x);
    __syncthreads();
    apply(sm.op);
    double norm_b[RB], err[RB];
    bool fin[RB];  // converged, inactive, or a zero right-hand side
    int maxIt[RB];
#pragma unroll
    for (int r = 0; r < RB; r++) {
        double bb = 0.0, rr = 0.0;
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            w[q][r] = b[q][r] - w[q][r];
            if (ev[q]) {
                bb += (double)cnorm2(b[q][r]);
                rr += (double)cnorm2(w[q][r]);
            }
        }
        partial(make_double2(bb, rr), r);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RB; r++) {
        const double2 t = total(rbuf, r);
        norm_b[r] = sqrt(t.x);
        err[r] = sqrt(t.y);
        // a zero block right-hand side has the zero solution (the reference would divide by zero)
        fin[r] = !act[r] || norm_b[r] == 0.0;
        maxIt[r] = m;
    }
    rbuf ^= 1;
    for (int k = 0; k < p.restarts; k++) {
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
#pragma unroll
            for (int q = 0; q < EPT; q++)
                if (ev[q]) sm.basis[(size_t)r * NE + sidx(q)] = inv * w[q][r];
            if (threadIdx.x == 0) sm.gm[r * (m + 1)] = make_double2(err[r], 0.0);
        }
        for (int j = 0; j < m; j++) {
            anyarn = false;
#pragma unroll
            for (int r = 0; r < RB; r++) anyarn |= arn[r];
            if (!anyarn) break;
            __syncthreads();
            apply(sm.basis + (size_t)j * NE * RB);  // w = D_B V_j
            // classical Gram-Schmidt coefficients <w, V_i>, i <= j, and ||w||^2 (slot j + 1) in one
            // reduction: the warp sums of up to kGsBatch values share one interleaved butterfly, and the
            // CTA totals are formed once (a thread per value) instead of by every thread that needs them
            const int dbuf = rbuf;
#pragma unroll
            for (int r = 0; r < RB; r++) {
                if (!arn[r]) continue;
                for (int i0 = 0; i0 <= j + 1; i0 += kGsBatch) {
                    double2 sv[kGsBatch];
#pragma unroll
                    for (int g2 = 0; g2 < kGsBatch; g2++) {
                        sv[g2] = make_double2(0.0, 0.0);
                        if (i0 + g2 <= j) {
#pragma unroll
                            for (int q = 0; q < EPT; q++)
                                if (ev[q])
                                    sv[g2] = cfmac(to_d(sm.basis[((size_t)(i0 + g2) * RB + r) * NE + sidx(q)]),
                                                   to_d(w[q][r]), sv[g2]);
                        } else if (i0 + g2 == j + 1) {
#pragma unroll
                            for (int q = 0; q < EPT; q++)
                                if (ev[q]) sv[g2].x += (double)cnorm2(w[q][r]);
                        }
                    }
                    warp_sum_n<kGsBatch>(sv);
                    if (lane == 0)
#pragma unroll
                        for (int g2 = 0; g2 < kGsBatch; g2++)
                            if (i0 + g2 <= j + 1) sm.red[((size_t)rbuf * nw + wid) * SL + r * (kSapMaxM + 1) + i0 + g2] = sv[g2];
                }
            }
            __syncthreads();
            for (int t = threadIdx.x; t < RB * (j + 2); t += blockDim.x) {
                const int r = t / (j + 2), slot = r * (kSapMaxM + 1) + (t - r * (j + 2));
                sm.tot[slot] = total(dbuf, slot);
            }
            __syncthreads();
            rbuf ^= 1;
            // ||w - V h||^2 = ||w||^2 - sum |h_i|^2 for orthonormal V: no second reduction, unless the
            // difference cancels below 1e-4 of ||w||^2 (1e-2 for an FP32 basis, whose orthogonality holds
            // to ~1e-6); then the norm of the updated w is reduced as is
            constexpr double kCancel = sizeof(R) == 8 ? 1e-4 : 1e-2;
            double hn[RB];
            bool reduce_norm = false;
#pragma unroll
            for (int r = 0; r < RB; r++) {
                hn[r] = 0.0;
                if (!arn[r]) continue;
                const double w2 = sm.tot[r * (kSapMaxM + 1) + j + 1].x;
                double hh = 0.0;
                for (int i = 0; i <= j; i++) hh += cnorm2(sm.tot[r * (kSapMaxM + 1) + i]);
                const double d = w2 - hh;
                if (d > kCancel * w2) hn[r] = sqrt(d);
                else reduce_norm = true;  // identical in every thread: the totals are shared
            }
#pragma unroll
            for (int r = 0; r < RB; r++) {
                if (!arn[r]) continue;
                for (int i = 0; i <= j; i++) {
                    const V h = from_d<V>(sm.tot[r * (kSapMaxM + 1) + i]);
#pragma unroll
                    for (int q = 0; q < EPT; q++)
                        if (ev[q]) w[q][r] = w[q][r] - cmul(h, sm.basis[((size_t)i * RB + r) * NE + sidx(q)]);
                }
            }
            if (reduce_norm) {
                double2 wn[RB];
#pragma unroll
                for (int r = 0; r < RB; r++) {
                    double ww = 0.0;
                    if (arn[r])
#pragma unroll
                        for (int q = 0; q < EPT; q++)
                            if (ev[q]) ww += (double)cnorm2(w[q][r]);
                    wn[r] = make_double2(ww, 0.0);
                }
                warp_sum_n<RB>(wn);
                if (lane == 0)
#pragma unroll
                    for (int r = 0; r < RB; r++) sm.red[((size_t)rbuf * nw + wid) * SL + r] = wn[r];
                __syncthreads();
#pragma unroll
                for (int r = 0; r < RB; r++) hn[r] = sqrt(total(rbuf, r).x);
                rbuf ^= 1;
            }
#pragma unroll
            for (int r = 0; r < RB; r++) {
                if (arn[r] && hn[r] > 0) {
                    const R inv = R(1.0 / hn[r]);
#pragma unroll
                    for (int q = 0; q < EPT; q++)
                        if (ev[q]) sm.basis[((size_t)(j + 1) * RB + r) * NE + sidx(q)] = inv * w[q][r];
                }
            }
            if (threadIdx.x < RB && arn[threadIdx.x]) {  // thread r: Hessenberg column j of RHS r
                const int r = threadIdx.x;
                double2* H = sm.H + r * (m + 1) * m;
                double2* cn = sm.cn + r * m;
                double2* sn = sm.sn + r * m;
                double2* gm = sm.gm + r * (m + 1);
                for (int i = 0; i <= j; i++) H[i * m + j] = sm.tot[r * (kSapMaxM + 1) + i];
                H[(j + 1) * m + j] = make_double2(hn[r], 0.0);
                for (int i = 0; i < j; i++) {  // FGMRES::rotation (src/fgmres.cpp:99-115)
                    double2 hij = H[i * m + j], hi1 = H[(i + 1) * m + j];
                    double2 tmp = cmulc(cn[i], hij) + cmulc(sn[i], hi1);
                    H[(i + 1) * m + j] = cmul(cn[i], hi1) - cmul(sn[i], hij);
                    H[i * m + j] = tmp;
                }
                double2 hjj = H[j * m + j], hj1 = H[(j + 1) * m + j];
                double den = sqrt(cnorm2(hjj) + cnorm2(hj1));
                sn[j] = make_double2(hj1.x / den, hj1.y / den);
                cn[j] = make_double2(hjj.x / den, hjj.y / den);
                H[j * m + j] = cmulc(cn[j], hjj) + cmulc(sn[j], hj1);
                H[(j + 1) * m + j] = make_double2(0.0, 0.0);
                gm[j + 1] = -cmul(sn[j], gm[j]);
                gm[j] = cmulc(cn[j], gm[j]);
                sm.flag[r] = (sqrt(cnorm2(gm[j + 1])) < p.tol * norm_b[r]) ? 1 : 0;
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < RB; r++)
                if (arn[r] && sm.flag[r]) {
                    maxIt[r] = j + 1;  // not reset at the next restart (src/fgmres.cpp:14,56)
                    arn[r] = false;
                }
        }
        // solve_upper_triangular (src/fgmres.cpp:118-128), thread r for RHS r
        if (threadIdx.x < RB && !fin[threadIdx.x]) {
            const int r = threadIdx.x;
            const double2* H = sm.H + r * (m + 1) * m;
            double2* eta = sm.eta + r * m;
            for (int i = maxIt[r] - 1; i >= 0; i--) {
                double2 e = sm.gm[r * (m + 1) + i];
                for (int jj = i + 1; jj < maxIt[r]; jj++) e = e - cmul(H[i * m + jj], eta[jj]);
                eta[i] = cdiv(e, H[i * m + i]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RB; r++) {
            if (fin[r]) continue;
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                if (!ev[q]) continue;
                V a = x[q][r];
                for (int jj = 0; jj < maxIt[r]; jj++)
                    a = cfma(from_d<V>(sm.eta[r * m + jj]), sm.basis[((size_t)jj * RB + r) * NE + sidx(q)], a);
                x[q][r] = a;
            }
        }
        store_op(x);
        __syncthreads();
        apply(sm.op);
#pragma unroll
        for (int r = 0; r < RB; r++) {
            double rr = 0.0;
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                w[q][r] = b[q][r] - w[q][r];
                if (ev[q]) rr += (double)cnorm2(w[q][r]);
            }
            partial(make_double2(rr, 0.0), r);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RB; r++) {
            err[r] = sqrt(total(rbuf, r).x);
            if (!fin[r] && err[r] < p.tol * norm_b[r]) fin[r] = true;
        }
        rbuf ^= 1;
    }
    // x_B += e  (src/sap.cpp:106-113)
#pragma unroll
    for (int r = 0; r < RB; r++) {
        if (!act[r] || norm_b[r] == 0.0) continue;
#pragma unroll
        for (int q = 0; q < EPT; q++)
            if (ev[q]) {
                V* o = xg + (long)(r0 + r) * g.size() + (long)en[q] * dof + ei[q];
                *o = *o + x[q][r];
            }
    }
}

// ---------------------------------------------------------------- level 0: one warp per block
// The fine-level block solve is small (2 * sites unknowns), so a whole warp owns one Schwarz block:
// lane l owns sites l, l+32, ...; the block operator is the Wilson stencil restricted to the block
// (Level::SAP_level_l::D_local at level 0, src/level.cpp:607-653, with makeDirac's links), applied
// in spin-projected form from links held in registers; every reduction is a warp shuffle and the
// only synchronisation is __syncwarp.  Per-warp shared memory: Krylov basis, operand, Hessenberg.
template <typename V> struct WarpSmem {
    V* basis;      // (m+1) x S x 2
    V* op;         // S x 2
    double2* H;    // (m+1) x m
    double2* gm;   // m+1
    double2* cn;   // m
    double2* sn;   // m
    double2* eta;  // m
    __device__ WarpSmem(unsigned char* raw, int m, int S) {
        double2* d = reinterpret_cast<double2*>(raw);
        H = d;
        gm = H + (m + 1) * m;
        cn = gm + (m + 1);
        sn = cn + m;
        eta = sn + m;
        basis = reinterpret_cast<V*>(eta + m);
        op = basis + (size_t)(m + 1) * S * 2;
    }
    static size_t bytes(int m, int S) {
        return sizeof(double2) * ((size_t)(m + 1) * m + (m + 1) + 3 * m) + sizeof(V) * (size_t)(m + 2) * S * 2;
    }
};

template <typename V, int SPL>
__global__ void __launch_bounds__(128) sap_fine_warp_kernel(Geom g, const V* __restrict__ U, const V* __restrict__ rg,
                                                            V* __restrict__ xg, SapKParams p, int wpc, size_t wbytes) {
    typedef typename RealOf<V>::R R;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int task = blockIdx.x * wpc + wib;
    if (wib >= wpc || task >= p.nblocks * p.nrhs) return;
    const int kb = task / p.nrhs, rhs = task - kb * p.nrhs;  // block-major
    if (p.done && p.done[rhs]) return;
    const int et = g.sel_t, ex = g.sel_x, S = ex * et, m = p.m;
    WarpSmem<V> sm(smraw + wib * wbytes, m, S);
    const int blk = p.blocks[kb];
    const int bx = blk / g.sap_t, bt = blk - bx * g.sap_t;
    const long ro = (long)rhs * g.size();
    const R mm = R(p.m0) + R(2), half = R(0.5);

    bool sv[SPL];
    int sk[SPL], sn_[SPL];
    V u0[SPL], u1[SPL], ul0[SPL], ul1[SPL];
    V b[SPL][2], x[SPL][2], w[SPL][2];
#pragma unroll
    for (int q = 0; q < SPL; q++) {
        const int k = lane + 32 * q;
        sv[q] = k < S;
        const int kk = sv[q] ? k : 0;
        const int kx = kk / et, kt = kk - kx * et;
        const int xx = bx * ex + kx, tt = bt * et + kt;
        const int n = xx * g.Nt + tt;
        sk[q] = kk;
        sn_[q] = n;
        u0[q] = sv[q] ? __ldg(U + 2 * n) : czero<V>();
        u1[q] = sv[q] ? __ldg(U + 2 * n + 1) : czero<V>();
        ul0[q] = (sv[q] && kt > 0) ? conjc(__ldg(U + 2 * (n - 1))) : czero<V>();
        ul1[q] = (sv[q] && kx > 0) ? conjc(__ldg(U + 2 * (n - g.Nt) + 1)) : czero<V>();
#pragma unroll
        for (int a = 0; a < 2; a++) {
            b[q][a] = sv[q] ? rg[ro + (long)n * 2 + a] : czero<V>();
            x[q][a] = b[q][a];
        }
    }
    // w = D_B op  (op in per-warp shared memory, written and __syncwarp'ed by the caller)
    auto apply = [&](const V* op) {
#pragma unroll
        for (int q = 0; q < SPL; q++) {
            if (!sv[q]) {
                w[q][0] = w[q][1] = czero<V>();
                continue;
            }
            const int k = sk[q], kx = k / et, kt = k - kx * et;
            const V p0 = op[2 * k], p1 = op[2 * k + 1];
            V a = czero<V>(), c = czero<V>(), e = czero<V>(), gg = czero<V>();
            if (kt + 1 < et) a = cmul(u0[q], op[2 * (k + 1)] - op[2 * (k + 1) + 1]);          // +t: (1 - sigma_x)
            if (kx + 1 < ex) c = cmul(u1[q], op[2 * (k + et)] + imul(op[2 * (k + et) + 1]));  // +x: (1 - sigma_y)
            if (kt > 0) e = cmul(ul0[q], op[2 * (k - 1)] + op[2 * (k - 1) + 1]);              // -t: (1 + sigma_x)
            if (kx > 0) gg = cmul(ul1[q], op[2 * (k - et)] - imul(op[2 * (k - et) + 1]));      // -x: (1 + sigma_y)
            w[q][0] = mm * p0 - half * (a + c + e + gg);
            w[q][1] = mm * p1 - half * (imul(gg) - imul(c) + e - a);
        }
    };
    auto store = [&](V* dst, V (&v)[SPL][2]) {
#pragma unroll
        for (int q = 0; q < SPL; q++)
            if (sv[q]) {
                dst[2 * sk[q]] = v[q][0];
                dst[2 * sk[q] + 1] = v[q][1];
            }
    };
    auto dotw = [&](const V* vi) {  // sum_own w * conj(vi)
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < SPL; q++)
            if (sv[q])
#pragma unroll
                for (int a = 0; a < 2; a++) s = cfmac(to_d(vi[2 * sk[q] + a]), to_d(w[q][a]), s);
        return warp_sum(s);
    };
    auto nrm2 = [&](V (&v)[SPL][2]) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < SPL; q++)
            if (sv[q]) s += (double)cnorm2(v[q][0]) + (double)cnorm2(v[q][1]);
        return warp_sum(s);
    };

    store(sm.op, x);
    __syncwarp();
    apply(sm.op);
#pragma unroll
    for (int q = 0; q < SPL; q++)
#pragma unroll
        for (int a = 0; a < 2; a++) w[q][a] = b[q][a] - w[q][a];
    const double norm_b = sqrt(nrm2(b));
    double err = sqrt(nrm2(w));
    // a zero block right-hand side has the zero solution (the reference would divide by zero)
    if (norm_b == 0.0) return;
    int maxIt = m;
    for (int k = 0; k < p.restarts; k++) {
        const R inv = R(1.0 / err);
#pragma unroll
        for (int q = 0; q < SPL; q++)
#pragma unroll
            for (int a = 0; a < 2; a++) w[q][a] = inv * w[q][a];
        store(sm.basis, w);
        if (lane == 0) sm.gm[0] = make_double2(err, 0.0);
        __syncwarp();
        for (int j = 0; j < m; j++) {
            const V* vj = sm.basis + (size_t)j * S * 2;
            apply(vj);
            for (int i = 0; i <= j; i++) {  // modified Gram-Schmidt (src/fgmres.cpp:28-40)
                const V* vi = sm.basis + (size_t)i * S * 2;
                const double2 h = dotw(vi);
                if (lane == 0) sm.H[i * m + j] = h;
                const V hv = from_d<V>(h);
#pragma unroll
                for (int q = 0; q < SPL; q++)
                    if (sv[q])
#pragma unroll
                        for (int a = 0; a < 2; a++) w[q][a] = w[q][a] - cmul(hv, vi[2 * sk[q] + a]);
            }
            const double hn = sqrt(nrm2(w));
            if (hn > 0) {
                const R ih = R(1.0 / hn);
                V t[SPL][2];
#pragma unroll
                for (int q = 0; q < SPL; q++)
#pragma unroll
                    for (int a = 0; a < 2; a++) t[q][a] = ih * w[q][a];
                store(sm.basis + (size_t)(j + 1) * S * 2, t);
            }
            int brk = 0;
            if (lane == 0) {
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
                brk = (sqrt(cnorm2(sm.gm[j + 1])) < p.tol * norm_b) ? 1 : 0;
            }
            brk = __shfl_sync(0xffffffffu, brk, 0);
            __syncwarp();
            if (brk) {
                maxIt = j + 1;  // not reset at the next restart (src/fgmres.cpp:14,56)
                break;
            }
        }
        if (lane == 0) {  // solve_upper_triangular (src/fgmres.cpp:118-128)
            for (int i = maxIt - 1; i >= 0; i--) {
                double2 e = sm.gm[i];
                for (int jj = i + 1; jj < maxIt; jj++) e = e - cmul(sm.H[i * m + jj], sm.eta[jj]);
                sm.eta[i] = cdiv(e, sm.H[i * m + i]);
            }
        }
        __syncwarp();
        for (int jj = 0; jj < maxIt; jj++) {
            const V ej = from_d<V>(sm.eta[jj]);
            const V* vj = sm.basis + (size_t)jj * S * 2;
#pragma unroll
            for (int q = 0; q < SPL; q++)
                if (sv[q])
#pragma unroll
                    for (int a = 0; a < 2; a++) x[q][a] = cfma(ej, vj[2 * sk[q] + a], x[q][a]);
        }
        __syncwarp();
        store(sm.op, x);
        __syncwarp();
        apply(sm.op);
#pragma unroll
        for (int q = 0; q < SPL; q++)
#pragma unroll
            for (int a = 0; a < 2; a++) w[q][a] = b[q][a] - w[q][a];
        err = sqrt(nrm2(w));
        if (err < p.tol * norm_b) break;
    }
    // x_B += e  (src/sap.cpp:106-113)
#pragma unroll
    for (int q = 0; q < SPL; q++)
        if (sv[q])
#pragma unroll
            for (int a = 0; a < 2; a++) {
                V* o = xg + ro + (long)sn_[q] * 2 + a;
                *o = *o + x[q][a];
            }
}

// The same block solve with the Krylov basis in registers, for a restart length M fixed at compile
// time: every lane keeps its own elements of V_0..V_M, so the Gram-Schmidt dots and updates and the
// solution update touch no shared memory; only the stencil operand (whose neighbour values belong
// to other lanes) passes through the warp's shared buffer.  Gram-Schmidt is classical: the j+1
// dots of an Arnoldi step are reduced in one interleaved butterfly.  Dots and norms accumulate in
// the working precision.
template <typename V, int SPL, int M>
__global__ void __launch_bounds__(128, (sizeof(V) == 8 || SPL == 1) ? 4 : 1) sap_fine_reg_kernel(Geom g, const V* __restrict__ U, const V* __restrict__ rg,
                                                           V* __restrict__ xg, SapKParams p, int wpc, size_t wbytes) {
    typedef typename RealOf<V>::R R;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int task = blockIdx.x * wpc + wib;
    if (wib >= wpc || task >= p.nblocks * p.nrhs) return;
    const int kb = task / p.nrhs, rhs = task - kb * p.nrhs;  // block-major
    if (p.done && p.done[rhs]) return;
    const int et = g.sel_t, ex = g.sel_x, S = ex * et;
    // Hessenberg matrix, rotations and triangular solve in the working precision (lane 0 only)
    V* H = reinterpret_cast<V*>(smraw + wib * wbytes);  // (M+1) x M
    V* gm = H + (M + 1) * M;
    V* cn = gm + (M + 1);
    V* sn = cn + M;
    V* eta = sn + M;
    V* op = reinterpret_cast<V*>(eta + M);
    const int blk = p.blocks[kb];
    const int bx = blk / g.sap_t, bt = blk - bx * g.sap_t;
    const long ro = (long)rhs * g.size();
    const R mm = R(p.m0) + R(2), half = R(0.5);

    bool sv[SPL];
    int sk[SPL], sn_[SPL];
    V u0[SPL], u1[SPL], ul0[SPL], ul1[SPL];
    V b[SPL][2], x[SPL][2], w[SPL][2];
    V Vb[M + 1][SPL][2];
#pragma unroll
    for (int q = 0; q < SPL; q++) {
        const int k = lane + 32 * q;
        sv[q] = k < S;
        const int kk = sv[q] ? k : 0;
        const int kx = kk / et, kt = kk - kx * et;
        const int n = (bx * ex + kx) * g.Nt + bt * et + kt;
        sk[q] = kk;
        sn_[q] = n;
        u0[q] = sv[q] ? __ldg(U + 2 * n) : czero<V>();
        u1[q] = sv[q] ? __ldg(U + 2 * n + 1) : czero<V>();
        ul0[q] = (sv[q] && kt > 0) ? conjc(__ldg(U + 2 * (n - 1))) : czero<V>();
        ul1[q] = (sv[q] && kx > 0) ? conjc(__ldg(U + 2 * (n - g.Nt) + 1)) : czero<V>();
#pragma unroll
        for (int a = 0; a < 2; a++) {
            b[q][a] = sv[q] ? rg[ro + (long)n * 2 + a] : czero<V>();
            x[q][a] = b[q][a];
        }
    }
    // w = D_B v: v goes to the shared operand buffer, the stencil reads the neighbours from it
    auto apply = [&](const V (&v)[SPL][2]) {
        __syncwarp();
#pragma unroll
        for (int q = 0; q < SPL; q++)
            if (sv[q]) {
                op[2 * sk[q]] = v[q][0];
                op[2 * sk[q] + 1] = v[q][1];
            }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < SPL; q++) {
            if (!sv[q]) {
                w[q][0] = w[q][1] = czero<V>();
                continue;
            }
            const int k = sk[q], kx = k / et, kt = k - kx * et;
            V a = czero<V>(), c = czero<V>(), e = czero<V>(), gg = czero<V>();
            if (kt + 1 < et) a = cmul(u0[q], op[2 * (k + 1)] - op[2 * (k + 1) + 1]);          // +t: (1 - sigma_x)
            if (kx + 1 < ex) c = cmul(u1[q], op[2 * (k + et)] + imul(op[2 * (k + et) + 1]));  // +x: (1 - sigma_y)
            if (kt > 0) e = cmul(ul0[q], op[2 * (k - 1)] + op[2 * (k - 1) + 1]);              // -t: (1 + sigma_x)
            if (kx > 0) gg = cmul(ul1[q], op[2 * (k - et)] - imul(op[2 * (k - et) + 1]));      // -x: (1 + sigma_y)
            w[q][0] = mm * v[q][0] - half * (a + c + e + gg);
            w[q][1] = mm * v[q][1] - half * (imul(gg) - imul(c) + e - a);
        }
    };
    auto nrm2 = [&](const V (&v)[SPL][2]) {
        R s = R(0);
#pragma unroll
        for (int q = 0; q < SPL; q++)
            if (sv[q]) s += cnorm2(v[q][0]) + cnorm2(v[q][1]);
        return (double)warp_sum(s);
    };

    apply(x);
#pragma unroll
    for (int q = 0; q < SPL; q++)
#pragma unroll
        for (int a = 0; a < 2; a++) w[q][a] = b[q][a] - w[q][a];
    const double norm_b = sqrt(nrm2(b));
    double err = sqrt(nrm2(w));
    // a zero block right-hand side has the zero solution (the reference would divide by zero)
    if (norm_b == 0.0) return;
    int maxIt = M;
    for (int k = 0; k < p.restarts; k++) {
        const R inv = R(1.0 / err);
#pragma unroll
        for (int q = 0; q < SPL; q++)
#pragma unroll
            for (int a = 0; a < 2; a++) Vb[0][q][a] = inv * w[q][a];
        if (lane == 0) gm[0] = mkc(R(err), R(0));
#pragma unroll
        for (int j = 0; j < M; j++) {
            apply(Vb[j]);
            V h[M];
#pragma unroll
            for (int i = 0; i <= j; i++) {
                V t = czero<V>();
#pragma unroll
                for (int q = 0; q < SPL; q++)
                    if (sv[q])
#pragma unroll
                        for (int a = 0; a < 2; a++) t = cfmac(Vb[i][q][a], w[q][a], t);
                h[i] = t;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int i = 0; i <= j; i++) {
                    h[i].x += __shfl_xor_sync(0xffffffffu, h[i].x, o);
                    h[i].y += __shfl_xor_sync(0xffffffffu, h[i].y, o);
                }
#pragma unroll
            for (int i = 0; i <= j; i++)
#pragma unroll
                for (int q = 0; q < SPL; q++)
#pragma unroll
                    for (int a = 0; a < 2; a++) w[q][a] = w[q][a] - cmul(h[i], Vb[i][q][a]);
            const double hn = sqrt(nrm2(w));
            if (hn > 0) {
                const R ih = R(1.0 / hn);
#pragma unroll
                for (int q = 0; q < SPL; q++)
#pragma unroll
                    for (int a = 0; a < 2; a++) Vb[j + 1][q][a] = ih * w[q][a];
            }
            int brk = 0;
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i <= j; i++) H[i * M + j] = h[i];
                H[(j + 1) * M + j] = mkc(R(hn), R(0));
                for (int i = 0; i < j; i++) {  // FGMRES::rotation (src/fgmres.cpp:99-115)
                    const V hij = H[i * M + j], hi1 = H[(i + 1) * M + j];
                    const V tmp = cmulc(cn[i], hij) + cmulc(sn[i], hi1);
                    H[(i + 1) * M + j] = cmul(cn[i], hi1) - cmul(sn[i], hij);
                    H[i * M + j] = tmp;
                }
                const V hjj = H[j * M + j], hj1 = H[(j + 1) * M + j];
                const R den = sqrt(cnorm2(hjj) + cnorm2(hj1));
                sn[j] = mkc(hj1.x / den, hj1.y / den);
                cn[j] = mkc(hjj.x / den, hjj.y / den);
                H[j * M + j] = cmulc(cn[j], hjj) + cmulc(sn[j], hj1);
                H[(j + 1) * M + j] = czero<V>();
                gm[j + 1] = -cmul(sn[j], gm[j]);
                gm[j] = cmulc(cn[j], gm[j]);
                brk = (sqrt(cnorm2(gm[j + 1])) < p.tol * norm_b) ? 1 : 0;
            }
            brk = __shfl_sync(0xffffffffu, brk, 0);
            if (brk) {
                maxIt = j + 1;  // not reset at the next restart (src/fgmres.cpp:14,56)
                break;
            }
        }
        if (lane == 0) {  // solve_upper_triangular (src/fgmres.cpp:118-128)
            for (int i = maxIt - 1; i >= 0; i--) {
                V e = gm[i];
                for (int jj = i + 1; jj < maxIt; jj++) e = e - cmul(H[i * M + jj], eta[jj]);
                eta[i] = cdiv(e, H[i * M + i]);
            }
        }
        __syncwarp();
#pragma unroll
        for (int jj = 0; jj < M; jj++) {
            if (jj >= maxIt) break;
            const V ej = eta[jj];
#pragma unroll
            for (int q = 0; q < SPL; q++)
#pragma unroll
                for (int a = 0; a < 2; a++) x[q][a] = cfma(ej, Vb[jj][q][a], x[q][a]);
        }
        apply(x);
#pragma unroll
        for (int q = 0; q < SPL; q++)
#pragma unroll
            for (int a = 0; a < 2; a++) w[q][a] = b[q][a] - w[q][a];
        err = sqrt(nrm2(w));
        if (err < p.tol * norm_b) break;
    }
    // x_B += e  (src/sap.cpp:106-113)
#pragma unroll
    for (int q = 0; q < SPL; q++)
        if (sv[q])
#pragma unroll
            for (int a = 0; a < 2; a++) {
                V* o = xg + ro + (long)sn_[q] * 2 + a;
                *o = *o + x[q][a];
            }
}

// The register kernel for blocks of at most 16 sites with two (block, rhs) tasks per warp, one per
// half-warp, so that no lane idles (one task per warp would leave lanes 16-31 without a site).  The
// halves run the block GMRES in lockstep: each keeps its own Arnoldi / restart state, and the loops
// continue while either half is still working; a half that has finished computes values it never uses.
// Every reduction is a butterfly over the half (xor 8, 4, 2, 1).  In FP64 the Arnoldi control is trimmed
// for latency: ||w||^2 rides in the Gram-Schmidt butterfly and the new norm follows from
// ||w - V h||^2 = ||w||^2 - sum |h_i|^2 (w is reduced again only where that cancels), the norm and the
// Givens rotation use reciprocal square roots, the Hessenberg column is rotated in the lead lane's
// registers, and the restart's triangular solve multiplies by reciprocal diagonal entries formed with the
// rotation; the results agree with sap_fine_reg_kernel's to rounding.  FP32 blocks keep that kernel's
// control (FP32 half-warp sums, square roots and divisions): with the trimmed control the smoothed test
// vectors of a mixed-precision setup drifted from the FP64 ones (coarse operator 5.5e-3 apart instead of
// about 1e-4).
template <typename V, int M>
__global__ void __launch_bounds__(128, 4) sap_fine_pair_kernel(Geom g, const V* __restrict__ U, const V* __restrict__ rg,
                                                              V* __restrict__ xg, SapKParams p, size_t tbytes) {
    typedef typename RealOf<V>::R R;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, half = lane >> 4, l16 = lane & 15;
    const int task = (blockIdx.x * 4 + wib) * 2 + half;
    const int ntask = p.nblocks * p.nrhs;
    const int kb = task / p.nrhs, rhs = task - kb * p.nrhs;  // block-major
    const bool valid = task < ntask && !(p.done && p.done[rhs]);
    const int et = g.sel_t, ex = g.sel_x, S = ex * et;
    // per task: Hessenberg matrix, rotations and triangular solve (lane 0 of the half), stencil operand
    V* H = reinterpret_cast<V*>(smraw + (size_t)(wib * 2 + half) * tbytes);  // (M+1) x M
    V* gm = H + (M + 1) * M;
    V* cn = gm + (M + 1);
    V* sn = cn + M;
    V* eta = sn + M;
    V* op = eta + M;
    const int blk = valid ? p.blocks[kb] : 0;
    const int bx = blk / g.sap_t, bt = blk - bx * g.sap_t;
    const long ro = (long)(valid ? rhs : 0) * g.size();
    const R mm = R(p.m0) + R(2), half_ = R(0.5);
    const bool sv = valid && l16 < S;
    const int k = sv ? l16 : 0, kx = k / et, kt = k - kx * et;
    const int nsite = (bx * ex + kx) * g.Nt + bt * et + kt;
    const V u0 = sv ? __ldg(U + 2 * nsite) : czero<V>();
    const V u1 = sv ? __ldg(U + 2 * nsite + 1) : czero<V>();
    const V ul0 = (sv && kt > 0) ? conjc(__ldg(U + 2 * (nsite - 1))) : czero<V>();
    const V ul1 = (sv && kx > 0) ? conjc(__ldg(U + 2 * (nsite - g.Nt) + 1)) : czero<V>();
    V b[2], x[2], w[2];
    V Vb[M + 1][2];
#pragma unroll
    for (int a = 0; a < 2; a++) {
        b[a] = sv ? rg[ro + (long)nsite * 2 + a] : czero<V>();
        x[a] = b[a];
    }
    // w = D_B v through the half's operand buffer (the stencil reads the neighbours from it)
    auto apply = [&](const V (&v)[2]) {
        __syncwarp();
        if (sv) {
            op[2 * k] = v[0];
            op[2 * k + 1] = v[1];
        }
        __syncwarp();
        if (!sv) {
            w[0] = w[1] = czero<V>();
            return;
        }
        V a = czero<V>(), c = czero<V>(), e = czero<V>(), gg = czero<V>();
        if (kt + 1 < et) a = cmul(u0, op[2 * (k + 1)] - op[2 * (k + 1) + 1]);          // +t: (1 - sigma_x)
        if (kx + 1 < ex) c = cmul(u1, op[2 * (k + et)] + imul(op[2 * (k + et) + 1]));  // +x: (1 - sigma_y)
        if (kt > 0) e = cmul(ul0, op[2 * (k - 1)] + op[2 * (k - 1) + 1]);              // -t: (1 + sigma_x)
        if (kx > 0) gg = cmul(ul1, op[2 * (k - et)] - imul(op[2 * (k - et) + 1]));      // -x: (1 + sigma_y)
        w[0] = mm * v[0] - half_ * (a + c + e + gg);
        w[1] = mm * v[1] - half_ * (imul(gg) - imul(c) + e - a);
    };
    auto hsum = [](R s) {  // sum over the half-warp
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        return s;
    };
    auto nrm2 = [&](const V (&v)[2]) {
        const R s = sv ? cnorm2(v[0]) + cnorm2(v[1]) : R(0);
        return (double)hsum(s);
    };
    const int lead = lane & 16;  // the half's first lane
    V* const dinv = H + M * M;  // 1 / H[q][q] once column q is rotated (row M of H is not kept)
    // FP64: ||w - V h||^2 = ||w||^2 - sum |h_i|^2 for an orthonormal V, so ||w||^2 joins the Gram-Schmidt
    // butterfly and w is reduced again only where the difference cancels below this share of ||w||^2
    constexpr double kCancel = 1e-4;

    apply(x);
#pragma unroll
    for (int a = 0; a < 2; a++) w[a] = b[a] - w[a];
    const double norm_b = sqrt(nrm2(b));
    double err = sqrt(nrm2(w));
    // a zero block right-hand side has the zero solution (the reference would divide by zero)
    bool fin = !valid || norm_b == 0.0;
    int maxIt = M;
    if constexpr (sizeof(R) == 8) {
        const double thr = p.tol * norm_b, thr2 = thr * thr;
        for (int kr = 0; kr < p.restarts; kr++) {
            const bool act = !fin;
            if (!__any_sync(0xffffffffu, act)) break;
            bool arn = act;
            const R inv = R(act ? 1.0 / err : 0.0);
    #pragma unroll
            for (int a = 0; a < 2; a++) Vb[0][a] = inv * w[a];
            if (l16 == 0 && act) gm[0] = mkc(R(err), R(0));
    #pragma unroll
            for (int j = 0; j < M; j++) {
                if (!__any_sync(0xffffffffu, arn)) break;
                apply(Vb[j]);
                V h[M];
    #pragma unroll
                for (int i = 0; i <= j; i++) {
                    V t = czero<V>();
                    if (sv)
    #pragma unroll
                        for (int a = 0; a < 2; a++) t = cfmac(Vb[i][a], w[a], t);
                    h[i] = t;
                }
                R s2 = sv ? cnorm2(w[0]) + cnorm2(w[1]) : R(0);
    #pragma unroll
                for (int o = 8; o > 0; o >>= 1) {
    #pragma unroll
                    for (int i = 0; i <= j; i++) {
                        h[i].x += __shfl_xor_sync(0xffffffffu, h[i].x, o);
                        h[i].y += __shfl_xor_sync(0xffffffffu, h[i].y, o);
                    }
                    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                }
    #pragma unroll
                for (int i = 0; i <= j; i++)
    #pragma unroll
                    for (int a = 0; a < 2; a++) w[a] = w[a] - cmul(h[i], Vb[i][a]);
                double hh = 0.0;
    #pragma unroll
                for (int i = 0; i <= j; i++) hh += (double)cnorm2(h[i]);
                double hn2 = (double)s2 - hh;
                const bool redo = !(hn2 > kCancel * (double)s2);
                if (__any_sync(0xffffffffu, redo)) {  // warp-uniform: both halves take part in the butterfly
                    const double t = nrm2(w);
                    if (redo) hn2 = t;
                }
                double ih = 0.0, hn = 0.0;
                if (hn2 > 0.0) {
                    ih = rsqrt(hn2);
                    hn = hn2 * ih;
                }
                if (arn && hn > 0) {
    #pragma unroll
                    for (int a = 0; a < 2; a++) Vb[j + 1][a] = R(ih) * w[a];
                }
                int brk = 0;
                if (l16 == 0 && arn) {  // column j of the Hessenberg matrix, FGMRES::rotation (src/fgmres.cpp:99-115)
                    V hc[M + 1];
    #pragma unroll
                    for (int i = 0; i <= j; i++) hc[i] = h[i];
                    hc[j + 1] = mkc(R(hn), R(0));
    #pragma unroll
                    for (int i = 0; i < j; i++) {
                        const V ci = cn[i], si = sn[i];
                        const V tmp = cmulc(ci, hc[i]) + cmulc(si, hc[i + 1]);
                        hc[i + 1] = cmul(ci, hc[i + 1]) - cmul(si, hc[i]);
                        hc[i] = tmp;
                    }
                    const R iden = R(rsqrt((double)cnorm2(hc[j]) + (double)cnorm2(hc[j + 1])));
                    const V s_j = mkc(hc[j + 1].x * iden, hc[j + 1].y * iden);
                    const V c_j = mkc(hc[j].x * iden, hc[j].y * iden);
                    sn[j] = s_j;
                    cn[j] = c_j;
                    const V hd = cmulc(c_j, hc[j]) + cmulc(s_j, hc[j + 1]);
    #pragma unroll
                    for (int i = 0; i < j; i++) H[i * M + j] = hc[i];
                    const R id2 = R(1.0 / (double)cnorm2(hd));
                    dinv[j] = mkc(hd.x * id2, -hd.y * id2);
                    const V gj = gm[j], g1 = -cmul(s_j, gj);
                    gm[j + 1] = g1;
                    gm[j] = cmulc(c_j, gj);
                    brk = ((double)cnorm2(g1) < thr2) ? 1 : 0;
                }
                brk = __shfl_sync(0xffffffffu, brk, lead);
                if (arn && brk) {
                    maxIt = j + 1;  // not reset at the next restart (src/fgmres.cpp:14,56)
                    arn = false;
                }
            }
            if (l16 == 0 && act) {  // solve_upper_triangular (src/fgmres.cpp:118-128) with the reciprocal diagonal
                V et[M];
    #pragma unroll
                for (int q = M - 1; q >= 0; q--) {
                    et[q] = czero<V>();
                    if (q >= maxIt) continue;
                    V e = gm[q];
    #pragma unroll
                    for (int jj = q + 1; jj < M; jj++)
                        if (jj < maxIt) e = e - cmul(H[q * M + jj], et[jj]);
                    et[q] = cmul(e, dinv[q]);
                    eta[q] = et[q];
                }
            }
            __syncwarp();
            if (act) {
    #pragma unroll
                for (int jj = 0; jj < M; jj++) {
                    if (jj >= maxIt) break;
                    const V ej = eta[jj];
    #pragma unroll
                    for (int a = 0; a < 2; a++) x[a] = cfma(ej, Vb[jj][a], x[a]);
                }
            }
            apply(x);
    #pragma unroll
            for (int a = 0; a < 2; a++) w[a] = b[a] - w[a];
            const double e2 = sqrt(nrm2(w));
            if (act) {
                err = e2;
                if (err < p.tol * norm_b) fin = true;
            }
        }
    } else {  // FP32: the control of the reg kernel (FP32 sums, sqrt norms, divisions)
        for (int kr = 0; kr < p.restarts; kr++) {
            const bool act = !fin;
            if (!__any_sync(0xffffffffu, act)) break;
            bool arn = act;
            const R inv = R(act ? 1.0 / err : 0.0);
    #pragma unroll
            for (int a = 0; a < 2; a++) Vb[0][a] = inv * w[a];
            if (l16 == 0 && act) gm[0] = mkc(R(err), R(0));
    #pragma unroll
            for (int j = 0; j < M; j++) {
                if (!__any_sync(0xffffffffu, arn)) break;
                apply(Vb[j]);
                V h[M];
    #pragma unroll
                for (int i = 0; i <= j; i++) {
                    V t = czero<V>();
                    if (sv)
    #pragma unroll
                        for (int a = 0; a < 2; a++) t = cfmac(Vb[i][a], w[a], t);
                    h[i] = t;
                }
    #pragma unroll
                for (int o = 8; o > 0; o >>= 1)
    #pragma unroll
                    for (int i = 0; i <= j; i++) {
                        h[i].x += __shfl_xor_sync(0xffffffffu, h[i].x, o);
                        h[i].y += __shfl_xor_sync(0xffffffffu, h[i].y, o);
                    }
    #pragma unroll
                for (int i = 0; i <= j; i++)
    #pragma unroll
                    for (int a = 0; a < 2; a++) w[a] = w[a] - cmul(h[i], Vb[i][a]);
                const double hn = sqrt(nrm2(w));
                if (arn && hn > 0) {
                    const R ih = R(1.0 / hn);
    #pragma unroll
                    for (int a = 0; a < 2; a++) Vb[j + 1][a] = ih * w[a];
                }
                int brk = 0;
                if (l16 == 0 && arn) {
    #pragma unroll
                    for (int i = 0; i <= j; i++) H[i * M + j] = h[i];
                    H[(j + 1) * M + j] = mkc(R(hn), R(0));
                    for (int i = 0; i < j; i++) {  // FGMRES::rotation (src/fgmres.cpp:99-115)
                        const V hij = H[i * M + j], hi1 = H[(i + 1) * M + j];
                        const V tmp = cmulc(cn[i], hij) + cmulc(sn[i], hi1);
                        H[(i + 1) * M + j] = cmul(cn[i], hi1) - cmul(sn[i], hij);
                        H[i * M + j] = tmp;
                    }
                    const V hjj = H[j * M + j], hj1 = H[(j + 1) * M + j];
                    const R den = sqrt(cnorm2(hjj) + cnorm2(hj1));
                    sn[j] = mkc(hj1.x / den, hj1.y / den);
                    cn[j] = mkc(hjj.x / den, hjj.y / den);
                    H[j * M + j] = cmulc(cn[j], hjj) + cmulc(sn[j], hj1);
                    H[(j + 1) * M + j] = czero<V>();
                    gm[j + 1] = -cmul(sn[j], gm[j]);
                    gm[j] = cmulc(cn[j], gm[j]);
                    brk = (sqrt(cnorm2(gm[j + 1])) < p.tol * norm_b) ? 1 : 0;
                }
                brk = __shfl_sync(0xffffffffu, brk, lead);
                if (arn && brk) {
                    maxIt = j + 1;  // not reset at the next restart (src/fgmres.cpp:14,56)
                    arn = false;
                }
            }
            if (l16 == 0 && act) {  // solve_upper_triangular (src/fgmres.cpp:118-128)
                for (int i = maxIt - 1; i >= 0; i--) {
                    V e = gm[i];
                    for (int jj = i + 1; jj < maxIt; jj++) e = e - cmul(H[i * M + jj], eta[jj]);
                    eta[i] = cdiv(e, H[i * M + i]);
                }
            }
            __syncwarp();
            if (act) {
    #pragma unroll
                for (int jj = 0; jj < M; jj++) {
                    if (jj >= maxIt) break;
                    const V ej = eta[jj];
    #pragma unroll
                    for (int a = 0; a < 2; a++) x[a] = cfma(ej, Vb[jj][a], x[a]);
                }
            }
            apply(x);
    #pragma unroll
            for (int a = 0; a < 2; a++) w[a] = b[a] - w[a];
            const double e2 = sqrt(nrm2(w));
            if (act) {
                err = e2;
                if (err < p.tol * norm_b) fin = true;
            }
        }
    }
    // x_B += e  (src/sap.cpp:106-113)
    if (sv && norm_b != 0.0)
#pragma unroll
        for (int a = 0; a < 2; a++) {
            V* o = xg + ro + (long)nsite * 2 + a;
            *o = *o + x[a];
        }
}

template <typename V, int M>
static void launch_fine_pair(cudaStream_t s, const Geom& g, const V* U, const V* r, V* x, SapKParams p) {
    const int S = g.sel_x * g.sel_t;
    const size_t tb = (sizeof(V) * ((M + 1) * M + (M + 1) + 3 * M) + sizeof(V) * 2 * S + 15) / 16 * 16;
    const int tasks = p.nblocks * p.nrhs;
    DDAMG_LAUNCH((sap_fine_pair_kernel<V, M>), ceil_div(tasks, 8), 128, tb * 8, s, g, U, r, x, p, tb);
}

template <typename V, int SPL, int M>
static void launch_fine_reg(cudaStream_t s, const Geom& g, const V* U, const V* r, V* x, SapKParams p) {
    const int S = g.sel_x * g.sel_t;
    const size_t wb = (sizeof(V) * ((M + 1) * M + (M + 1) + 3 * M) + sizeof(V) * 2 * S + 15) / 16 * 16;
    const int wpc = 4;
    const int tasks = p.nblocks * p.nrhs;
    DDAMG_LAUNCH((sap_fine_reg_kernel<V, SPL, M>), ceil_div(tasks, wpc), 32 * wpc, wb * wpc, s, g, U, r, x, p, wpc,
                 wb);
}

template <typename V, int SPL>
static void launch_fine_warp(cudaStream_t s, const Geom& g, const V* U, const V* r, V* x, SapKParams p) {
    const int S = g.sel_x * g.sel_t;
    const size_t wb = (WarpSmem<V>::bytes(p.m, S) + 15) / 16 * 16;
    const int wpc = (int)std::max<size_t>(1, std::min<size_t>(4, (48 * 1024) / wb));
    const size_t smem = wb * wpc;
    const int tasks = p.nblocks * p.nrhs;
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(sap_fine_warp_kernel<V, SPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    DDAMG_LAUNCH((sap_fine_warp_kernel<V, SPL>), ceil_div(tasks, wpc), 32 * wpc, smem, s, g, U, r, x, p, wpc, wb);
}

template <typename V, bool DENSE, int EPT, int MAXT, int RB, int CH = 8>
static void launch_sap_k(cudaStream_t s, int threads, const Geom& g, const V* L, const V* r, V* x, SapKParams p) {
    const int NE = g.sel_x * g.sel_t * g.dof;
    p.ngroups = (p.nrhs + RB - 1) / RB;
    const size_t smem = SapSmem<V, RB>::bytes(p.m, NE, threads / 32);
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(sap_block_kernel<V, DENSE, EPT, MAXT, RB, CH>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DDAMG_LAUNCH((sap_block_kernel<V, DENSE, EPT, MAXT, RB, CH>), dim3(p.nblocks * p.ngroups), threads, smem,
                 s, g, L, r, x, p);
}

// right-hand sides per CTA: as many as fit in shared memory (and in registers for small
// element counts), preferring a count that divides nrhs
static int pick_rb(int nrhs, int ept, int m, int NE, int threads, size_t vbytes) {
    auto fits = [&](int rb) {
        const size_t smem = sizeof(double2) * ((size_t)2 * (threads / 32) * rb * (kSapMaxM + 1) +
                                               (size_t)rb * ((m + 1) * m + (m + 1) + 3 * m + kSapMaxM + 1)) +
                            16 + vbytes * (size_t)(m + 2) * NE * rb;
        return smem <= 227 * 1024 && ept * rb * (int)(vbytes / 8) <= 8;  // register budget
    };
    if (nrhs <= 1) return 1;
    int best = 1;
    for (int rb : {8, 4, 2}) {
        if (rb > nrhs || !fits(rb)) continue;
        if (nrhs % rb == 0) return rb;
        if (best == 1) best = rb;
    }
    return best;
}

// right-hand sides per CTA the launcher below supports for a block of NE unknowns
static bool rb_admissible(int rb, int nrhs, int m, int NE, size_t vbytes) {
    const int threads = std::min(1024, ((NE + 31) / 32) * 32);
    const int ept = (NE + threads - 1) / threads;
    if (rb == 1) return true;
    if (rb > nrhs || ept != 1 || (threads > 512 && rb > 2)) return false;
    const size_t smem = sizeof(double2) * ((size_t)2 * (threads / 32) * rb * (kSapMaxM + 1) +
                                           (size_t)rb * ((m + 1) * m + (m + 1) + 3 * m + kSapMaxM + 1)) +
                        16 + vbytes * (size_t)(m + 2) * NE * rb;
    return smem <= 227 * 1024 && rb * (int)(vbytes / 8) <= 8;  // shared memory and register budget
}

// A coarse sweep variant is rb * 4 + kernel: rb right-hand sides per CTA and kernel 0 = sap_block_kernel,
// 1 = sap_block2_kernel; variant 0 lets the launcher choose.
static bool variant_admissible(int variant, int nrhs, int m, int NE, size_t vbytes) {
    const int rb = variant / 4, kern = variant % 4;
    if (rb < 1 || kern > 1 || !rb_admissible(rb, nrhs, m, NE, vbytes)) return false;
    return kern == 0 || sap2_fits(rb, m, NE, vbytes);
}

template <typename V, bool DENSE>
static void launch_sap(cudaStream_t s, const Geom& g, const V* L, const V* r, V* x, const SapArgs& a, int nrhs,
                       int variant = 0) {
    if (a.m > kSapMaxM) throw ParamFailure{"SAP block GMRES restart length above 8 is not supported"};
    const int NE = g.sel_x * g.sel_t * g.dof;
    const int threads = std::min(1024, ((NE + 31) / 32) * 32);
    const int ept = (NE + threads - 1) / threads;
    SapKParams p{a.m, a.restarts, a.tol, a.m0, a.blocks, a.nblocks, a.done, nrhs, 1};
    p.vres = a.vres;
    // level 0 keeps one vector per CTA: its links are 32 B per site, so there is nothing to share,
    // and a wider CTA would only cost shared memory and occupancy
    int rb = DENSE ? pick_rb(nrhs, ept, a.m, NE, threads, sizeof(V)) : 1, kern = 0;
    if (DENSE && variant > 0 && variant_admissible(variant, nrhs, a.m, NE, sizeof(V))) {
        rb = variant / 4;
        kern = variant % 4;
    }
    if (a.vres && !(DENSE && kern == 1))
        throw ParamFailure{"internal: a fused-residual sweep needs the sap_block2_kernel variant"};
    if (DENSE && kern == 1) {
        if (rb == 4) launch_sap2<V, 4>(s, g, L, r, x, p);
        else if (rb == 2) launch_sap2<V, 2>(s, g, L, r, x, p);
        else launch_sap2<V, 1>(s, g, L, r, x, p);
        return;
    }
    // blocks of at most 384 unknowns: a 384-thread bound leaves 168 registers per thread, enough to
    // keep 12 link loads in flight per right-hand side group
    if (DENSE && ept == 1 && threads <= 384 && (rb == 1 || rb == 4)) {
        if (rb == 4) launch_sap_k<V, DENSE, 1, 384, 4, 12>(s, threads, g, L, r, x, p);
        else launch_sap_k<V, DENSE, 1, 384, 1, 12>(s, threads, g, L, r, x, p);
        return;
    }
    if (ept == 1 && threads <= 512) {
        if (rb == 8) launch_sap_k<V, DENSE, 1, 512, 8>(s, threads, g, L, r, x, p);
        else if (rb == 4) launch_sap_k<V, DENSE, 1, 512, 4>(s, threads, g, L, r, x, p);
        else if (rb == 2) launch_sap_k<V, DENSE, 1, 512, 2>(s, threads, g, L, r, x, p);
        else launch_sap_k<V, DENSE, 1, 512, 1>(s, threads, g, L, r, x, p);
    } else if (ept == 1) {
        if (rb >= 2) launch_sap_k<V, DENSE, 1, 1024, 2>(s, threads, g, L, r, x, p);
        else launch_sap_k<V, DENSE, 1, 1024, 1>(s, threads, g, L, r, x, p);
    } else if (ept == 2) {
        launch_sap_k<V, DENSE, 2, 1024, 1>(s, threads, g, L, r, x, p);
    } else if (ept <= 4) {
        launch_sap_k<V, DENSE, 4, 1024, 1>(s, threads, g, L, r, x, p);
    } else {
        throw ParamFailure{"SAP block too large (more than 4096 unknowns per block)"};
    }
}
size_t sap_smem_bytes(int m, int NE, bool fp64) {
    const int nw = std::min(32, (NE + 31) / 32);
    return fp64 ? SapSmem<double2, 1>::bytes(m, NE, nw) : SapSmem<float2, 1>::bytes(m, NE, nw);
}

template <typename V>
void launch_sap_sweep_fine(cudaStream_t s, const Geom& g, const V* U, const V* r, V* x, const SapArgs& a, int nrhs) {
    const int S = g.sel_x * g.sel_t;
    if (a.m > kSapMaxM) throw ParamFailure{"SAP block GMRES restart length above 8 is not supported"};
    if (a.vres) throw ParamFailure{"internal: the level-0 sweeps read the residual"};
    SapKParams p{a.m, a.restarts, a.tol, a.m0, a.blocks, a.nblocks, a.done, nrhs, 1};
    if (a.m == 5 && S <= 16) launch_fine_pair<V, 5>(s, g, U, r, x, p);
    else if (a.m == 5 && S <= 32) launch_fine_reg<V, 1, 5>(s, g, U, r, x, p);
    else if (a.m == 5 && S <= 64) launch_fine_reg<V, 2, 5>(s, g, U, r, x, p);
    else if (S <= 32) launch_fine_warp<V, 1>(s, g, U, r, x, p);
    else if (S <= 64) launch_fine_warp<V, 2>(s, g, U, r, x, p);
    else if (S <= 128) launch_fine_warp<V, 4>(s, g, U, r, x, p);
    else if (S <= 256) launch_fine_warp<V, 8>(s, g, U, r, x, p);
    else launch_sap<V, false>(s, g, U, r, x, a, nrhs);
}
template <typename V>
void launch_sap_sweep_coarse(cudaStream_t s, const Geom& g, const V* links, const V* r, V* x, const SapArgs& a,
                             int nrhs, int variant) {
    launch_sap<V, true>(s, g, links, r, x, a, nrhs, variant);
}

// Autotuner for the CUDA-core coarse sweep: times one sweep per admissible variant (rb 1, 2, 4, 8
// right-hand sides per CTA, each with the kernels that take it), accumulating into the scratch field xs
// (its contents do not matter), and returns the fastest variant; us[i] gets the time of
// kSapVariants[i] (negative: not admissible).  Synchronises.
template <typename V>
int tune_sap_rb(cudaStream_t s, const Geom& g, const V* links, const V* r, V* xs, const SapArgs& a, int nrhs,
                double* us) {
    const int NE = g.sel_x * g.sel_t * g.dof;
    cudaEvent_t e0, e1;
    DDAMG_CUDA_TRY(cudaEventCreate(&e0));
    DDAMG_CUDA_TRY(cudaEventCreate(&e1));
    int best = 0;
    double best_us = -1;
    // where sap_block2_kernel takes the shape, only its variants compete: they give bit-identical results
    // for every right-hand side whatever their width, so two handles agree whichever one the timing picks
    bool new_ok = false;
    for (int i = 0; i < kSapVariantCount; i++)
        new_ok |= kSapVariants[i] % 4 == 1 && variant_admissible(kSapVariants[i], nrhs, a.m, NE, sizeof(V));
    for (int i = 0; i < kSapVariantCount; i++) {
        us[i] = -1;
        const int v = kSapVariants[i];
        if (!variant_admissible(v, nrhs, a.m, NE, sizeof(V)) || (new_ok && v % 4 == 0)) continue;
        launch_sap<V, true>(s, g, links, r, xs, a, nrhs, v);  // warm-up
        DDAMG_CUDA_TRY(cudaEventRecord(e0, s));
        launch_sap<V, true>(s, g, links, r, xs, a, nrhs, v);
        DDAMG_CUDA_TRY(cudaEventRecord(e1, s));
        DDAMG_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        us[i] = 1e3 * ms;
        if (best_us < 0 || us[i] < best_us) {
            best_us = us[i];
            best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best > 0 ? best : 4;
}
template int tune_sap_rb<double2>(cudaStream_t, const Geom&, const double2*, const double2*, double2*,
                                  const SapArgs&, int, double*);
template int tune_sap_rb<float2>(cudaStream_t, const Geom&, const float2*, const float2*, float2*, const SapArgs&,
                                 int, double*);
template void launch_sap_sweep_fine<double2>(cudaStream_t, const Geom&, const double2*, const double2*, double2*,
                                             const SapArgs&, int);
template void launch_sap_sweep_fine<float2>(cudaStream_t, const Geom&, const float2*, const float2*, float2*,
                                            const SapArgs&, int);
template void launch_sap_sweep_coarse<double2>(cudaStream_t, const Geom&, const double2*, const double2*, double2*,
                                               const SapArgs&, int, int);
template void launch_sap_sweep_coarse<float2>(cudaStream_t, const Geom&, const float2*, const float2*, float2*,
                                              const SapArgs&, int, int);

}  // namespace ddamg
