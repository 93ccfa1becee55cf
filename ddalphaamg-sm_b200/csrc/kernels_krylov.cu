// Comparison solvers of the reference (src/conjugate_gradient.cpp): BiCGstab on D_W (bi_cgstab,
// :87-176) and CG on the normal equations D^dagger D x = phi (conjugate_gradient, :4-83), FP64
// on the fine lattice.
//
// Every scalar of the iteration (alpha, beta, omega, rho, the residual norm) lives in device
// memory.  Each kernel is one fused pass over the lattice, one thread per site: it forms its
// operand on the fly at the five stencil sites (e.g. BiCGstab's new search direction
// d = r + beta (d_old - omega A d_old) is never stored before D is applied to it), applies D or
// D^dagger, does the vector updates of the site and leaves per-CTA partial sums.  The last CTA to
// finish (a ticket counter) adds the partials in a fixed order and advances the scalars, so the
// sums are deterministic and no kernel waits on another CTA.  A device word ends the iteration:
// kernels launched after convergence return at once, so the host enqueues iterations in batches
// (or replays a captured batch) and reads the word once per batch.
#include "internal.h"

namespace ddamg {

// BiCGstab reads its direction pair (d, A d) of the previous iteration from set (k-1)&1 and
// writes the new pair to set k&1; CG keeps its direction the same way.
struct KrylovVecs {
    const double2* U;
    const double2* b;  // right-hand side (BiCGstab: b, CG: phi)
    double2* rt;       // BiCGstab shadow residual r~ = r_0
    double2 *x, *r, *s, *t, *y;
    double2* d[2];
    double2* Ad[2];
    double2* part;     // per-CTA partial sums, 3 per CTA
    KrylovState* st;
    int Nx, Nt;
    double m0, tol;
    int max_iter;
};

// D_phi / D_dagger_phi (src/dirac_operator.cpp:24-85) at site n, the operand given by fld(site, a, b)
template <bool DAG, class F>
__device__ __forceinline__ void wilson_at(const double2* __restrict__ U, int Nx, int Nt, double m0, int n, F fld,
                                          double2& o0, double2& o1) {
    const int x = n / Nt, t = n - x * Nt;
    const int tp = (t + 1 == Nt) ? 0 : t + 1, tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1, xm = (x == 0) ? Nx - 1 : x - 1;
    const int r0 = x * Nt + tp, l0 = x * Nt + tm, r1 = xp * Nt + t, l1 = xm * Nt + t;
    const double sr = (t == Nt - 1) ? -1.0 : 1.0, sl = (t == 0) ? -1.0 : 1.0;
    double2 u0, u1;
    ld2w(U + 2 * n, u0, u1);
    const double2 ul0 = __ldg(U + 2 * l0), ul1 = __ldg(U + 2 * l1 + 1);
    double2 p0, p1, a0, a1, c0, c1, e0, e1, g0, g1;
    fld(n, p0, p1);
    fld(r0, a0, a1);
    fld(r1, c0, c1);
    fld(l0, e0, e1);
    fld(l1, g0, g1);
    double2 s0, s1;
    if (!DAG) {
        const double2 a = sr * cmul(u0, a0 - a1);     // +t: (1 - sigma_x)
        const double2 c = cmul(u1, c0 + imul(c1));   // +x: (1 - sigma_y)
        const double2 e = sl * cmulc(ul0, e0 + e1);  // -t: (1 + sigma_x)
        const double2 g = cmulc(ul1, g0 - imul(g1)); // -x: (1 + sigma_y)
        s0 = a + c + e + g;
        s1 = -a - imul(c) + e + imul(g);
    } else {
        const double2 a = sl * cmulc(ul0, e0 - e1);  // -t: (1 - sigma_x)
        const double2 c = cmulc(ul1, g0 + imul(g1)); // -x: (1 - sigma_y)
        const double2 e = sr * cmul(u0, a0 + a1);    // +t: (1 + sigma_x)
        const double2 g = cmul(u1, c0 - imul(c1));   // +x: (1 + sigma_y)
        s0 = a + c + e + g;
        s1 = -a - imul(c) + e + imul(g);
    }
    o0 = (m0 + 2.0) * p0 - 0.5 * s0;
    o1 = (m0 + 2.0) * p1 - 0.5 * s1;
}

// Leaves the CTA's NQ partial sums in part and returns true in the last CTA to finish, after
// it has added every CTA's partials (fixed order: lanes stride over the CTAs, then a shuffle
// tree) into tot[0..NQ).  Every thread of the CTA must call it.
template <int NQ>
__device__ bool reduce_last(const double2 (&v)[NQ], double2* __restrict__ part, unsigned* ticket, double2* tot) {
    __shared__ double2 scratch[33];
    __shared__ bool last;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        const double2 sum = block_sum(v[q], scratch);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * 3 + q] = sum;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // thread i adds the partials of CTAs i, i + blockDim, ... (a fixed assignment), then a CTA tree
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        double2 s = make_double2(0.0, 0.0);
        for (int bk = threadIdx.x; bk < (int)gridDim.x; bk += blockDim.x) s += __ldcg(part + (size_t)bk * 3 + q);
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) tot[q] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0;
    return true;
}

// ---------------------------------------------------------------- BiCGstab
// r = b - D x0, r~ = r; ||b|| and rho = (r, r~)
__global__ void __launch_bounds__(256) bicg_init_kernel(KrylovVecs k) {
    const int sites = k.Nx * k.Nt;
    double2 q[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 o0, o1;
        wilson_at<false>(k.U, k.Nx, k.Nt, k.m0, n,
                         [&](int m, double2& a, double2& c) { a = k.x[2 * m]; c = k.x[2 * m + 1]; }, o0, o1);
        const double2 b0 = k.b[2 * n], b1 = k.b[2 * n + 1];
        const double2 r0 = b0 - o0, r1 = b1 - o1;
        k.r[2 * n] = r0;
        k.r[2 * n + 1] = r1;
        k.rt[2 * n] = r0;
        k.rt[2 * n + 1] = r1;
        q[0] = cfmac(b0, b0, cfmac(b1, b1, q[0]));
        q[1] = cfmac(r0, r0, cfmac(r1, r1, q[1]));
    }
    __shared__ double2 tot[2];
    if (reduce_last<2>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) {
        k.st->norm_b = sqrt(tot[0].x);
        k.st->rho = tot[1];
        k.st->k = 0;
        k.st->done = 0;
        k.st->iters = 0;
    }
}

// d_k = r + beta (d_{k-1} - omega A d_{k-1}) (d_0 = r), A d_k; alpha = rho / (A d_k, r~)
__global__ void __launch_bounds__(256) bicg_dir_kernel(KrylovVecs k) {
    const KrylovState* st = k.st;
    if (st->done) return;
    const int it = st->k;
    const int sites = k.Nx * k.Nt;
    const double2* dp = k.d[(it + 1) & 1];
    const double2* Adp = k.Ad[(it + 1) & 1];
    double2* dn = k.d[it & 1];
    double2* Adn = k.Ad[it & 1];
    const double2 omega = st->omega;
    const double2 beta = it ? cdiv(cmul(st->alpha, st->rho), cmul(omega, st->rho_prev)) : make_double2(0.0, 0.0);
    auto dir = [&](int m, double2& a, double2& c) {
        ld2w(k.r + 2 * m, a, c);
        if (it) {
            double2 d0, d1, A0, A1;
            ld2w(dp + 2 * m, d0, d1);
            ld2w(Adp + 2 * m, A0, A1);
            a = a + cmul(beta, d0 - cmul(omega, A0));
            c = c + cmul(beta, d1 - cmul(omega, A1));
        }
    };
    double2 q[1] = {make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 o0, o1, d0, d1;
        wilson_at<false>(k.U, k.Nx, k.Nt, k.m0, n, dir, o0, o1);
        dir(n, d0, d1);
        st2w(dn + 2 * n, d0, d1);
        st2w(Adn + 2 * n, o0, o1);
        double2 t0, t1;
        ld2w(k.rt + 2 * n, t0, t1);
        q[0] = cfmac(t0, o0, cfmac(t1, o1, q[0]));  // sum A d conj(r~)
    }
    __shared__ double2 tot[1];
    if (reduce_last<1>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) k.st->alpha = cdiv(st->rho, tot[0]);
}

// s = r - alpha A d, t = D s; ||s|| (convergence test), omega = (s, t) / (t, t)
__global__ void __launch_bounds__(256) bicg_s_kernel(KrylovVecs k) {
    const KrylovState* st = k.st;
    if (st->done) return;
    const int it = st->k;
    const int sites = k.Nx * k.Nt;
    const double2* Ad = k.Ad[it & 1];
    const double2 alpha = st->alpha;
    auto sv = [&](int m, double2& a, double2& c) {
        double2 r0, r1, A0, A1;
        ld2w(k.r + 2 * m, r0, r1);
        ld2w(Ad + 2 * m, A0, A1);
        a = r0 - cmul(alpha, A0);
        c = r1 - cmul(alpha, A1);
    };
    double2 q[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 t0, t1, s0, s1;
        wilson_at<false>(k.U, k.Nx, k.Nt, k.m0, n, sv, t0, t1);
        sv(n, s0, s1);
        st2w(k.s + 2 * n, s0, s1);
        st2w(k.t + 2 * n, t0, t1);
        q[0] = cfmac(t0, s0, cfmac(t1, s1, q[0]));  // sum s conj(t)
        q[1] = cfmac(t0, t0, cfmac(t1, t1, q[1]));
        q[2] = cfmac(s0, s0, cfmac(s1, s1, q[2]));
    }
    __shared__ double2 tot[3];
    if (reduce_last<3>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) {
        KrylovState* w = k.st;
        w->err = sqrt(tot[2].x);
        if (w->err < k.tol * w->norm_b) {
            w->done = 1;  // x += alpha d still to do
            w->iters = it + 1;
        } else {
            w->omega = cdiv(tot[0], tot[1]);
        }
    }
}

// r = s - omega t, x = x + alpha d + omega s, rho = (r, r~); at convergence only x += alpha d
__global__ void __launch_bounds__(256) bicg_update_kernel(KrylovVecs k) {
    const KrylovState* st = k.st;
    const int done = st->done;
    if (done > 1) return;
    const int it = st->k;
    const int sites = k.Nx * k.Nt;
    const double2* d = k.d[it & 1];
    const double2 alpha = st->alpha, omega = st->omega;
    double2 q[1] = {make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 x0, x1, d0, d1;
        ld2wc(k.x + 2 * n, x0, x1);
        ld2w(d + 2 * n, d0, d1);
        if (done == 1) {
            st2w(k.x + 2 * n, x0 + cmul(alpha, d0), x1 + cmul(alpha, d1));
        } else {
            double2 s0, s1, t0, t1, q0, q1;
            ld2w(k.s + 2 * n, s0, s1);
            ld2w(k.t + 2 * n, t0, t1);
            ld2w(k.rt + 2 * n, q0, q1);
            const double2 r0 = s0 - cmul(omega, t0), r1 = s1 - cmul(omega, t1);
            st2w(k.r + 2 * n, r0, r1);
            st2w(k.x + 2 * n, (x0 + cmul(alpha, d0)) + cmul(omega, s0), (x1 + cmul(alpha, d1)) + cmul(omega, s1));
            q[0] = cfmac(q0, r0, cfmac(q1, r1, q[0]));
        }
    }
    __shared__ double2 tot[1];
    if (reduce_last<1>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) {
        KrylovState* w = k.st;
        if (done == 1) {
            w->done = 2;
        } else {
            w->rho_prev = w->rho;
            w->rho = tot[0];
            w->k = it + 1;
            if (it + 1 >= k.max_iter) {
                w->done = 3;
                w->iters = k.max_iter;
            }
        }
    }
}

// ---------------------------------------------------------------- CG on D^dagger D
// x = phi, y = D x
__global__ void __launch_bounds__(256) cg_init_a_kernel(KrylovVecs k) {
    const int sites = k.Nx * k.Nt;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 o0, o1;
        wilson_at<false>(k.U, k.Nx, k.Nt, k.m0, n,
                         [&](int m, double2& a, double2& c) { a = k.b[2 * m]; c = k.b[2 * m + 1]; }, o0, o1);
        k.x[2 * n] = k.b[2 * n];
        k.x[2 * n + 1] = k.b[2 * n + 1];
        k.y[2 * n] = o0;
        k.y[2 * n + 1] = o1;
    }
}
// r = phi - D^dagger y, d_0 = r; (r, r) and ||phi||
__global__ void __launch_bounds__(256) cg_init_b_kernel(KrylovVecs k) {
    const int sites = k.Nx * k.Nt;
    double2 q[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 o0, o1;
        wilson_at<true>(k.U, k.Nx, k.Nt, k.m0, n, [&](int m, double2& a, double2& c) { ld2w(k.y + 2 * m, a, c); },
                        o0, o1);
        const double2 p0 = k.b[2 * n], p1 = k.b[2 * n + 1];
        const double2 r0 = p0 - o0, r1 = p1 - o1;
        k.r[2 * n] = r0;
        k.r[2 * n + 1] = r1;
        k.d[0][2 * n] = r0;
        k.d[0][2 * n + 1] = r1;
        q[0] = cfmac(r0, r0, cfmac(r1, r1, q[0]));
        q[1] = cfmac(p0, p0, cfmac(p1, p1, q[1]));
    }
    __shared__ double2 tot[2];
    if (reduce_last<2>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) {
        k.st->rnorm2 = tot[0];
        k.st->norm_b = sqrt(tot[1].x);
        k.st->k = 0;
        k.st->done = 0;
        k.st->iters = 0;
    }
}
// d_k = d_{k-1} beta + r (d_0 already stored), y = D d_k
__global__ void __launch_bounds__(256) cg_y_kernel(KrylovVecs k) {
    const KrylovState* st = k.st;
    if (st->done) return;
    const int it = st->k;
    const int sites = k.Nx * k.Nt;
    const double2* dp = k.d[(it + 1) & 1];
    double2* dn = k.d[it & 1];
    const double2 beta = st->beta;
    auto dir = [&](int m, double2& a, double2& c) {
        double2 d0, d1, r0, r1;
        ld2w(dp + 2 * m, d0, d1);
        ld2w(k.r + 2 * m, r0, r1);
        a = cmul(d0, beta) + r0;
        c = cmul(d1, beta) + r1;
    };
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 o0, o1;
        if (it == 0) {
            wilson_at<false>(k.U, k.Nx, k.Nt, k.m0, n,
                             [&](int m, double2& a, double2& c) { ld2w(dn + 2 * m, a, c); }, o0, o1);
        } else {
            wilson_at<false>(k.U, k.Nx, k.Nt, k.m0, n, dir, o0, o1);
            double2 d0, d1;
            dir(n, d0, d1);
            st2w(dn + 2 * n, d0, d1);
        }
        st2w(k.y + 2 * n, o0, o1);
    }
}
// A d = D^dagger y; alpha = (r, r) / (d, A d)
__global__ void __launch_bounds__(256) cg_ad_kernel(KrylovVecs k) {
    const KrylovState* st = k.st;
    if (st->done) return;
    const int it = st->k;
    const int sites = k.Nx * k.Nt;
    const double2* d = k.d[it & 1];
    double2 q[1] = {make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 o0, o1;
        wilson_at<true>(k.U, k.Nx, k.Nt, k.m0, n, [&](int m, double2& a, double2& c) { ld2w(k.y + 2 * m, a, c); },
                        o0, o1);
        st2w(k.Ad[0] + 2 * n, o0, o1);
        double2 d0, d1;
        ld2w(d + 2 * n, d0, d1);
        q[0] = cfmac(o0, d0, cfmac(o1, d1, q[0]));  // sum d conj(A d)
    }
    __shared__ double2 tot[1];
    if (reduce_last<1>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) k.st->alpha = cdiv(st->rnorm2, tot[0]);
}
// x += alpha d, r -= alpha A d; ||r|| (convergence test), beta = ||r||^2 / (r_old, r_old)
__global__ void __launch_bounds__(256) cg_update_kernel(KrylovVecs k) {
    const KrylovState* st = k.st;
    if (st->done) return;
    const int it = st->k;
    const int sites = k.Nx * k.Nt;
    const double2* d = k.d[it & 1];
    const double2 alpha = st->alpha;
    double2 q[1] = {make_double2(0.0, 0.0)};
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < sites; n += gridDim.x * blockDim.x) {
        double2 x0, x1, d0, d1, r0, r1, A0, A1;
        ld2wc(k.x + 2 * n, x0, x1);
        ld2w(d + 2 * n, d0, d1);
        ld2wc(k.r + 2 * n, r0, r1);
        ld2w(k.Ad[0] + 2 * n, A0, A1);
        st2w(k.x + 2 * n, x0 + cmul(alpha, d0), x1 + cmul(alpha, d1));
        r0 = r0 - cmul(alpha, A0);
        r1 = r1 - cmul(alpha, A1);
        st2w(k.r + 2 * n, r0, r1);
        q[0] = cfmac(r0, r0, cfmac(r1, r1, q[0]));
    }
    __shared__ double2 tot[1];
    if (reduce_last<1>(q, k.part, &k.st->ticket, tot) && threadIdx.x == 0) {
        KrylovState* w = k.st;
        const double e2 = tot[0].x;
        w->err = sqrt(e2);
        if (w->err < k.tol * w->norm_b) {
            w->done = 2;
            w->iters = it + 1;
        } else {
            w->beta = cdiv(make_double2(e2, 0.0), w->rnorm2);
            w->rnorm2 = make_double2(e2, 0.0);
            w->k = it + 1;
            if (it + 1 >= k.max_iter) {
                w->done = 3;
                w->iters = k.max_iter;
            }
        }
    }
}

// sets the condition of the solve graph's while node: run another body while the solve is going
__global__ void krylov_continue_kernel(cudaGraphConditionalHandle hc, const KrylovState* st) {
    cudaGraphSetConditional(hc, st->done < 2 ? 1u : 0u);
}

// ---------------------------------------------------------------- host side
// a few CTAs per SM with grid-stride loops: enough warps to keep HBM busy, few partial sums for
// the last CTA to add
int krylov_grid(int sites) { return std::min(ceil_div(sites, 256), 1184); }

static KrylovVecs make_vecs(const KrylovWork& w, const double2* U, int Nx, int Nt, double m0, double tol,
                            int max_iter) {
    KrylovVecs k;
    k.U = U;
    k.b = w.b;
    k.rt = w.rt;
    k.x = w.x;
    k.r = w.r;
    k.s = w.s;
    k.t = w.t;
    k.y = w.y;
    k.d[0] = w.d[0];
    k.d[1] = w.d[1];
    k.Ad[0] = w.Ad[0];
    k.Ad[1] = w.Ad[1];
    k.part = w.part;
    k.st = w.st;
    k.Nx = Nx;
    k.Nt = Nt;
    k.m0 = m0;
    k.tol = tol;
    k.max_iter = max_iter;
    return k;
}

void launch_krylov_init(cudaStream_t s, int solver, const KrylovWork& w, const double2* U, int Nx, int Nt, double m0,
                        double tol, int max_iter) {
    const KrylovVecs k = make_vecs(w, U, Nx, Nt, m0, tol, max_iter);
    const int G = krylov_grid(Nx * Nt);
    DDAMG_CUDA_TRY(cudaMemsetAsync(w.st, 0, sizeof(KrylovState), s));
    if (solver == 0) {
        DDAMG_LAUNCH(bicg_init_kernel, G, 256, 0, s, k);
    } else {
        DDAMG_LAUNCH(cg_init_a_kernel, G, 256, 0, s, k);
        DDAMG_LAUNCH(cg_init_b_kernel, G, 256, 0, s, k);
    }
}

void launch_krylov_iterations(cudaStream_t s, int solver, const KrylovWork& w, const double2* U, int Nx, int Nt,
                              double m0, double tol, int max_iter, int count) {
    const KrylovVecs k = make_vecs(w, U, Nx, Nt, m0, tol, max_iter);
    const int G = krylov_grid(Nx * Nt);
    for (int i = 0; i < count; i++) {
        if (solver == 0) {
            DDAMG_LAUNCH(bicg_dir_kernel, G, 256, 0, s, k);
            DDAMG_LAUNCH(bicg_s_kernel, G, 256, 0, s, k);
            DDAMG_LAUNCH(bicg_update_kernel, G, 256, 0, s, k);
        } else {
            DDAMG_LAUNCH(cg_y_kernel, G, 256, 0, s, k);
            DDAMG_LAUNCH(cg_ad_kernel, G, 256, 0, s, k);
            DDAMG_LAUNCH(cg_update_kernel, G, 256, 0, s, k);
        }
    }
}

void launch_krylov_continue(cudaStream_t s, cudaGraphConditionalHandle hc, const KrylovWork& w) {
    DDAMG_LAUNCH(krylov_continue_kernel, 1, 1, 0, s, hc, w.st);
}

}  // namespace ddamg
