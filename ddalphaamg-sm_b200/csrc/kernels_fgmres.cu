// Device-driven FGMRES (FGMRES::fgmres, src/fgmres.cpp:5-128) for R right-hand sides in lockstep: the
// Arnoldi bookkeeping that the host loop does between launches (Hessenberg column, Givens rotations,
// convergence test, back substitution, restart test) runs in small one-CTA kernels, and the loop
// control goes to CUDA graph conditional nodes (cudaGraphSetConditional), so a whole solve runs as one
// graph without a host round trip.  The arithmetic is the host loop's, operation for operation.
//
// Basis slots are addressed through the step counter on the device (ctl[kFgJ]), so one captured body
// serves every Arnoldi step: the multi-dot, multi-axpy and scaling kernels below read k = j + 1 there.
#include "internal.h"

namespace ddamg {

constexpr int kFgThreads = 128;

// ---------------------------------------------------------------- loop control (one CTA)
// start of a solve: norms of b and of r = b - A x0 (nrm[0, R) and nrm[R, 2R)), per-rhs state
__global__ void __launch_bounds__(kFgThreads) fg_start_kernel(FgDev f, int R, int m, int restarts,
                                                              cudaGraphConditionalHandle hc_outer) {
    bool active = false;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const double nb = sqrt(f.nrm[r]), e = sqrt(f.nrm[R + r]);
        int done = nb == 0.0;  // zero right-hand side: x = x0 = 0
        if (!(nb == nb) || !(e == e)) {
            f.ctl[kFgNan] = 1;
            done = 1;
        }
        f.norm_b[r] = nb;
        f.err[r] = e;
        f.maxIt[r] = m;
        f.ret[r] = restarts * m;
        f.done[r] = done;
        active |= !done;
    }
    const bool any = __syncthreads_or(active);
    if (threadIdx.x == 0) {
        f.ctl[kFgJ] = 0;
        f.ctl[kFgK] = 0;
        cudaGraphSetConditional(hc_outer, (any && restarts > 0) ? 1u : 0u);
    }
}

// top of a restart: V_0 = r / ||r|| for the right-hand sides still running (alpha), g = (||r||, 0, ...);
// with select, the K-cycle's if/else node runs the loop of restart 0 (preconditioner from zero) or the
// loop of later restarts (from the previous Z_j, src/amg.cpp:43-45)
__global__ void __launch_bounds__(kFgThreads) fg_restart_kernel(FgDev f, int R, int m, cudaGraphConditionalHandle hc0,
                                                                cudaGraphConditionalHandle hc1,
                                                                cudaGraphConditionalHandle hc_sel, int select) {
    bool active = false;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const int run = !f.done[r];
        f.arn[r] = run;
        f.alpha[r] = make_double2(run ? 1.0 / f.err[r] : 0.0, 0.0);
        f.gm[(long)r * (m + 1)] = make_double2(f.err[r], 0.0);
        active |= run;
    }
    const bool any = __syncthreads_or(active);
    if (threadIdx.x == 0) {
        f.ctl[kFgJ] = 0;
        f.ctl[kFgRunsOuter]++;
        cudaGraphSetConditional(hc0, any ? 1u : 0u);
        if (select) {
            const bool first = f.ctl[kFgK] == 0;
            cudaGraphSetConditional(hc1, any ? 1u : 0u);
            cudaGraphSetConditional(hc_sel, first ? 1u : 0u);
            f.ctl[first ? kFgRunsFirst : kFgRunsLater]++;
        }
    }
}

// end of Arnoldi step j: column j of H from the two Gram-Schmidt passes (dots[0] + dots[1]) and
// ||w||, the previous rotations, a new rotation, the residual estimate |g_{j+1}| and the scale of
// V_{j+1} (src/fgmres.cpp:35-70, FGMRES::rotation src/fgmres.cpp:99-115)
__global__ void __launch_bounds__(kFgThreads) fg_arnoldi_kernel(FgDev f, int R, int m, double tol,
                                                                cudaGraphConditionalHandle hc_inner, int counter) {
    const int j = f.ctl[kFgJ];
    bool active = false;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        f.alpha[r] = make_double2(0.0, 0.0);
        if (!f.arn[r]) continue;
        double2* Hr = f.H + (long)r * (m + 1) * m;
        double2* gr = f.gm + (long)r * (m + 1);
        double2* cr = f.cn + (long)r * m;
        double2* sr = f.sn + (long)r * m;
        const double2* d1 = f.dots + (long)r * (m + 1);
        const double2* d2 = f.dots + (long)(R + r) * (m + 1);
        for (int i = 0; i <= j; i++) Hr[(long)i * m + j] = d1[i] + d2[i];
        const double hn = sqrt(f.nrm[r]);
        if (!(hn == hn)) {  // NaN in the Krylov basis: stop this right-hand side, report after the solve
            f.ctl[kFgNan] = 1;
            f.arn[r] = 0;
            f.done[r] = 1;
            continue;
        }
        Hr[(long)(j + 1) * m + j] = make_double2(hn, 0.0);
        if (hn > 0) f.alpha[r] = make_double2(1.0 / hn, 0.0);
        for (int i = 0; i < j; i++) {
            const double2 a = Hr[(long)i * m + j], b = Hr[(long)(i + 1) * m + j];
            const double2 tmp = cmulc(cr[i], a) + cmulc(sr[i], b);
            Hr[(long)(i + 1) * m + j] = cmul(cr[i], b) - cmul(sr[i], a);
            Hr[(long)i * m + j] = tmp;
        }
        const double2 hjj = Hr[(long)j * m + j], hj1 = Hr[(long)(j + 1) * m + j];
        const double den = sqrt(cnorm2(hjj) + cnorm2(hj1));
        sr[j] = make_double2(hj1.x / den, hj1.y / den);
        cr[j] = make_double2(hjj.x / den, hjj.y / den);
        Hr[(long)j * m + j] = cmulc(cr[j], hjj) + cmulc(sr[j], hj1);
        Hr[(long)(j + 1) * m + j] = make_double2(0.0, 0.0);
        gr[j + 1] = -cmul(sr[j], gr[j]);
        gr[j] = cmulc(cr[j], gr[j]);
        if (sqrt(cnorm2(gr[j + 1])) < tol * f.norm_b[r]) {
            f.maxIt[r] = j + 1;
            f.arn[r] = 0;
            f.alpha[r] = make_double2(0.0, 0.0);  // V_{j+1} is not used again
        }
        active |= f.arn[r] != 0;
    }
    const bool any = __syncthreads_or(active);
    if (threadIdx.x == 0) {
        f.ctl[kFgJ] = j + 1;
        f.ctl[counter]++;
        cudaGraphSetConditional(hc_inner, (any && j + 1 < m) ? 1u : 0u);
    }
}

// solve_upper_triangular (src/fgmres.cpp:118-128): coef = H^-1 g over the first maxIt columns
__global__ void __launch_bounds__(kFgThreads) fg_backsub_kernel(FgDev f, int R, int m) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        double2* cf = f.coef + (long)r * m;
        for (int i = 0; i < m; i++) cf[i] = make_double2(0.0, 0.0);
        if (f.done[r]) continue;
        const double2* Hr = f.H + (long)r * (m + 1) * m;
        const double2* gr = f.gm + (long)r * (m + 1);
        const int mi = f.maxIt[r];
        for (int i = mi - 1; i >= 0; i--) {
            double2 e = gr[i];
            for (int jj = i + 1; jj < mi; jj++) e = e - cmul(Hr[(long)i * m + jj], cf[jj]);
            cf[i] = cdiv(e, Hr[(long)i * m + i]);
        }
    }
}

// end of restart k: the true residual norm (nrm[0, R)) decides convergence (src/fgmres.cpp:72-90)
__global__ void __launch_bounds__(kFgThreads) fg_restart_end_kernel(FgDev f, int R, int m, int restarts, double tol,
                                                                    cudaGraphConditionalHandle hc_outer) {
    const int k = f.ctl[kFgK];
    bool left = false;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        if (f.done[r]) continue;
        const double e = sqrt(f.nrm[r]);
        f.err[r] = e;
        if (!(e == e)) {
            f.ctl[kFgNan] = 1;
            f.done[r] = 1;
            continue;
        }
        if (e < tol * f.norm_b[r]) {
            f.ret[r] = k * m + f.maxIt[r];
            f.done[r] = 1;
        }
        left |= !f.done[r];
    }
    const bool any = __syncthreads_or(left);
    if (threadIdx.x == 0) {
        f.ctl[kFgK] = k + 1;
        cudaGraphSetConditional(hc_outer, (any && k + 1 < restarts) ? 1u : 0u);
    }
}

// ---------------------------------------------------------------- basis kernels indexed on the device
constexpr int kDotChunkDev = 8;

// dots[(pass*R + r)*(m+1) + i] partials over V_0..V_j (k = j + 1 from the device) against w; the same
// per-thread order and grid as the host loop's multi-dot
template <typename V>
__global__ void __launch_bounds__(256) multidot_dev_kernel(const V* __restrict__ B, long ldb, long bstride,
                                                           const int* __restrict__ jdev, int ldk,
                                                           const V* __restrict__ w, long wstride, long n,
                                                           double2* __restrict__ partial) {
    __shared__ double2 red[kDotChunkDev][8];
    const int k = *jdev + 1;
    const int r = blockIdx.z, i0 = blockIdx.y * kDotChunkDev;
    if (i0 >= k) return;  // uniform over the CTA
    const int kc = min(kDotChunkDev, k - i0);
    const V* wr = w + r * wstride;
    const V* Br = B + r * bstride + i0 * ldb;
    double2 acc[kDotChunkDev];
#pragma unroll
    for (int q = 0; q < kDotChunkDev; q++) acc[q] = make_double2(0.0, 0.0);
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const double2 we = to_d(wr[e]);
#pragma unroll
        for (int q = 0; q < kDotChunkDev; q++)
            if (q < kc) acc[q] = cfmac(to_d(Br[q * ldb + e]), we, acc[q]);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kDotChunkDev; q++) {
        double2 v = warp_sum(acc[q]);
        if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < kc) {
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) s += red[threadIdx.x][j];
        partial[((long)r * ldk + i0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
}
__global__ void finalize_dev_kernel(const double2* __restrict__ partial, int nb, int R, int ldk,
                                    const int* __restrict__ jdev, double2* __restrict__ out) {
    const int idx = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (idx >= R * ldk || idx % ldk > *jdev) return;
    double2 s = make_double2(0.0, 0.0);
    for (int b = lane; b < nb; b += 32) s += partial[(long)idx * nb + b];
    s = warp_sum(s);
    if (lane == 0) out[idx] = s;
}
template <typename V>
void launch_multidot_dev(cudaStream_t s, const V* B, long ldb, long bstride, int kmax, const int* jdev, int ldk,
                         const V* w, long wstride, long n, int nrhs, double2* partial, double2* out) {
    int nb = (int)std::min<long>(kRedBlocks, ceil_div(n, 256));
    dim3 grid(nb, ceil_div(kmax, kDotChunkDev), nrhs);
    DDAMG_LAUNCH(multidot_dev_kernel<V>, grid, 256, 0, s, B, ldb, bstride, jdev, ldk, w, wstride, n, partial);
    DDAMG_LAUNCH(finalize_dev_kernel, ceil_div(nrhs * ldk, 8), 256, 0, s, partial, nb, nrhs, ldk, jdev, out);
}

// w_r -= sum_{i <= j} coef[r*ldk + i] B_r,i
template <typename V>
__global__ void __launch_bounds__(256) multiaxpy_dev_kernel(const V* __restrict__ B, long ldb, long bstride,
                                                            const int* __restrict__ jdev,
                                                            const double2* __restrict__ coef, int ldk,
                                                            V* __restrict__ w, long wstride, long n) {
    const int r = blockIdx.y;
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int k = *jdev + 1;
    const V* Br = B + r * bstride;
    const double2* cr = coef + (long)r * ldk;
    double2 acc = make_double2(0.0, 0.0);
    for (int i = 0; i < k; i++) acc = cfma(__ldg(cr + i), to_d(Br[i * ldb + e]), acc);
    V* wr = w + r * wstride;
    double2 v = to_d(wr[e]);
    v.x += -1.0 * acc.x;
    v.y += -1.0 * acc.y;
    wr[e] = from_d<V>(v);
}
template <typename V>
void launch_multiaxpy_dev(cudaStream_t s, const V* B, long ldb, long bstride, const int* jdev, const double2* coef,
                          int ldk, V* w, long wstride, long n, int nrhs) {
    DDAMG_LAUNCH(multiaxpy_dev_kernel<V>, dim3(ceil_div(n, 256), nrhs), 256, 0, s, B, ldb, bstride, jdev, coef, ldk,
                 w, wstride, n);
}

// V_j = alpha_r x_r with j from the device (slot stride: R n)
template <typename V>
__global__ void scale_slot_kernel(const double2* __restrict__ alpha, const V* __restrict__ x, V* __restrict__ Vb,
                                  long slot, const int* __restrict__ jdev, long n) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const long o = blockIdx.y * n;
    Vb[*jdev * slot + o + e] = from_d<V>(cmul(alpha[blockIdx.y], to_d(x[o + e])));
}
template <typename V>
void launch_scale_slot(cudaStream_t s, const double2* alpha, const V* x, V* Vb, long slot, const int* jdev, long n,
                       int nrhs) {
    DDAMG_LAUNCH(scale_slot_kernel<V>, dim3(ceil_div(n, 256), nrhs), 256, 0, s, alpha, x, Vb, slot, jdev, n);
}

// copies between basis slot j (from the device) and a fixed buffer, converting the element type
template <typename A, typename B>
__global__ void slot_copy_kernel(const A* __restrict__ src, B* __restrict__ dst, long slot, const int* __restrict__ jdev,
                                 int to_slot, long count) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= count) return;
    const long o = (long)*jdev * slot;
    if (to_slot) dst[o + e] = from_d<B>(to_d(src[e]));
    else dst[e] = from_d<B>(to_d(src[o + e]));
}
template <typename A, typename B>
void launch_slot_copy(cudaStream_t s, const A* src, B* dst, long slot, const int* jdev, int to_slot, long count) {
    DDAMG_LAUNCH((slot_copy_kernel<A, B>), ceil_div(count, 256), 256, 0, s, src, dst, slot, jdev, to_slot, count);
}

// ---------------------------------------------------------------- launchers of the control kernels
void launch_fg_start(cudaStream_t s, const FgDev& f, int R, int m, int restarts, cudaGraphConditionalHandle hc) {
    DDAMG_LAUNCH(fg_start_kernel, 1, kFgThreads, 0, s, f, R, m, restarts, hc);
}
void launch_fg_restart(cudaStream_t s, const FgDev& f, int R, int m, cudaGraphConditionalHandle hc0,
                       cudaGraphConditionalHandle hc1, cudaGraphConditionalHandle hc_sel, int select) {
    DDAMG_LAUNCH(fg_restart_kernel, 1, kFgThreads, 0, s, f, R, m, hc0, hc1, hc_sel, select);
}
void launch_fg_arnoldi(cudaStream_t s, const FgDev& f, int R, int m, double tol, cudaGraphConditionalHandle hc,
                       int counter) {
    DDAMG_LAUNCH(fg_arnoldi_kernel, 1, kFgThreads, 0, s, f, R, m, tol, hc, counter);
}
void launch_fg_backsub(cudaStream_t s, const FgDev& f, int R, int m) {
    DDAMG_LAUNCH(fg_backsub_kernel, 1, kFgThreads, 0, s, f, R, m);
}
void launch_fg_restart_end(cudaStream_t s, const FgDev& f, int R, int m, int restarts, double tol,
                           cudaGraphConditionalHandle hc) {
    DDAMG_LAUNCH(fg_restart_end_kernel, 1, kFgThreads, 0, s, f, R, m, restarts, tol, hc);
}
#define DDAMG_FG_INST(V)                                                                                      \
    template void launch_multidot_dev<V>(cudaStream_t, const V*, long, long, int, const int*, int, const V*,  \
                                         long, long, int, double2*, double2*);                                \
    template void launch_multiaxpy_dev<V>(cudaStream_t, const V*, long, long, const int*, const double2*, int, \
                                          V*, long, long, int);                                               \
    template void launch_scale_slot<V>(cudaStream_t, const double2*, const V*, V*, long, const int*, long, int);
DDAMG_FG_INST(double2)
DDAMG_FG_INST(float2)
template void launch_slot_copy<double2, double2>(cudaStream_t, const double2*, double2*, long, const int*, int, long);
template void launch_slot_copy<double2, float2>(cudaStream_t, const double2*, float2*, long, const int*, int, long);
template void launch_slot_copy<float2, double2>(cudaStream_t, const float2*, double2*, long, const int*, int, long);
template void launch_slot_copy<float2, float2>(cudaStream_t, const float2*, float2*, long, const int*, int, long);

}  // namespace ddamg
