// Vector algebra for the Krylov solvers: fused multi-dot (classical Gram-Schmidt), norms,
// multi-axpy, scaling.  Reductions are two-pass over a fixed grid (deterministic order) and
// accumulate in FP64 whatever the storage precision.
#include "internal.h"

namespace ddamg {

constexpr int kDotChunk = 8;  // basis vectors per multi-dot CTA

// partial[(r*k + i)*kRedBlocks + blk] = sum over this CTA's elements of w_r * conj(B_r,i)
template <typename V>
__global__ void __launch_bounds__(256) multidot_kernel(const V* __restrict__ B, long ldb, long bstride, int k,
                                                       const V* __restrict__ w, long wstride, long n,
                                                       double2* __restrict__ partial) {
    __shared__ double2 red[kDotChunk][8];
    const int r = blockIdx.z, i0 = blockIdx.y * kDotChunk;
    const int kc = min(kDotChunk, k - i0);
    const V* wr = w + r * wstride;
    const V* Br = B + r * bstride + i0 * ldb;
    double2 acc[kDotChunk];
#pragma unroll
    for (int q = 0; q < kDotChunk; q++) acc[q] = make_double2(0.0, 0.0);
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const double2 we = to_d(wr[e]);
#pragma unroll
        for (int q = 0; q < kDotChunk; q++)
            if (q < kc) acc[q] = cfmac(to_d(Br[q * ldb + e]), we, acc[q]);  // w * conj(B)
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kDotChunk; q++) {
        double2 v = warp_sum(acc[q]);
        if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < kc) {
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) s += red[threadIdx.x][j];
        partial[((long)r * k + i0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
}
// out[j] = sum_b partial[j*nb + b], one warp per j
__global__ void finalize_kernel(const double2* __restrict__ partial, int nb, int count, double2* __restrict__ out) {
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= count) return;
    double2 s = make_double2(0.0, 0.0);
    for (int b = lane; b < nb; b += 32) s += partial[(long)j * nb + b];
    s = warp_sum(s);
    if (lane == 0) out[j] = s;
}

template <typename V>
void launch_multidot(cudaStream_t s, const V* B, long ldb, long bstride, int k, const V* w, long wstride, long n,
                     int nrhs, double2* partial, double2* out) {
    if (k <= 0) return;
    int nb = (int)std::min<long>(kRedBlocks, ceil_div(n, 256));
    dim3 grid(nb, ceil_div(k, kDotChunk), nrhs);
    DDAMG_LAUNCH(multidot_kernel<V>, grid, 256, 0, s, B, ldb, bstride, k, w, wstride, n, partial);
    int count = k * nrhs;
    DDAMG_LAUNCH(finalize_kernel, ceil_div(count, 8), 256, 0, s, partial, nb, count, out);
}

template <typename V>
__global__ void __launch_bounds__(256) norm2_kernel(const V* __restrict__ x, long xstride, long n,
                                                    double2* __restrict__ partial) {
    __shared__ double red[8];
    const V* xr = x + blockIdx.y * xstride;
    double acc = 0.0;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        double2 v = to_d(xr[e]);
        acc = fma(v.x, v.x, fma(v.y, v.y, acc));
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) s += red[j];
        partial[(long)blockIdx.y * gridDim.x + blockIdx.x] = make_double2(s, 0.0);
    }
}
__global__ void finalize_real_kernel(const double2* __restrict__ partial, int nb, int count, double* __restrict__ out) {
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= count) return;
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += partial[(long)j * nb + b].x;
    s = warp_sum(s);
    if (lane == 0) out[j] = s;
}
template <typename V>
void launch_norm2(cudaStream_t s, const V* x, long xstride, long n, int nrhs, double2* partial, double* out) {
    int nb = (int)std::min<long>(kRedBlocks, ceil_div(n, 256));
    DDAMG_LAUNCH(norm2_kernel<V>, dim3(nb, nrhs), 256, 0, s, x, xstride, n, partial);
    DDAMG_LAUNCH(finalize_real_kernel, ceil_div(nrhs, 8), 256, 0, s, partial, nb, nrhs, out);
}

// w_r += sign * sum_i coef[r*k+i] * B_r,i
template <typename V>
__global__ void __launch_bounds__(256) multiaxpy_kernel(const V* __restrict__ B, long ldb, long bstride, int k,
                                                        const double2* __restrict__ coef, V* __restrict__ w,
                                                        long wstride, long n, double sign) {
    typedef typename RealOf<V>::R R;
    const int r = blockIdx.y;
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const V* Br = B + r * bstride;
    const double2* cr = coef + (long)r * k;
    double2 acc = make_double2(0.0, 0.0);
    for (int i = 0; i < k; i++) acc = cfma(__ldg(cr + i), to_d(Br[i * ldb + e]), acc);
    V* wr = w + r * wstride;
    double2 v = to_d(wr[e]);
    v.x += sign * acc.x;
    v.y += sign * acc.y;
    wr[e] = from_d<V>(v);
    (void)sizeof(R);
}
template <typename V>
void launch_multiaxpy(cudaStream_t s, const V* B, long ldb, long bstride, int k, const double2* coef, V* w,
                      long wstride, long n, int nrhs, double sign) {
    if (k <= 0) return;
    DDAMG_LAUNCH(multiaxpy_kernel<V>, dim3(ceil_div(n, 256), nrhs), 256, 0, s, B, ldb, bstride, k, coef, w, wstride,
                 n, sign);
}

template <typename V>
__global__ void scale_kernel(const double2* __restrict__ alpha, const V* __restrict__ x, V* __restrict__ y, long n) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const long o = blockIdx.y * n;
    y[o + e] = from_d<V>(cmul(alpha[blockIdx.y], to_d(x[o + e])));
}
template <typename V> void launch_scale(cudaStream_t s, const double2* alpha, const V* x, V* y, long n, int nrhs) {
    DDAMG_LAUNCH(scale_kernel<V>, dim3(ceil_div(n, 256), nrhs), 256, 0, s, alpha, x, y, n);
}
template <typename V> __global__ void sub_kernel(const V* a, const V* b, V* r, long n) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) r[e] = a[e] - b[e];
}
template <typename V> void launch_sub(cudaStream_t s, const V* a, const V* b, V* r, long n) {
    if (n <= 0) return;
    DDAMG_LAUNCH(sub_kernel<V>, ceil_div(n, 256), 256, 0, s, a, b, r, n);
}
template <typename V> __global__ void add_kernel(const V* x, V* y, long n) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) y[e] += x[e];
}
template <typename V> void launch_add(cudaStream_t s, const V* x, V* y, long n) {
    if (n <= 0) return;
    DDAMG_LAUNCH(add_kernel<V>, ceil_div(n, 256), 256, 0, s, x, y, n);
}
// done[r] = it + 1 the first time sqrt(rr[r]) < tol * sqrt(vv[r]) (SAP's early return, src/sap.cpp:152-158)
__global__ void flag_converged_kernel(const double* rr, const double* vv, double tol, int nrhs, int it, int* done) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrhs && done[r] == 0 && sqrt(rr[r]) < tol * sqrt(vv[r])) done[r] = it + 1;
}
void launch_flag_converged(cudaStream_t s, const double* rr, const double* vv, double tol, int nrhs, int it,
                           int* done) {
    DDAMG_LAUNCH(flag_converged_kernel, ceil_div(nrhs, 128), 128, 0, s, rr, vv, tol, nrhs, it, done);
}
template <typename V> __global__ void scale_host_kernel(double2 alpha, const V* x, V* y, long n) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e < n) y[e] = from_d<V>(cmul(alpha, to_d(x[e])));
}
template <typename V> void launch_scale_host(cudaStream_t s, double2 alpha, const V* x, V* y, long n) {
    if (n <= 0) return;
    DDAMG_LAUNCH(scale_host_kernel<V>, ceil_div(n, 256), 256, 0, s, alpha, x, y, n);
}
// sigma_3 on fine spinors: negate spin component 1
__global__ void sigma3_kernel(const double2* x, double2* y, long sites) {
    const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (n < sites) {
        y[2 * n] = x[2 * n];
        y[2 * n + 1] = -x[2 * n + 1];
    }
}
void launch_sigma3(cudaStream_t s, const double2* x, double2* y, long sites) {
    DDAMG_LAUNCH(sigma3_kernel, ceil_div(sites, 256), 256, 0, s, x, y, sites);
}

#define DDAMG_INST_BLAS(V)                                                                                 \
    template void launch_multidot<V>(cudaStream_t, const V*, long, long, int, const V*, long, long, int,   \
                                     double2*, double2*);                                                  \
    template void launch_norm2<V>(cudaStream_t, const V*, long, long, int, double2*, double*);             \
    template void launch_multiaxpy<V>(cudaStream_t, const V*, long, long, int, const double2*, V*, long,   \
                                      long, int, double);                                                  \
    template void launch_scale<V>(cudaStream_t, const double2*, const V*, V*, long, int);                  \
    template void launch_sub<V>(cudaStream_t, const V*, const V*, V*, long);                               \
    template void launch_add<V>(cudaStream_t, const V*, V*, long);                                         \
    template void launch_scale_host<V>(cudaStream_t, double2, const V*, V*, long);
DDAMG_INST_BLAS(double2)
DDAMG_INST_BLAS(float2)

}  // namespace ddamg
