// Shared device/host helpers for the DD-alphaAMG B200 library.
#pragma once
#include <atomic>

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "ddamg.h"

namespace ddamg {

// ---------------------------------------------------------------- complex arithmetic
// Complex numbers are CUDA's double2 / float2 (x = re, y = im); fields are arrays of them.
template <typename R> struct CxT;
template <> struct CxT<double> { typedef double2 V; };
template <> struct CxT<float> { typedef float2 V; };
template <typename V> struct RealOf;
template <> struct RealOf<double2> { typedef double R; };
template <> struct RealOf<float2> { typedef float R; };

#define DDAMG_HD __host__ __device__ __forceinline__

DDAMG_HD double2 mkc(double a, double b) { return make_double2(a, b); }
DDAMG_HD float2 mkc(float a, float b) { return make_float2(a, b); }
template <typename V> DDAMG_HD V czero() { return mkc(typename RealOf<V>::R(0), typename RealOf<V>::R(0)); }

#define DDAMG_CX_OPS(V, R)                                                                        \
    DDAMG_HD V operator+(V a, V b) { return mkc(a.x + b.x, a.y + b.y); }                          \
    DDAMG_HD V operator-(V a, V b) { return mkc(a.x - b.x, a.y - b.y); }                          \
    DDAMG_HD V operator-(V a) { return mkc(-a.x, -a.y); }                                         \
    DDAMG_HD V operator*(R s, V a) { return mkc(s * a.x, s * a.y); }                              \
    DDAMG_HD V& operator+=(V& a, V b) { a.x += b.x; a.y += b.y; return a; }                       \
    DDAMG_HD V& operator-=(V& a, V b) { a.x -= b.x; a.y -= b.y; return a; }                       \
    /* a * b */                                                                                   \
    DDAMG_HD V cmul(V a, V b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }      \
    /* conj(a) * b */                                                                             \
    DDAMG_HD V cmulc(V a, V b) { return mkc(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }     \
    /* acc + a * b */                                                                             \
    DDAMG_HD V cfma(V a, V b, V acc) {                                                            \
        return mkc(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));    \
    }                                                                                             \
    /* acc + conj(a) * b */                                                                       \
    DDAMG_HD V cfmac(V a, V b, V acc) {                                                           \
        return mkc(fma(a.x, b.x, fma(a.y, b.y, acc.x)), fma(a.x, b.y, fma(-a.y, b.x, acc.y)));    \
    }                                                                                             \
    DDAMG_HD V conjc(V a) { return mkc(a.x, -a.y); }                                              \
    /* i * a */                                                                                   \
    DDAMG_HD V imul(V a) { return mkc(-a.y, a.x); }                                               \
    DDAMG_HD R cnorm2(V a) { return a.x * a.x + a.y * a.y; }

DDAMG_CX_OPS(double2, double)
DDAMG_CX_OPS(float2, float)

DDAMG_HD double2 to_d(float2 a) { return make_double2(a.x, a.y); }
DDAMG_HD double2 to_d(double2 a) { return a; }
template <typename V> DDAMG_HD V from_d(double2 a);
template <> DDAMG_HD double2 from_d<double2>(double2 a) { return a; }
template <> DDAMG_HD float2 from_d<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

// complex division (Smith's algorithm), used for Givens rotations / back substitution
DDAMG_HD double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    } else {
        double r = b.x / b.y, den = b.x * r + b.y;
        return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
    }
}
DDAMG_HD float2 cdiv(float2 a, float2 b) {
    if (fabsf(b.x) >= fabsf(b.y)) {
        float r = b.y / b.x, den = b.x + b.y * r;
        return make_float2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    } else {
        float r = b.x / b.y, den = b.x * r + b.y;
        return make_float2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
    }
}

// ---------------------------------------------------------------- 256-bit site accesses
// One 32-byte access for the two spin components of an FP64 fine-lattice site (ld.global.nc.v4.f64 /
// st.global.v4.f64, sm_100).  The address must be 32-byte aligned: device buffers from cudaMalloc and
// site offsets (32 bytes each) keep it; callers that take outside pointers check first.
__device__ __forceinline__ void ld2w(const double2* __restrict__ p, double2& a, double2& b) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p));
}
// the same through the coherent path, for a field the kernel also writes
__device__ __forceinline__ void ld2wc(const double2* p, double2& a, double2& b) {
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p)
                 : "memory");
}
__device__ __forceinline__ void st2w(double2* p, double2 a, double2 b) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
                 : "memory");
}

// ---------------------------------------------------------------- warp / block reductions
__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ float2 warp_sum(float2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Sum over the whole CTA; every thread gets the result. `scratch` holds >= 33 V (shared).
template <typename V>
__device__ __forceinline__ V block_sum(V v, V* scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();  // protect scratch from the previous use
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    if (wid == 0) {
        V s = (lane < nw) ? scratch[lane] : V{};
        s = warp_sum(s);
        if (lane == 0) scratch[32] = s;
    }
    __syncthreads();
    return scratch[32];
}

// ---------------------------------------------------------------- counter-based RNG
// splitmix64 finaliser (Steele, Lea & Flood 2014), keyed by (seed, stream, counter);
// identical to orc_rng in the CPU oracle so device draws match it bit for bit.
DDAMG_HD uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
DDAMG_HD uint64_t rng64(uint64_t seed, uint64_t stream, uint64_t counter) {
    return mix64(mix64(seed ^ mix64(stream)) + counter);
}
DDAMG_HD double u01(uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; }
constexpr uint64_t kStreamUniform = 0x7E57ull;   // test vectors, re/im ~ U(-1,1)
constexpr uint64_t kStreamGauss = 0x6A55ull;     // Gaussian right-hand sides
constexpr uint64_t kStreamHotStart = 0xC0FFEEull;  // Metropolis hot start

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
struct Status {
    ddamg_status code = DDAMG_OK;
};
#define DDAMG_CUDA_TRY(expr)                                                                      \
    do {                                                                                          \
        cudaError_t e__ = (expr);                                                                 \
        if (e__ != cudaSuccess) {                                                                 \
            ::ddamg::set_error(std::string(#expr) + ": " + cudaGetErrorString(e__) + " (" +       \
                               __FILE__ + ":" + std::to_string(__LINE__) + ")");                  \
            throw ::ddamg::CudaFailure();                                                         \
        }                                                                                         \
    } while (0)
struct CudaFailure {};
struct ParamFailure {
    std::string msg;
};
struct TimeoutFailure {};
struct NanFailure {  // a NaN / Inf in an input or an iterate -> DDAMG_ERR_NAN
    std::string msg;
};
struct NotConvergedFailure {  // an inner solve that a call depends on missed its tolerance -> DDAMG_NOT_CONVERGED
    std::string msg;
};
struct IoFailure {  // a file that cannot be opened or written -> DDAMG_ERR_IO
    std::string msg;
};

// launch bookkeeping: every kernel launch in the library goes through this counter
extern std::atomic<long long> g_launches;  // kernels launched by the library (all handles)
#define DDAMG_LAUNCH(kernel, grid, block, smem, stream, ...)                                      \
    do {                                                                                          \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                               \
        ++::ddamg::g_launches;                                                                    \
        DDAMG_CUDA_TRY(cudaGetLastError());                                                       \
    } while (0)

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace ddamg
