// Fine-level kernels: Wilson-Dirac stencil D_W / D_W^dagger on U(1) links, the link
// derivative of L = Re(eta^dagger D^-1 b), the U(1) Metropolis generator and field fills.
#include "internal.h"

namespace ddamg {

// Two complex values per site; one 16-byte (float2 x 2) or two 16-byte (double2 x 2) loads.
__device__ __forceinline__ void ld2(const double2* __restrict__ p, double2& a, double2& b) {
    a = __ldg(p);
    b = __ldg(p + 1);
}
__device__ __forceinline__ void ld2(const float2* __restrict__ p, float2& a, float2& b) {
    float4 v = __ldg(reinterpret_cast<const float4*>(p));
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
}
__device__ __forceinline__ void st2(double2* p, double2 a, double2 b) {
    p[0] = a;
    p[1] = b;
}
__device__ __forceinline__ void st2(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void ld2w(const float2* __restrict__ p, float2& a, float2& b) { ld2(p, a, b); }
__device__ __forceinline__ void st2w(float2* p, float2 a, float2 b) { st2(p, a, b); }

// D_phi / D_dagger_phi, src/dirac_operator.cpp:24-85, written with the spin projections
// (1 -/+ sigma_mu) factored: each hop is one link multiply.  sigma_0 = sigma_x acts along t
// (mu = 0), sigma_1 = sigma_y along x (mu = 1); the t-wrap hop carries the antiperiodic sign.
template <typename V, bool DAG, bool RESID, bool W = false>
__global__ void __launch_bounds__(256) wilson_kernel(const V* __restrict__ U, const V* __restrict__ in,
                                                     V* __restrict__ out, const V* __restrict__ b, int Nx, int Nt,
                                                     typename RealOf<V>::R m0, long stride) {
    typedef typename RealOf<V>::R R;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nx * Nt) return;
    const long ro = (long)blockIdx.y * stride;
    in += ro;
    out += ro;
    const int x = n / Nt, t = n - x * Nt;
    const int tp = (t + 1 == Nt) ? 0 : t + 1, tm = (t == 0) ? Nt - 1 : t - 1;
    const int xp = (x + 1 == Nx) ? 0 : x + 1, xm = (x == 0) ? Nx - 1 : x - 1;
    const int r0 = x * Nt + tp, l0 = x * Nt + tm, r1 = xp * Nt + t, l1 = xm * Nt + t;
    const R sr = (t == Nt - 1) ? R(-1) : R(1), sl = (t == 0) ? R(-1) : R(1);

    V u0, u1, ul0, ul1;
    V p0, p1, a0, a1, c0, c1, e0, e1, g0, g1;
    if (W) {
        ld2w(U + 2 * n, u0, u1);
        ld2w(in + 2 * n, p0, p1);
        ld2w(in + 2 * r0, a0, a1);
        ld2w(in + 2 * r1, c0, c1);
        ld2w(in + 2 * l0, e0, e1);
        ld2w(in + 2 * l1, g0, g1);
    } else {
        ld2(U + 2 * n, u0, u1);
        ld2(in + 2 * n, p0, p1);
        ld2(in + 2 * r0, a0, a1);
        ld2(in + 2 * r1, c0, c1);
        ld2(in + 2 * l0, e0, e1);
        ld2(in + 2 * l1, g0, g1);
    }
    ul0 = __ldg(U + 2 * l0);
    ul1 = __ldg(U + 2 * l1 + 1);
    V s0, s1;
    if (!DAG) {
        V a = sr * cmul(u0, a0 - a1);             // +t: (1 - sigma_x)
        V c = cmul(u1, c0 + imul(c1));           // +x: (1 - sigma_y)
        V e = sl * cmulc(ul0, e0 + e1);          // -t: (1 + sigma_x)
        V g = cmulc(ul1, g0 - imul(g1));         // -x: (1 + sigma_y)
        s0 = a + c + e + g;
        s1 = -a - imul(c) + e + imul(g);
    } else {
        V a = sl * cmulc(ul0, e0 - e1);          // -t: (1 - sigma_x)
        V c = cmulc(ul1, g0 + imul(g1));         // -x: (1 - sigma_y)
        V e = sr * cmul(u0, a0 + a1);            // +t: (1 + sigma_x)
        V g = cmul(u1, c0 - imul(c1));           // +x: (1 + sigma_y)
        s0 = a + c + e + g;
        s1 = -a - imul(c) + e + imul(g);
    }
    const R mm = m0 + R(2), h = R(0.5);
    V o0 = mm * p0 - h * s0;
    V o1 = mm * p1 - h * s1;
    if (RESID) {
        V b0, b1;
        if (W) ld2w(b + ro + 2 * n, b0, b1);
        else ld2(b + ro + 2 * n, b0, b1);
        o0 = b0 - o0;
        o1 = b1 - o1;
    }
    if (W) st2w(out + 2 * n, o0, o1);
    else st2(out + 2 * n, o0, o1);
}

// FP32 D_W with the two sites (x, t0), (x, t0 + 1), t0 even, per thread: the pair's psi, its links
// and its output are each one 32-byte access (ld.global.nc.v8.f32 / st.global.v8.f32), so every warp
// instruction covers 1 KB of contiguous memory; the t-neighbours inside the pair come from registers.
__device__ __forceinline__ void ld8f(const float2* __restrict__ p, float2& a, float2& b, float2& c, float2& d) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(b.x), "=f"(b.y), "=f"(c.x), "=f"(c.y), "=f"(d.x), "=f"(d.y)
        : "l"(p));
}
__device__ __forceinline__ void st8f(float2* p, float2 a, float2 b, float2 c, float2 d) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x), "f"(a.y), "f"(b.x),
                 "f"(b.y), "f"(c.x), "f"(c.y), "f"(d.x), "f"(d.y)
                 : "memory");
}
// one site of D_phi / D_dagger_phi from its links and neighbours (the arithmetic of wilson_kernel)
template <bool DAG>
__device__ __forceinline__ void wilson_site(float2 u0, float2 u1, float2 ul0, float2 ul1, float2 p0, float2 p1,
                                            float2 a0, float2 a1, float2 c0, float2 c1, float2 e0, float2 e1,
                                            float2 g0, float2 g1, float sr, float sl, float mm, float2& o0,
                                            float2& o1) {
    float2 s0, s1;
    if (!DAG) {
        float2 a = sr * cmul(u0, a0 - a1);      // +t: (1 - sigma_x)
        float2 c = cmul(u1, c0 + imul(c1));    // +x: (1 - sigma_y)
        float2 e = sl * cmulc(ul0, e0 + e1);   // -t: (1 + sigma_x)
        float2 g = cmulc(ul1, g0 - imul(g1));  // -x: (1 + sigma_y)
        s0 = a + c + e + g;
        s1 = -a - imul(c) + e + imul(g);
    } else {
        float2 a = sl * cmulc(ul0, e0 - e1);   // -t: (1 - sigma_x)
        float2 c = cmulc(ul1, g0 + imul(g1));  // -x: (1 - sigma_y)
        float2 e = sr * cmul(u0, a0 + a1);     // +t: (1 + sigma_x)
        float2 g = cmul(u1, c0 - imul(c1));    // +x: (1 + sigma_y)
        s0 = a + c + e + g;
        s1 = -a - imul(c) + e + imul(g);
    }
    o0 = mm * p0 - 0.5f * s0;
    o1 = mm * p1 - 0.5f * s1;
}
template <bool DAG, bool RESID>
__global__ void __launch_bounds__(256) wilson_pair_kernel(const float2* __restrict__ U, const float2* __restrict__ in,
                                                          float2* __restrict__ out, const float2* __restrict__ b,
                                                          int Nx, int Nt, float m0, long stride) {
    const int n0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (n0 >= Nx * Nt) return;
    const long ro = (long)blockIdx.y * stride;
    in += ro;
    out += ro;
    const int x = n0 / Nt, t0 = n0 - x * Nt;
    const int xp = (x + 1 == Nx) ? 0 : x + 1, xm = (x == 0) ? Nx - 1 : x - 1;
    const int tm = (t0 == 0) ? Nt - 1 : t0 - 1, tp = (t0 + 2 == Nt) ? 0 : t0 + 2;
    float2 pa0, pa1, pb0, pb1;  // own sites t0 (a) and t0 + 1 (b), spins 0, 1
    float2 ca0, ca1, cb0, cb1;  // x + 1
    float2 ga0, ga1, gb0, gb1;  // x - 1
    float2 e0, e1, f0, f1;      // t0 - 1 and t0 + 2
    ld8f(in + 2 * n0, pa0, pa1, pb0, pb1);
    ld8f(in + 2 * (xp * Nt + t0), ca0, ca1, cb0, cb1);
    ld8f(in + 2 * (xm * Nt + t0), ga0, ga1, gb0, gb1);
    ld2(in + 2 * (x * Nt + tm), e0, e1);
    ld2(in + 2 * (x * Nt + tp), f0, f1);
    float2 u0a, u1a, u0b, u1b, w0a, w1a, w0b, w1b;  // links of the pair, and of the pair at x - 1
    ld8f(U + 2 * n0, u0a, u1a, u0b, u1b);
    ld8f(U + 2 * (xm * Nt + t0), w0a, w1a, w0b, w1b);
    const float2 ul0 = __ldg(U + 2 * (x * Nt + tm));
    (void)w0a;
    (void)w0b;
    const float mm = m0 + 2.f;
    float2 oa0, oa1, ob0, ob1;
    // site t0: +t neighbour t0 + 1, -t neighbour t0 - 1 (the t-wrap sign when t0 = 0)
    wilson_site<DAG>(u0a, u1a, ul0, w1a, pa0, pa1, pb0, pb1, ca0, ca1, e0, e1, ga0, ga1, 1.f, t0 == 0 ? -1.f : 1.f,
                     mm, oa0, oa1);
    // site t0 + 1: +t neighbour t0 + 2 (the sign when t0 + 1 = Nt - 1), -t neighbour t0
    wilson_site<DAG>(u0b, u1b, u0a, w1b, pb0, pb1, f0, f1, cb0, cb1, pa0, pa1, gb0, gb1, t0 + 2 == Nt ? -1.f : 1.f,
                     1.f, mm, ob0, ob1);
    if (RESID) {
        float2 b0, b1, b2, b3;
        ld8f(b + ro + 2 * n0, b0, b1, b2, b3);
        oa0 = b0 - oa0;
        oa1 = b1 - oa1;
        ob0 = b2 - ob0;
        ob1 = b3 - ob1;
    }
    st8f(out + 2 * n0, oa0, oa1, ob0, ob1);
}

template <typename V>
void launch_wilson(cudaStream_t s, const V* U, const V* in, V* out, const V* b, int Nx, int Nt, double m0,
                   int dagger, int nrhs) {
    typedef typename RealOf<V>::R R;
    dim3 grid(ceil_div((long)Nx * Nt, 256), nrhs);
    long stride = 2L * Nx * Nt;
    // FP64 sites are 32 bytes: one 256-bit access per site when every field starts on a 32-byte
    // boundary (sites and right-hand sides then stay on one)
    auto a32 = [](const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 31) == 0; };
    const bool wide = sizeof(V) == 16 && a32(U) && a32(in) && a32(out) && a32(b);
    if (sizeof(V) == 8 && Nt % 2 == 0 && a32(U) && a32(in) && a32(out) && a32(b)) {
        // FP32: two sites per thread (t0 even), a pair of sites is 32 bytes
        const float2* Uf = reinterpret_cast<const float2*>(U);
        const float2* inf = reinterpret_cast<const float2*>(in);
        float2* outf = reinterpret_cast<float2*>(out);
        const float2* bf = reinterpret_cast<const float2*>(b);
        dim3 pg(ceil_div((long)Nx * Nt / 2, 256), nrhs);
        if (dagger) {
            if (b) DDAMG_LAUNCH((wilson_pair_kernel<true, true>), pg, 256, 0, s, Uf, inf, outf, bf, Nx, Nt, (float)m0, stride);
            else DDAMG_LAUNCH((wilson_pair_kernel<true, false>), pg, 256, 0, s, Uf, inf, outf, bf, Nx, Nt, (float)m0, stride);
        } else {
            if (b) DDAMG_LAUNCH((wilson_pair_kernel<false, true>), pg, 256, 0, s, Uf, inf, outf, bf, Nx, Nt, (float)m0, stride);
            else DDAMG_LAUNCH((wilson_pair_kernel<false, false>), pg, 256, 0, s, Uf, inf, outf, bf, Nx, Nt, (float)m0, stride);
        }
        return;
    }
    if (wide) {
        if (dagger) {
            if (b) DDAMG_LAUNCH((wilson_kernel<V, true, true, true>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
            else DDAMG_LAUNCH((wilson_kernel<V, true, false, true>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
        } else {
            if (b) DDAMG_LAUNCH((wilson_kernel<V, false, true, true>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
            else DDAMG_LAUNCH((wilson_kernel<V, false, false, true>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
        }
        return;
    }
    if (dagger) {
        if (b) DDAMG_LAUNCH((wilson_kernel<V, true, true>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
        else DDAMG_LAUNCH((wilson_kernel<V, true, false>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
    } else {
        if (b) DDAMG_LAUNCH((wilson_kernel<V, false, true>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
        else DDAMG_LAUNCH((wilson_kernel<V, false, false>), grid, 256, 0, s, U, in, out, b, Nx, Nt, (R)m0, stride);
    }
}
template void launch_wilson<double2>(cudaStream_t, const double2*, const double2*, double2*, const double2*, int, int,
                                     double, int, int);
template void launch_wilson<float2>(cudaStream_t, const float2*, const float2*, float2*, const float2*, int, int,
                                    double, int, int);

// dL/dtheta_mu(n) = -Re[ lam(n)^+ (-1/2)(1-sigma_mu)(i U_mu(n)) s psi(n+mu)
//                      + lam(n+mu)^+ (-1/2)(1+sigma_mu)(-i U*_mu(n)) s psi(n) ]
// the derivative of the two hop terms of D that carry theta_mu(n) (src/dirac_operator.cpp:37-48).
__global__ void link_derivative_kernel(const double2* __restrict__ U, const double2* __restrict__ psi,
                                       const double2* __restrict__ lam, double* __restrict__ out, int Nx, int Nt) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nx * Nt) return;
    const int x = n / Nt, t = n - x * Nt;
    const int r0 = x * Nt + ((t + 1 == Nt) ? 0 : t + 1);
    const int r1 = ((x + 1 == Nx) ? 0 : x + 1) * Nt + t;
    const double sr = (t == Nt - 1) ? -1.0 : 1.0;
    const double2 pn0 = psi[2 * n], pn1 = psi[2 * n + 1];
    const double2 ln0 = lam[2 * n], ln1 = lam[2 * n + 1];
#pragma unroll
    for (int mu = 0; mu < 2; mu++) {
        const int np = mu == 0 ? r0 : r1;
        const double s = mu == 0 ? sr : 1.0;
        const double2 u = U[2 * n + mu];
        const double2 q0 = psi[2 * np], q1 = psi[2 * np + 1];
        const double2 m0 = lam[2 * np], m1 = lam[2 * np + 1];
        double2 h10, h11, h20, h21;  // (1 - sigma) psi(n+mu), (1 + sigma) psi(n)
        if (mu == 0) {
            h10 = q0 - q1;
            h11 = q1 - q0;
            h20 = pn0 + pn1;
            h21 = pn0 + pn1;
        } else {
            h10 = q0 + imul(q1);
            h11 = q1 - imul(q0);
            h20 = pn0 - imul(pn1);
            h21 = pn1 + imul(pn0);
        }
        // term 1: lam(n)^+ (-1/2) (i u) s h1 ; term 2: lam(n+mu)^+ (-1/2) (-i conj u) s h2
        double2 iu = imul(u);
        double2 t1 = cmul(iu, cfmac(ln0, h10, cmulc(ln1, h11)));
        double2 mic = -imul(conjc(u));
        double2 t2 = cmul(mic, cfmac(m0, h20, cmulc(m1, h21)));
        double acc = -0.5 * s * (t1.x + t2.x);
        out[2 * n + mu] = -acc;
    }
}
void launch_link_derivative(cudaStream_t s, const double2* U, const double2* psi, const double2* lam, double* out,
                            int Nx, int Nt) {
    DDAMG_LAUNCH(link_derivative_kernel, ceil_div((long)Nx * Nt, 256), 256, 0, s, U, psi, lam, out, Nx, Nt);
}

// ---------------------------------------------------------------- U(1) Metropolis
// Sweep = 4 sub-sweeps (mu = 0 on even / odd x, mu = 1 on even / odd t); links of one
// sub-sweep share no plaquette, so one thread per link updates a whole sub-sweep at once.
// Same chain as orc_metropolis in the CPU oracle (same counter RNG streams).
__device__ __forceinline__ int wrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }
__device__ __forceinline__ double plaq(const double* th, int Nx, int Nt, int x, int t) {
    int n = x * Nt + t, ntp = x * Nt + wrap(t + 1, Nt), nxp = wrap(x + 1, Nx) * Nt + t;
    return th[2 * n] + th[2 * ntp + 1] - th[2 * nxp] - th[2 * n + 1];
}
__global__ void metropolis_init_kernel(double* th, long n2, uint64_t seed) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n2) return;
    const double pi = 3.14159265358979323846;
    th[i] = -pi + 2.0 * pi * u01(rng64(seed, kStreamHotStart, (uint64_t)i));
}
__global__ void metropolis_sub_kernel(double* th, int Nx, int Nt, double beta, double delta, uint64_t seed,
                                      int sweep, int sub, unsigned long long* acc) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nx * Nt) return;
    const int x = n / Nt, t = n - x * Nt;
    const int mu = sub >> 1, par = sub & 1;
    if (((mu == 0) ? x : t) % 2 != par) return;
    const double pi = 3.14159265358979323846;
    const long li = 2L * n + mu;
    const uint64_t sprop = ((uint64_t)sweep * 4 + sub) * 2 + 1, sacc = sprop + 1;
    const double d = delta * (2.0 * u01(rng64(seed, sprop, (uint64_t)li)) - 1.0);
    double p1, p2, s1, s2;
    if (mu == 0) {
        p1 = plaq(th, Nx, Nt, x, t);
        s1 = 1.0;
        p2 = plaq(th, Nx, Nt, wrap(x - 1, Nx), t);
        s2 = -1.0;
    } else {
        p1 = plaq(th, Nx, Nt, x, t);
        s1 = -1.0;
        p2 = plaq(th, Nx, Nt, x, wrap(t - 1, Nt));
        s2 = 1.0;
    }
    const double dS = -beta * (cos(p1 + s1 * d) + cos(p2 + s2 * d) - cos(p1) - cos(p2));
    const double u = u01(rng64(seed, sacc, (uint64_t)li));
    if (dS <= 0.0 || u < exp(-dS)) {
        double v = th[li] + d;
        if (v >= pi) v -= 2.0 * pi;
        if (v < -pi) v += 2.0 * pi;
        th[li] = v;
        atomicAdd(acc, 1ull);
    }
}
void launch_metropolis_init(cudaStream_t s, double* th, int Nx, int Nt, uint64_t seed) {
    long n2 = 2L * Nx * Nt;
    DDAMG_LAUNCH(metropolis_init_kernel, ceil_div(n2, 256), 256, 0, s, th, n2, seed);
}
void launch_metropolis_sub(cudaStream_t s, double* th, int Nx, int Nt, double beta, double delta, uint64_t seed,
                           int sweep, int sub, unsigned long long* acc) {
    DDAMG_LAUNCH(metropolis_sub_kernel, ceil_div((long)Nx * Nt, 256), 256, 0, s, th, Nx, Nt, beta, delta, seed, sweep,
                 sub, acc);
}
__global__ void theta_to_links_kernel(const double* th, double2* U, long n) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sn, cs;
    sincos(th[i], &sn, &cs);
    U[i] = make_double2(cs, sn);
}
void launch_theta_to_links(cudaStream_t s, const double* th, double2* U, long n) {
    DDAMG_LAUNCH(theta_to_links_kernel, ceil_div(n, 256), 256, 0, s, th, U, n);
}

// test-vector draws, re/im ~ U(-1, 1): complex k uses counters 2k and 2k+1 (orc_uniform)
__global__ void fill_uniform_kernel(double2* out, long n, uint64_t seed, long off) {
    long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint64_t c = 2 * (uint64_t)(off + k);
    out[k] = make_double2(-1.0 + 2.0 * u01(rng64(seed, kStreamUniform, c)),
                          -1.0 + 2.0 * u01(rng64(seed, kStreamUniform, c + 1)));
}
void launch_fill_uniform(cudaStream_t s, double2* out, long n, uint64_t seed, long off) {
    if (n <= 0) return;
    DDAMG_LAUNCH(fill_uniform_kernel, ceil_div(n, 256), 256, 0, s, out, n, seed, off);
}

template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ in, B* __restrict__ out, long n) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = from_d<B>(to_d(in[i]));
}
template <typename A, typename B> void launch_convert(cudaStream_t s, const A* in, B* out, long n) {
    if (n <= 0) return;
    DDAMG_LAUNCH((convert_kernel<A, B>), ceil_div(n, 256), 256, 0, s, in, out, n);
}
template void launch_convert<double2, float2>(cudaStream_t, const double2*, float2*, long);
template void launch_convert<float2, double2>(cudaStream_t, const float2*, double2*, long);
template void launch_convert<double2, double2>(cudaStream_t, const double2*, double2*, long);
template void launch_convert<float2, float2>(cudaStream_t, const float2*, float2*, long);

}  // namespace ddamg
