// Fine-level kernels: Wilson-Dirac stencil D_W / D_W^dagger on U(1) links, the link
// derivative of L = Re(eta^dagger D^-1 b), the U(1) Metropolis generator and field fills.
#include <atomic>

#include "internal.h"
#include "tc_sm100.cuh"

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

// D_W with staged tiles: a persistent CTA walks over tiles of TX x-rows by TT t-sites (and right-hand
// sides), and for each tile one thread brings the tile's psi with its one-site halo and the links it
// needs into shared memory with 1-D bulk asynchronous copies (TMA, cp.async.bulk; one copy per row
// segment, the periodic wrap as separate one-site copies), two stages deep, completion counted on an
// mbarrier.  The 256 threads then read every operand from shared memory: each psi value crosses L2
// once per tile instead of five times.  Same arithmetic as wilson_kernel.
constexpr int kStageThreads = 256;
template <typename V> struct SiteStore;
template <> struct SiteStore<double2> {
    static __device__ __forceinline__ void ld(const double2* p, double2& a, double2& b) { ld2w(p, a, b); }
    static __device__ __forceinline__ void st(double2* p, double2 a, double2 b) { st2w(p, a, b); }
};
template <> struct SiteStore<float2> {
    static __device__ __forceinline__ void ld(const float2* p, float2& a, float2& b) { ld2(p, a, b); }
    static __device__ __forceinline__ void st(float2* p, float2 a, float2 b) { st2(p, a, b); }
};
template <typename V, int TX, int TT>
struct StageGeom {
    static constexpr int S = 2 * sizeof(V);  // bytes per site: two complex numbers (psi spins, or U_0 U_1)
    static constexpr int psi_bytes = (TX + 2) * (TT + 2) * S;
    static constexpr int u_bytes = (TX + 1) * (TT + 1) * S;
    static constexpr int stage_bytes = ((psi_bytes + u_bytes) + 127) / 128 * 128;
    static constexpr int smem = 128 + 2 * stage_bytes;
};
// one thread: the copies of tile `tile` into the stage at `dst`, counted on *bar
template <typename V, int TX, int TT>
__device__ __forceinline__ void stage_issue(const V* U, const V* in, long stride, int Nx, int Nt, int R, int tile,
                                            unsigned char* dst, uint64_t* bar) {
    typedef StageGeom<V, TX, TT> G;
    const int r = tile % R, tt = (tile / R) % (Nt / TT), tx = tile / R / (Nt / TT);
    const int x0 = tx * TX, t0 = tt * TT;
    tc::mbar_arrive_expect_tx(bar, G::psi_bytes + G::u_bytes);
    const unsigned char* pin = reinterpret_cast<const unsigned char*>(in + r * stride);
    const unsigned char* pu = reinterpret_cast<const unsigned char*>(U);
    const long row = (long)Nt * G::S;
    const int tl = t0 == 0 ? Nt - 1 : t0 - 1, tr = t0 + TT == Nt ? 0 : t0 + TT;
    for (int i = 0; i < TX + 2; i++) {  // psi rows x0 - 1 .. x0 + TX, sites t0 - 1 .. t0 + TT
        int x = x0 - 1 + i;
        x = x < 0 ? x + Nx : (x >= Nx ? x - Nx : x);
        const unsigned char* src = pin + x * row;
        unsigned char* d = dst + i * (TT + 2) * G::S;
        if (t0 > 0 && t0 + TT < Nt) {
            tc::bulk_g2s(d, src + (long)(t0 - 1) * G::S, (TT + 2) * G::S, bar);
        } else {
            tc::bulk_g2s(d, src + (long)tl * G::S, G::S, bar);
            tc::bulk_g2s(d + G::S, src + (long)t0 * G::S, TT * G::S, bar);
            tc::bulk_g2s(d + (TT + 1) * G::S, src + (long)tr * G::S, G::S, bar);
        }
    }
    unsigned char* du = dst + G::psi_bytes;
    for (int i = 0; i < TX + 1; i++) {  // link rows x0 - 1 .. x0 + TX - 1, sites t0 - 1 .. t0 + TT - 1
        int x = x0 - 1 + i;
        x = x < 0 ? x + Nx : x;
        const unsigned char* src = pu + x * row;
        unsigned char* d = du + i * (TT + 1) * G::S;
        if (t0 > 0) {
            tc::bulk_g2s(d, src + (long)(t0 - 1) * G::S, (TT + 1) * G::S, bar);
        } else {
            tc::bulk_g2s(d, src + (long)tl * G::S, G::S, bar);
            tc::bulk_g2s(d + G::S, src + (long)t0 * G::S, TT * G::S, bar);
        }
    }
}
template <typename V, bool DAG, bool RESID, int TX, int TT>
__global__ void __launch_bounds__(kStageThreads) wilson_stage_kernel(const V* __restrict__ U, const V* __restrict__ in,
                                                                     V* __restrict__ out, const V* __restrict__ b,
                                                                     int Nx, int Nt, typename RealOf<V>::R m0,
                                                                     long stride, int R, int* status) {
    typedef typename RealOf<V>::R Rl;
    typedef StageGeom<V, TX, TT> G;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    unsigned char* stage = smem + 128;
    const int ntiles = (Nx / TX) * (Nt / TT) * R;
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 2; q++) {
            const int tile = blockIdx.x + q * gridDim.x;
            if (tile < ntiles)
                stage_issue<V, TX, TT>(U, in, stride, Nx, Nt, R, tile, stage + q * G::stage_bytes, &full[q]);
        }
    }
    const Rl mm = m0 + Rl(2), h = Rl(0.5);
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int st = it & 1;
        const bool ok = tc::mbar_wait(&full[st], (it >> 1) & 1, status);
        if (__syncthreads_or(!ok)) break;  // a copy never arrived: the status word says so
        const V* P = reinterpret_cast<const V*>(stage + st * G::stage_bytes);
        const V* Us = reinterpret_cast<const V*>(stage + st * G::stage_bytes + G::psi_bytes);
        const int r = tile % R, tt = (tile / R) % (Nt / TT), tx = tile / R / (Nt / TT);
        const int x0 = tx * TX, t0 = tt * TT;
        for (int q = threadIdx.x; q < TX * TT; q += kStageThreads) {
            const int i = q / TT, t = q - i * TT;
            const V* own = P + 2 * ((i + 1) * (TT + 2) + t + 1);
            const V p0 = own[0], p1 = own[1];
            const V a0 = own[2], a1 = own[3];                                     // +t
            const V e0 = own[-2], e1 = own[-1];                                   // -t
            const V c0 = own[2 * (TT + 2)], c1 = own[2 * (TT + 2) + 1];           // +x
            const V g0 = own[-2 * (TT + 2)], g1 = own[-2 * (TT + 2) + 1];         // -x
            const V* uo = Us + 2 * ((i + 1) * (TT + 1) + t + 1);
            const V u0 = uo[0], u1 = uo[1];
            const V ul0 = uo[-2];                                                 // U_0(x, t - 1)
            const V ul1 = uo[-2 * (TT + 1) + 1];                                  // U_1(x - 1, t)
            const int tg = t0 + t;
            const Rl sr = (tg == Nt - 1) ? Rl(-1) : Rl(1), sl = (tg == 0) ? Rl(-1) : Rl(1);
            V s0, s1;
            if (!DAG) {
                V a = sr * cmul(u0, a0 - a1);
                V c = cmul(u1, c0 + imul(c1));
                V e = sl * cmulc(ul0, e0 + e1);
                V g = cmulc(ul1, g0 - imul(g1));
                s0 = a + c + e + g;
                s1 = -a - imul(c) + e + imul(g);
            } else {
                V a = sl * cmulc(ul0, e0 - e1);
                V c = cmulc(ul1, g0 + imul(g1));
                V e = sr * cmul(u0, a0 + a1);
                V g = cmul(u1, c0 - imul(c1));
                s0 = a + c + e + g;
                s1 = -a - imul(c) + e + imul(g);
            }
            V o0 = mm * p0 - h * s0;
            V o1 = mm * p1 - h * s1;
            const long site = (long)(x0 + i) * Nt + tg;
            if (RESID) {
                V b0, b1;
                SiteStore<V>::ld(b + r * stride + 2 * site, b0, b1);
                o0 = b0 - o0;
                o1 = b1 - o1;
            }
            SiteStore<V>::st(out + r * stride + 2 * site, o0, o1);
        }
        __syncthreads();  // every thread is done with this stage
        if (threadIdx.x == 0 && tile + 2 * gridDim.x < ntiles)
            stage_issue<V, TX, TT>(U, in, stride, Nx, Nt, R, tile + 2 * gridDim.x, stage + st * G::stage_bytes,
                                   &full[st]);
    }
}

// which D_W kernel launch_wilson uses: 0 the default, 1 the register kernels (wilson_kernel /
// wilson_pair_kernel), 2 the staged-tile kernel where the lattice divides into its tiles
static std::atomic<int> g_stencil_variant{0};
static int* stencil_status();
void set_stencil_variant(int v) {
    stencil_status();  // allocated here, outside any stream capture
    g_stencil_variant = v;
}
int stencil_variant() { return g_stencil_variant; }
static int* stencil_status() {  // bounded-wait status word of the staged kernel, one per device
    static int* p[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!p[dev]) {
        DDAMG_CUDA_TRY(cudaMalloc(&p[dev], sizeof(int)));
        DDAMG_CUDA_TRY(cudaMemset(p[dev], 0, sizeof(int)));
    }
    return p[dev];
}
int stencil_status_read() {
    int v = 0;
    DDAMG_CUDA_TRY(cudaMemcpy(&v, stencil_status(), sizeof(int), cudaMemcpyDeviceToHost));
    return v;
}
template <typename V, int TX, int TT>
static bool launch_wilson_staged(cudaStream_t s, const V* U, const V* in, V* out, const V* b, int Nx, int Nt,
                                 double m0, int dagger, int nrhs) {
    typedef typename RealOf<V>::R R;
    typedef StageGeom<V, TX, TT> G;
    auto a = [](const void* p, int al) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) % al) == 0; };
    const int al = sizeof(V) == 16 ? 32 : 16;  // the site stores and loads of the epilogue
    if (Nx % TX || Nt % TT || Nx < 2 || !a(U, al) || !a(in, al) || !a(out, al) || !a(b, al)) return false;
    static int ctas_per_sm[2][2][2] = {};
    static int sms = 0;
    if (!sms) DDAMG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    const long stride = 2L * Nx * Nt;
    const int ntiles = (Nx / TX) * (Nt / TT) * nrhs;
    int* status = stencil_status();
    auto go = [&](auto kern, int& cps) {
        if (!cps) {
            DDAMG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::smem));
            DDAMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, kern, kStageThreads, G::smem));
            if (cps < 1) cps = 1;
        }
        const int grid = (int)std::min<long>(ntiles, (long)sms * cps);
        DDAMG_LAUNCH(kern, grid, kStageThreads, G::smem, s, U, in, out, b, Nx, Nt, (R)m0, stride, nrhs, status);
    };
    if (dagger) {
        if (b) go(wilson_stage_kernel<V, true, true, TX, TT>, ctas_per_sm[1][1][sizeof(V) == 16]);
        else go(wilson_stage_kernel<V, true, false, TX, TT>, ctas_per_sm[1][0][sizeof(V) == 16]);
    } else {
        if (b) go(wilson_stage_kernel<V, false, true, TX, TT>, ctas_per_sm[0][1][sizeof(V) == 16]);
        else go(wilson_stage_kernel<V, false, false, TX, TT>, ctas_per_sm[0][0][sizeof(V) == 16]);
    }
    return true;
}

template <typename V>
void launch_wilson(cudaStream_t s, const V* U, const V* in, V* out, const V* b, int Nx, int Nt, double m0,
                   int dagger, int nrhs) {
    typedef typename RealOf<V>::R R;
    if (g_stencil_variant == 2 && launch_wilson_staged<V, 8, 64>(s, U, in, out, b, Nx, Nt, m0, dagger, nrhs)) return;
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
