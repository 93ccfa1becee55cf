// Batched coarse-level SAP colour sweep with the block operator on tcgen05 tensor cores.
//
// A colour sweep solves, for every Schwarz block B of the colour and every right-hand side r,
// D_B e = r_B by GMRES(m) x restarts with x0 = r_B (SAP_C::SAP, src/sap.cpp:48-77,104-139;
// FGMRES::fgmres, src/fgmres.cpp:5-98).  With R right-hand sides in lockstep the operator
// application of one block is, per site s and hop d, the contraction of a dof x dof complex link
// with a dof x R block of vectors: in the real embedding a GEMM with M = 2 dof, K = 2 dof, N = R.
//
//   tc_block_apply_kernel   one CTA per (block, group of RG right-hand sides):
//                           w = D_B v (or b - D_B v) on tensor cores.  The embedded link tiles
//                           (one per site and hop, packed once after the setup) arrive by bulk
//                           copy; the vector tiles of the block's sites arrive by TMA straight from
//                           the interleaved block vectors into a shared-memory window holding sites
//                           s - sel_t .. s + sel_t + 1, so every vector tile is read once per
//                           application; the accumulators live in tensor memory, two buffers so
//                           the epilogue of site s overlaps the MMAs of site s + 1.
//   tcs_* kernels           one warp per (block, right-hand side): Gram-Schmidt, Givens rotations,
//                           restarts, and the gather / scatter between the level vectors and the
//                           block vectors, with the same per-rhs control flow (break point maxIt,
//                           convergence freeze) as the on-chip solver in kernels_sap.cu.
//
// Warp roles of the apply kernel: EW = 8 or 16 epilogue warps (warp w reads tensor-memory lanes
// 32 (w % 4) .. +31 and a quarter of the columns), then one warp whose lane 0 issues the copies
// and one whose lane 0 issues the MMAs.  Every mbarrier wait is
// bounded; a wait that gives up sets the status word and the CTA winds down.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "internal.h"
#include "tc_sm100.cuh"

namespace ddamg {

using namespace tc;

namespace {
// epilogue warps (16 for groups of >= 32 right-hand sides, else 8), plus one copy warp and one MMA
// warp
__host__ __device__ constexpr int epi_warps(int RG) { return RG >= 32 ? 16 : 8; }
__host__ __device__ constexpr int apply_threads(int RG) { return (epi_warps(RG) + 2) * 32; }
constexpr uint32_t kTileBytes = kTcTileFloats * 4;  // 64 rows x 64 fp32

constexpr int kMaxBlockSites = 256;  // sites per Schwarz block the apply kernel's tables hold
__host__ __device__ inline int release_lag(int sel_t) { return sel_t > 2 ? sel_t : 2; }
__host__ __device__ inline int window_slots(int sel_t) { return sel_t + release_lag(sel_t) + 2; }
inline size_t apply_smem(int RG, int NA, int sel_t) {
    const int nw = window_slots(sel_t);
    return 1024 + (size_t)NA * kTileBytes + (size_t)nw * 256 * RG + sizeof(uint64_t) * (2 * NA + 2 * nw + 5);
}
// tile shapes of the apply kernel the autotuner chooses from: right-hand sides per CTA and depth of
// the link-tile ring
struct TcShape {
    int rg, na, nch;  // right-hand sides per CTA, link-tile ring depth, accumulator chains per site
};
constexpr TcShape kShapes[] = {{64, 3, 1}, {64, 3, 2}, {64, 3, 4}, {32, 8, 2}, {32, 8, 4}, {16, 8, 4}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);
// dynamic shared memory plus the kernel's static tables (under 5 KB) within the 227 KB per CTA
inline bool shape_fits(int idx, int sel_t) {
    return apply_smem(kShapes[idx].rg, kShapes[idx].na, sel_t) + 5 * 1024 <= 227 * 1024 &&
           2 * kShapes[idx].nch * kShapes[idx].rg <= 512;
}
// without a tuning result: the widest shape that fits, its width rounded up from the batch
inline int default_shape(int nrhs, int sel_t) {
    for (int i = 0; i < kNumShapes; i++)
        if (shape_fits(i, sel_t) && (kShapes[i].rg / 2 < nrhs || kShapes[i].rg == 16)) return i;
    return kNumShapes - 1;
}

struct ApplyArgs {
    const float* tiles;  // operator tiles (site, hop)
    float2* dst;
    const float2* bsub;  // non-null: dst = bsub - D_B src
    const int* flag;     // per (kb, r): the rhs takes part when (flag != 0) != invert
    int invert;
    const int* blocks;
    int R, S, sel_x, sel_t, Nt, sap_t, dof;
    int ks;  // MMA K steps of 8: ceil(2 dof / 8)
    float mm;  // m0 + 2
    int* status;
};
}  // namespace

bool tc_sap_supported(const Geom& g) {
    const int S = g.sel_x * g.sel_t;
    return g.level >= 1 && g.dof <= 32 && S * g.dof <= 1024 && S <= kMaxBlockSites &&
           apply_smem(16, 4, g.sel_t) + 5 * 1024 <= 227 * 1024;
}

// Operator tile (n, d): the real 2dof x 2dof embedding of T = -s_d M_d, M_d the coarse link of hop
// d at site n and s_d the antiperiodic sign of a hop across the t boundary (the mass term of d = 0
// is added in FP32 by the epilogue):  rows m = 2i + p (p: real / imaginary part of output dof i),
// columns k = 2j + q (q: real / imaginary part of input dof j),
//     [Re T_ij  -Im T_ij]
//     [Im T_ij   Re T_ij],
// zero outside i, j < dof; 64 x 64 fp32 stored as two K-major 128B-swizzled 64 x 32 blocks (the
// shared-memory image, so one bulk copy lands it ready for tcgen05.mma).  A vector stored as
// interleaved (re, im) pairs is then the K-major B operand as it lies in memory.
__global__ void pack_tc_links_kernel(const float2* __restrict__ L, float* __restrict__ tiles, int Nt, int dof) {
    const long tile = blockIdx.x;
    const int n = (int)(tile / 5), d = (int)(tile - (long)n * 5);
    const int t = n % Nt;
    const float sg = ((d == 1 && t == Nt - 1) || (d == 3 && t == 0)) ? -1.f : 1.f;
    const float2* M = L + tile * dof * dof;
    char* base = reinterpret_cast<char*>(tiles + tile * kTcTileFloats);
    for (int e = threadIdx.x; e < kTcTileFloats; e += blockDim.x) {
        const int m = e >> 6, k = e & 63, i = m >> 1, p = m & 1, j = k >> 1, q = k & 1;
        float v = 0.f;
        if (i < dof && j < dof) {
            const float2 l = M[(long)j * dof + i];
            const float re = -sg * l.x, im = -sg * l.y;
            v = (p == q) ? re : (p ? im : -im);
        }
        *reinterpret_cast<float*>(base + (k >> 5) * 8192 + swz_off(m, k & 31)) = v;
    }
}

void launch_pack_tc_links(cudaStream_t s, const Geom& g, const float2* links, float* tiles) {
    DDAMG_LAUNCH(pack_tc_links_kernel, (long)g.sites * 5, 256, 0, s, links, tiles, g.Nt, g.dof);
}

// slow path of a barrier wait (kept out of line so the hot loops stay short): bounded, sets *abort
__device__ __noinline__ bool wait_slow(uint64_t* bar, uint32_t parity, int* status, volatile int* abort) {
    if (*abort) return false;
    if (mbar_wait(bar, parity, status)) return true;
    *abort = 1;
    return false;
}

// w = D_B src (or bsub - D_B src) for one block and RG right-hand sides.  src enters through the
// tensor map vmap: dims (2 dof floats, S sites, NB*R block-rhs rows), box (32, 1, RG), 128B swizzle,
// so a box lands as RG rows of 32 fp32 -- one K-major 128B-swizzled operand block.
// Warps 0 .. EW-1 run the epilogue, warp EW issues the copies, warp EW+1 the MMAs (one thread
// each); the control loops use tables built once per CTA (no divisions) and descriptor arithmetic
// by addition, since a single thread's instruction latency is what bounds them.
template <int RG, int NA, int NCH>
__global__ void __launch_bounds__(apply_threads(RG), 1)
    tc_block_apply_kernel(const __grid_constant__ CUtensorMap vmap, ApplyArgs a) {
    constexpr int EW = epi_warps(RG);
    constexpr int CW = 4 * RG / EW;  // accumulator columns per epilogue warp: 16 or 8
    constexpr uint32_t kBBytes = RG * 256;  // two 128-byte column blocks of RG rows
    extern __shared__ unsigned char smraw[];
    __shared__ int s_any;
    __shared__ volatile int s_abort;
    __shared__ uint32_t s_taddr;
    __shared__ short s_nb[kMaxBlockSites][5];         // neighbour site in the block, -1 outside
    __shared__ int s_gsite[kMaxBlockSites];           // lattice site
    __shared__ unsigned char s_slot[kMaxBlockSites];  // window slot of a site's vector tile
    __shared__ unsigned char s_par[kMaxBlockSites];   // fill parity of that slot
    unsigned char* sm =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    const int kb = blockIdx.x, r0 = blockIdx.y * RG;
    const int nr = min(RG, a.R - r0);
    const int S = a.S, NW = window_slots(a.sel_t), RL = release_lag(a.sel_t);
    const int katoms = (a.ks + 3) >> 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        s_any = 0;
        s_abort = 0;
    }
    __syncthreads();
    if (threadIdx.x < nr && ((a.flag[(long)kb * a.R + r0 + threadIdx.x] != 0) != (a.invert != 0))) s_any = 1;
    __syncthreads();
    if (!s_any) return;

    unsigned char* Abuf = sm;
    unsigned char* Bbuf = sm + NA * kTileBytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bbuf + (size_t)NW * kBBytes);
    uint64_t* fullA = bar;
    uint64_t* emptyA = bar + NA;
    uint64_t* fullB = bar + 2 * NA;
    uint64_t* emptyB = fullB + NW;
    uint64_t* accF = emptyB + NW;
    uint64_t* accE = accF + 2;
    uint64_t* drain = accE + 2;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NA; i++) {
            mbar_init(&fullA[i], 1);
            mbar_init(&emptyA[i], 1);
        }
        for (int i = 0; i < NW; i++) {
            mbar_init(&fullB[i], 1);
            mbar_init(&emptyB[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&accF[i], 1);
            mbar_init(&accE[i], EW);
        }
        mbar_init(drain, 1);
        mbar_fence_init();
    }
    {
        const int blk = a.blocks[kb];
        const int bx = blk / a.sap_t, bt = blk - bx * a.sap_t;
        for (int s = threadIdx.x; s < S; s += blockDim.x) {
            const int kx = s / a.sel_t, kt = s - kx * a.sel_t;
            s_nb[s][0] = (short)s;
            s_nb[s][1] = (short)(kt + 1 < a.sel_t ? s + 1 : -1);
            s_nb[s][2] = (short)(kx + 1 < a.sel_x ? s + a.sel_t : -1);
            s_nb[s][3] = (short)(kt > 0 ? s - 1 : -1);
            s_nb[s][4] = (short)(kx > 0 ? s - a.sel_t : -1);
            s_gsite[s] = (bx * a.sel_x + kx) * a.Nt + bt * a.sel_t + kt;
            s_slot[s] = (unsigned char)(s % NW);
            s_par[s] = (unsigned char)((s / NW) & 1);
        }
    }
    if (warp == 0) {
        tmem_alloc(&s_taddr, 2 * NCH * RG);
        tmem_relinquish();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = s_taddr;
    auto wait = [&](uint64_t* b, uint32_t parity) -> bool {
        return mbar_try_wait(b, parity) || wait_slow(b, parity, a.status, &s_abort);
    };

    if (warp == EW) {
        // ---------------- producer (one thread): vector tiles by TMA, link tiles by bulk copy
        if (lane == 0) {
            int stage = 0, lap = 0, a_issued = 0, t_next = 0;
            bool ok = true;
            for (int s = 0; s < S && ok; s++) {
                const int tmax = min(S - 1, s + a.sel_t + 1);
                for (; t_next <= tmax; t_next++) {
                    const int slot = s_slot[t_next];
                    if (t_next >= NW && !(ok = wait(&emptyB[slot], s_par[t_next] ^ 1u))) break;
                    unsigned char* tb = Bbuf + (size_t)slot * kBBytes;
                    mbar_arrive_expect_tx(&fullB[slot], (uint32_t)katoms * RG * 128);
                    for (int at = 0; at < katoms; at++)
                        tma_load_3d(tb + at * RG * 128, &vmap, 32 * at, t_next, kb * a.R + r0, &fullB[slot]);
                }
                if (!ok) break;
                const float* tsite = a.tiles + (long)s_gsite[s] * 5 * kTcTileFloats;
                for (int d = 0; d < 5; d++) {
                    if (s_nb[s][d] < 0) continue;
                    if (lap > 0 && !(ok = wait(&emptyA[stage], (uint32_t)(lap - 1) & 1u))) break;
                    mbar_arrive_expect_tx(&fullA[stage], kTileBytes);
                    bulk_g2s(Abuf + (size_t)stage * kTileBytes, tsite + d * kTcTileFloats, kTileBytes, &fullA[stage]);
                    a_issued++;
                    if (++stage == NA) {
                        stage = 0;
                        lap++;
                    }
                }
            }
            // every copy issued has landed before the CTA may exit
            for (int st = 0; st < NA; st++) {
                const int issued = a_issued > st ? (a_issued - 1 - st) / NA + 1 : 0;
                if (issued > 0) mbar_wait(&fullA[st], (issued - 1) & 1, a.status);
            }
            for (int sl = 0; sl < NW; sl++) {
                const int issued = t_next > sl ? (t_next - 1 - sl) / NW + 1 : 0;
                if (issued > 0) mbar_wait(&fullB[sl], (issued - 1) & 1, a.status);
            }
        }
    } else if (warp == EW + 1) {
        // ---------------- MMA issuer (one thread)
        if (lane == 0) {
            const uint32_t idesc = idesc_tf32(64, RG);
            const uint64_t ad0 = sdesc_k128(smem_u32(Abuf)), bd0 = sdesc_k128(smem_u32(Bbuf));
            int stage = 0;
            uint32_t phA = 0;
            const int ks = a.ks;
            for (int s = 0; s < S; s++) {
                const int b = s & 1;
                if (s >= 2 && !wait(&accE[b], (uint32_t)((s >> 1) - 1) & 1u)) break;
                tc_fence_after();
                // K step k of every hop accumulates into chain k % NCH: consecutive MMAs are
                // independent, so the tensor pipe overlaps them instead of serialising one chain
                const uint32_t dt = taddr + (uint32_t)(b * NCH * RG);
                bool first = true, ok = true;
                for (int d = 0; d < 5; d++) {
                    const int nb = s_nb[s][d];
                    if (nb < 0) continue;
                    const int slot = s_slot[nb];
                    if (!wait(&fullB[slot], s_par[nb]) || !wait(&fullA[stage], phA)) {
                        ok = false;
                        break;
                    }
                    const uint64_t ad = ad0 + (uint64_t)(stage * (kTileBytes >> 4));
                    const uint64_t bd = bd0 + (uint64_t)(slot * (kBBytes >> 4));
#pragma unroll
                    for (int k = 0; k < 8; k++) {  // K steps of 8 fp32 = 32 bytes within a 128-byte block
                        if (k >= ks) break;
                        mma_tf32(dt + (uint32_t)((k % NCH) * RG), ad + (uint64_t)((k >> 2) * (8192 >> 4) + (k & 3) * 2),
                                 bd + (uint64_t)((k >> 2) * (RG * 128 >> 4) + (k & 3) * 2), idesc,
                                 (first && k < NCH) ? 0u : 1u);
                    }
                    first = false;
                    mma_commit(&emptyA[stage]);
                    if (++stage == NA) {
                        stage = 0;
                        phA ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(&accF[b]);
                // site s is the last to read vector tile s - sel_t; the epilogue of site s - RL
                // (which reads that site's own tile) has finished before site s could start
                if (s >= RL) mma_commit(&emptyB[s_slot[s - RL]]);
            }
            mma_commit(drain);  // every MMA of this CTA has finished before TMEM is released
            mbar_wait(drain, 0, a.status);
        }
    } else {
        // ---------------- epilogue: warp w owns accumulator rows 16 q .. 16 q + 15 (lanes 0-15,
        // q = w % 4) and CW columns starting at (w / 4) CW; row m = 2i + p is part p of output
        // dof i for each right-hand side (column)
        const int q = warp & 3;
        const int c0 = (warp >> 2) * CW;
        const int m = 16 * q + (lane & 15);
        const bool rowok = lane < 16 && m < 2 * a.dof;
        const long ostride = (long)S * a.dof * 2;
        // shared-memory offsets of element (row c, column m) of a vector tile, for c % 8 = 0..7
        uint32_t soff[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
            soff[j] = (uint32_t)(m >> 5) * RG * 128 + ((uint32_t)(((m & 31) >> 2) ^ j) << 4) + ((uint32_t)(m & 3) << 2);
        const float mm = a.mm;
        float* __restrict__ dst0 = reinterpret_cast<float*>(a.dst) + ((long)kb * a.R + r0 + c0) * ostride + m;
        const float* __restrict__ b0 =
            a.bsub ? reinterpret_cast<const float*>(a.bsub) + ((long)kb * a.R + r0 + c0) * ostride + m : nullptr;
        const int ncol = min(CW, nr - c0);  // valid columns of this warp (may be <= 0)
        for (int s = 0; s < S; s++) {
            const int b = s & 1;
            // b of this site is loaded before the accumulator is waited for, and the accumulator is
            // released as soon as it is in registers, so no global-memory latency sits between the
            // MMAs of consecutive sites
            const long so = (long)s * a.dof * 2;
            float bv[CW];
#pragma unroll
            for (int c = 0; c < CW; c++) bv[c] = (rowok && b0 && c < ncol) ? b0[so + c * ostride] : 0.f;
            if (!wait(&accF[b], (uint32_t)(s >> 1) & 1u)) break;
            tc_fence_after();
            const uint32_t tb = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * NCH * RG + c0);
            float acc[CW];
            if constexpr (CW == 16) tmem_ld16(tb, acc);
            else tmem_ld8(tb, acc);
#pragma unroll
            for (int ch = 1; ch < NCH; ch++) {
                if (ch >= a.ks) break;
                float part[CW];
                if constexpr (CW == 16) tmem_ld16(tb + ch * RG, part);
                else tmem_ld8(tb + ch * RG, part);
#pragma unroll
                for (int c = 0; c < CW; c++) acc[c] += part[c];
            }
            // the site's own vector from the window before the release: once the accumulator is
            // released the MMA thread may let the producer refill this window slot
            float vv[CW];
            {
                const unsigned char* self = Bbuf + (size_t)s_slot[s] * kBBytes + (size_t)c0 * 128;
#pragma unroll
                for (int c = 0; c < CW; c++)
                    vv[c] = (rowok && c < ncol) ? *reinterpret_cast<const float*>(self + c * 128 + soff[c & 7]) : 0.f;
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&accE[b]);
            if (rowok) {
#pragma unroll
                for (int c = 0; c < CW; c++) {
                    if (c < ncol) {
                        float w = mm * vv[c] + acc[c];
                        if (b0) w = bv[c] - w;
                        dst0[so + c * ostride] = w;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(taddr, 2 * NCH * RG);
    }
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        DDAMG_CUDA_TRY(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw ParamFailure{"cuTensorMapEncodeTiled is unavailable"};
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// block vectors [kb*R + r][s][dof] (interleaved complex) as a 3-D fp32 tensor
static CUtensorMap vector_map(const float2* base, int dof, int S, long rows, int RG) {
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)(2 * dof), (cuuint64_t)S, (cuuint64_t)rows};
    cuuint64_t strides[2] = {(cuuint64_t)(2 * dof * 4), (cuuint64_t)S * 2 * dof * 4};
    cuuint32_t box[3] = {32, 1, (cuuint32_t)RG};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(base), dims,
                                            strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw ParamFailure{"tensor map encoding failed"};
    return m;
}

template <int RG, int NA, int NCH>
static void launch_apply_shape(cudaStream_t s, const CUtensorMap& vmap, const ApplyArgs& a, int NB) {
    const size_t smem = apply_smem(RG, NA, a.sel_t);
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(tc_block_apply_kernel<RG, NA, NCH>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(NB, (a.R + RG - 1) / RG);
    DDAMG_LAUNCH((tc_block_apply_kernel<RG, NA, NCH>), grid, apply_threads(RG), smem, s, vmap, a);
}
static void launch_apply(int shape, cudaStream_t s, const CUtensorMap& vmap, const ApplyArgs& a, int NB) {
    switch (shape) {
        case 0: launch_apply_shape<64, 3, 1>(s, vmap, a, NB); break;
        case 1: launch_apply_shape<64, 3, 2>(s, vmap, a, NB); break;
        case 2: launch_apply_shape<64, 3, 4>(s, vmap, a, NB); break;
        case 3: launch_apply_shape<32, 8, 2>(s, vmap, a, NB); break;
        case 4: launch_apply_shape<32, 8, 4>(s, vmap, a, NB); break;
        default: launch_apply_shape<16, 8, 4>(s, vmap, a, NB); break;
    }
}

// ---------------------------------------------------------------- the level operator on tensor cores
// out = D_c v (or b - D_c v) on the whole level for R right-hand sides (Level::D_operator,
// src/level.cpp:394-426, applied to a batch): per site and hop one M = 64, N = RG, K = 64 TF32 MMA
// chain of the packed operator tile (-s_d M_d, the tiles of the SAP sweeps) with the neighbour's
// vector tile, the five hops accumulating into one tensor-memory accumulator; the epilogue adds the
// mass term (m0 + 2) v in FP32.  One CTA per run of consecutive sites and group of RG right-hand sides:
// one thread streams (link tile, vector tile) pairs into an NA-deep ring (bulk copy + TMA, the periodic
// neighbour computed on the fly), one thread issues the MMAs, the epilogue warps drain kOpAcc
// accumulator buffers.  Every mbarrier wait is bounded as in tc_block_apply_kernel.
struct OpArgs {
    const float* tiles;
    float2* dst;
    const float2* src;   // v, for the mass term
    const float2* bsub;  // non-null: dst = bsub - D_c v
    int Nx, Nt, dof, ks, R, sites, spc;  // spc: sites per CTA
    long n;                              // complex values per vector
    float mm;
    int* status;
};
template <int RG> __host__ __device__ constexpr uint32_t op_stage_bytes() { return kTileBytes + RG * 256; }
constexpr int kOpAcc = 4;  // accumulator buffers in tensor memory: the epilogue of site s overlaps the MMAs of s + 1 .. s + 3
template <int RG, int NA> inline size_t op_smem() {
    return 1024 + (size_t)NA * op_stage_bytes<RG>() + 8 * (2 * NA + 2 * kOpAcc + 1);
}

template <int RG, int NA>
__global__ void __launch_bounds__(apply_threads(RG), 1)
    tc_coarse_op_kernel(const __grid_constant__ CUtensorMap vmap, OpArgs a) {
    constexpr int EW = epi_warps(RG);
    constexpr int CW = 4 * RG / EW;
    constexpr uint32_t SB = op_stage_bytes<RG>();
    extern __shared__ unsigned char smraw[];
    __shared__ volatile int s_abort;
    __shared__ uint32_t s_taddr;
    unsigned char* sm =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    const int sb = blockIdx.x * a.spc, se = min(a.sites, sb + a.spc);
    const int r0 = blockIdx.y * RG, nr = min(RG, a.R - r0);
    const int ns = se - sb;
    const int katoms = (a.ks + 3) >> 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (ns <= 0) return;  // uniform over the CTA
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + (size_t)NA * SB);
    uint64_t* fullS = bar;
    uint64_t* emptyS = bar + NA;
    uint64_t* accF = bar + 2 * NA;
    uint64_t* accE = accF + kOpAcc;
    uint64_t* drain = accE + kOpAcc;
    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int i = 0; i < NA; i++) {
            mbar_init(&fullS[i], 1);
            mbar_init(&emptyS[i], 1);
        }
        for (int i = 0; i < kOpAcc; i++) {
            mbar_init(&accF[i], 1);
            mbar_init(&accE[i], EW);
        }
        mbar_init(drain, 1);
        mbar_fence_init();
    }
    if (warp == 0) {
        tmem_alloc(&s_taddr, kOpAcc * RG);
        tmem_relinquish();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = s_taddr;
    auto wait = [&](uint64_t* b, uint32_t parity) -> bool {
        return mbar_try_wait(b, parity) || wait_slow(b, parity, a.status, &s_abort);
    };
    if (warp == EW) {
        // ---------------- producer: for every (site, hop) the operator tile and the neighbour's vector tile
        if (lane == 0) {
            int issued = 0;
            bool ok = true;
            for (int s = sb; s < se && ok; s++) {
                const int x = s / a.Nt, t = s - x * a.Nt;
                for (int d = 0; d < 5; d++) {
                    int nb;
                    switch (d) {
                        case 0: nb = s; break;
                        case 1: nb = x * a.Nt + (t + 1 == a.Nt ? 0 : t + 1); break;
                        case 2: nb = (x + 1 == a.Nx ? 0 : x + 1) * a.Nt + t; break;
                        case 3: nb = x * a.Nt + (t == 0 ? a.Nt - 1 : t - 1); break;
                        default: nb = (x == 0 ? a.Nx - 1 : x - 1) * a.Nt + t; break;
                    }
                    const int st = issued % NA;
                    if (issued >= NA && !(ok = wait(&emptyS[st], (uint32_t)(issued / NA - 1) & 1u))) break;
                    unsigned char* base = sm + (size_t)st * SB;
                    mbar_arrive_expect_tx(&fullS[st], kTileBytes + (uint32_t)katoms * RG * 128);
                    bulk_g2s(base, a.tiles + ((long)s * 5 + d) * kTcTileFloats, kTileBytes, &fullS[st]);
                    for (int at = 0; at < katoms; at++)
                        tma_load_3d(base + kTileBytes + at * RG * 128, &vmap, 32 * at, nb, r0, &fullS[st]);
                    issued++;
                }
            }
            for (int st = 0; st < NA; st++) {  // every copy issued has landed before the CTA may exit
                const int cnt = issued > st ? (issued - 1 - st) / NA + 1 : 0;
                if (cnt > 0) mbar_wait(&fullS[st], (uint32_t)(cnt - 1) & 1u, a.status);
            }
        }
    } else if (warp == EW + 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = idesc_tf32(64, RG);
            const uint64_t sd0 = sdesc_k128(smem_u32(sm));
            int consumed = 0;
            bool ok = true;
            for (int sl = 0; sl < ns && ok; sl++) {
                const int b = sl % kOpAcc;
                if (sl >= kOpAcc && !wait(&accE[b], (uint32_t)(sl / kOpAcc - 1) & 1u)) break;
                tc_fence_after();
                const uint32_t dt = taddr + (uint32_t)(b * RG);
                for (int d = 0; d < 5; d++) {
                    const int st = consumed % NA;
                    if (!(ok = wait(&fullS[st], (uint32_t)(consumed / NA) & 1u))) break;
                    const uint64_t ad = sd0 + (uint64_t)(st * (SB >> 4));
                    const uint64_t bd = ad + (uint64_t)(kTileBytes >> 4);
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        if (k >= a.ks) break;
                        mma_tf32(dt, ad + (uint64_t)((k >> 2) * (8192 >> 4) + (k & 3) * 2),
                                 bd + (uint64_t)((k >> 2) * (RG * 128 >> 4) + (k & 3) * 2), idesc,
                                 (d == 0 && k == 0) ? 0u : 1u);
                    }
                    mma_commit(&emptyS[st]);
                    consumed++;
                }
                if (!ok) break;
                mma_commit(&accF[b]);
            }
            mma_commit(drain);  // every MMA of this CTA has finished before TMEM is released
            mbar_wait(drain, 0, a.status);
        }
    } else {
        // ---------------- epilogue (the accumulator layout of tc_block_apply_kernel)
        const int q = warp & 3;
        const int c0 = (warp >> 2) * CW;
        const int m = 16 * q + (lane & 15);
        const bool rowok = lane < 16 && m < 2 * a.dof;
        const long ostride = a.n * 2;  // floats between right-hand sides
        const int ncol = min(CW, nr - c0);
        const float* __restrict__ v0 = reinterpret_cast<const float*>(a.src) + (long)(r0 + c0) * ostride + m;
        float* __restrict__ d0 = reinterpret_cast<float*>(a.dst) + (long)(r0 + c0) * ostride + m;
        const float* __restrict__ b0 =
            a.bsub ? reinterpret_cast<const float*>(a.bsub) + (long)(r0 + c0) * ostride + m : nullptr;
        for (int sl = 0; sl < ns; sl++) {
            const int b = sl % kOpAcc;
            // the site's own vector (mass term) and b are loaded before the accumulator is waited for
            const long so = (long)(sb + sl) * a.dof * 2;
            float vv[CW], bv[CW];
#pragma unroll
            for (int c = 0; c < CW; c++) {
                const bool ok = rowok && c < ncol;
                vv[c] = ok ? v0[so + c * ostride] : 0.f;
                bv[c] = (ok && b0) ? b0[so + c * ostride] : 0.f;
            }
            if (!wait(&accF[b], (uint32_t)(sl / kOpAcc) & 1u)) break;
            tc_fence_after();
            const uint32_t tb = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * RG + c0);
            float acc[CW];
            if constexpr (CW == 16) tmem_ld16(tb, acc);
            else tmem_ld8(tb, acc);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&accE[b]);
            if (rowok) {
#pragma unroll
                for (int c = 0; c < CW; c++) {
                    if (c < ncol) {
                        float w = a.mm * vv[c] + acc[c];
                        if (b0) w = bv[c] - w;
                        d0[so + c * ostride] = w;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(taddr, kOpAcc * RG);
    }
}

template <int RG, int NA>
static void launch_op_shape(cudaStream_t s, const Geom& g, const float* tiles, const float2* in, float2* out,
                            const float2* b, double m0, int nrhs, int* status) {
    const size_t smem = op_smem<RG, NA>();
    DDAMG_CUDA_TRY(cudaFuncSetAttribute(tc_coarse_op_kernel<RG, NA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    int sms = 0, dev = 0;
    DDAMG_CUDA_TRY(cudaGetDevice(&dev));
    DDAMG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int groups = (nrhs + RG - 1) / RG;
    // one CTA per SM over all (site run, rhs group) pairs: runs of consecutive sites
    const int runs = std::max(1, std::min(g.sites, sms / std::min(groups, sms)));
    OpArgs a;
    a.tiles = tiles;
    a.dst = out;
    a.src = in;
    a.bsub = b;
    a.Nx = g.Nx;
    a.Nt = g.Nt;
    a.dof = g.dof;
    a.ks = (2 * g.dof + 7) / 8;
    a.R = nrhs;
    a.sites = g.sites;
    a.spc = (g.sites + runs - 1) / runs;
    a.n = g.size();
    a.mm = (float)(m0 + 2.0);
    a.status = status;
    const CUtensorMap vmap = vector_map(in, g.dof, g.sites, nrhs, RG);
    dim3 grid((g.sites + a.spc - 1) / a.spc, groups);
    DDAMG_LAUNCH((tc_coarse_op_kernel<RG, NA>), grid, apply_threads(RG), smem, s, vmap, a);
}
// shapes: right-hand sides per CTA 64, 32, 16 (ring depths 6, 8, 10)
int tc_op_shapes() { return 3; }
int tc_op_shape_rg(int shape) { return shape == 0 ? 64 : shape == 1 ? 32 : 16; }
bool tc_op_supported(const Geom& g) { return g.level >= 1 && g.dof <= 32 && g.dof % 2 == 0; }
void launch_coarse_op_tc(cudaStream_t s, const Geom& g, const float* tiles, const float2* in, float2* out,
                         const float2* b, double m0, int nrhs, int shape, int* status) {
    switch (shape) {
        case 0: launch_op_shape<64, 6>(s, g, tiles, in, out, b, m0, nrhs, status); break;
        case 1: launch_op_shape<32, 8>(s, g, tiles, in, out, b, m0, nrhs, status); break;
        default: launch_op_shape<16, 10>(s, g, tiles, in, out, b, m0, nrhs, status); break;
    }
}

// ---------------------------------------------------------------- per (block, rhs) kernels
// one warp per task = kb * R + r; lanes stride over the block's NE = S * dof unknowns
struct TaskGeom {
    int R, NB, S, dof, NE, sel_x, sel_t, Nt, sap_t;
    long size;  // level vector length
};

__device__ __forceinline__ long level_index(const TaskGeom& t, int blk, int e) {
    const int s = e / t.dof, i = e - s * t.dof;
    const int kx = s / t.sel_t, kt = s - kx * t.sel_t;
    const int bx = blk / t.sap_t, bt = blk - bx * t.sap_t;
    return ((long)(bx * t.sel_x + kx) * t.Nt + bt * t.sel_t + kt) * t.dof + i;
}

__global__ void tcs_gather_kernel(TaskGeom t, TcSapWork w, const int* __restrict__ blocks,
                                  const float2* __restrict__ rg, const int* __restrict__ done) {
    const int task = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (task >= t.NB * t.R) return;
    const int kb = task / t.R, r = task - kb * t.R;
    const bool act = !(done && done[r]);
    if (lane == 0) w.act[task] = act ? 1 : 0;
    const int blk = blocks[kb];
    float2* bv = w.b + (long)task * t.NE;
    float2* xv = w.x + (long)task * t.NE;
    for (int e = lane; e < t.NE; e += 32) {
        const float2 v = act ? rg[(long)r * t.size + level_index(t, blk, e)] : make_float2(0.f, 0.f);
        bv[e] = v;
        xv[e] = v;
    }
}

// after a residual w = b - D_B x: norms, convergence, and V_0 = w / ||w|| for the next restart
__global__ void tcs_prep_kernel(TaskGeom t, TcSapWork w, int first, int m, double tol) {
    const int task = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (task >= t.NB * t.R) return;
    const float2* wv = w.w + (long)task * t.NE;
    const float2* bv = w.b + (long)task * t.NE;
    double rr = 0.0, bb = 0.0;
    for (int e = lane; e < t.NE; e += 32) {
        rr += (double)cnorm2(wv[e]);
        if (first) bb += (double)cnorm2(bv[e]);
    }
    rr = warp_sum(rr);
    bb = warp_sum(bb);
    const double err = sqrt(rr);
    int fin;
    if (first) {
        const double nb = sqrt(bb);
        // a zero block right-hand side has the zero solution (the reference would divide by zero)
        fin = (!w.act[task] || nb == 0.0) ? 1 : 0;
        if (lane == 0) {
            w.normb[task] = nb;
            w.maxit[task] = m;
        }
    } else {
        fin = w.fin[task];
        if (!fin && err < tol * w.normb[task]) fin = 1;
    }
    __syncwarp();
    if (lane == 0) {
        w.fin[task] = fin;
        w.arn[task] = fin ? 0 : 1;
        w.err[task] = err;
        if (!fin) w.gm[(long)task * (m + 1)] = make_double2(err, 0.0);
    }
    if (fin) return;
    const float inv = (float)(1.0 / err);
    float2* v0 = w.V + (long)task * t.NE;
    for (int e = lane; e < t.NE; e += 32) v0[e] = inv * wv[e];
}

// Arnoldi step j of every active (block, rhs): classical Gram-Schmidt against V_0..V_j, the new
// basis vector, and the Givens update of Hessenberg column j (FGMRES::rotation,
// src/fgmres.cpp:99-115); a rhs whose estimate meets tol stops its Arnoldi loop (maxIt = j + 1).
template <int EPL>
__global__ void __launch_bounds__(256, EPL <= 16 ? 3 : 1) tcs_arnoldi_kernel(TaskGeom t, TcSapWork w, int j, int m, double tol) {
    const int task = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (task >= t.NB * t.R) return;
    if (!w.arn[task]) return;
    const long off = (long)task * t.NE;
    float2 wl[EPL];
#pragma unroll
    for (int q = 0; q < EPL; q++) {
        const int e = lane + 32 * q;
        wl[q] = e < t.NE ? __ldg(w.w + off + e) : make_float2(0.f, 0.f);
    }
    // all j+1 partial dots first, then one interleaved butterfly
    double2 h[kSapMaxM];
#pragma unroll
    for (int i = 0; i < kSapMaxM; i++) {
        h[i] = make_double2(0.0, 0.0);
        if (i > j) continue;
        const float2* Vi = w.V + (long)i * w.vec + off;
#pragma unroll
        for (int q = 0; q < EPL; q++) {
            const int e = lane + 32 * q;
            if (e < t.NE) h[i] = cfmac(to_d(__ldg(Vi + e)), to_d(wl[q]), h[i]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int i = 0; i < kSapMaxM; i++) {
            if (i > j) continue;
            h[i].x += __shfl_xor_sync(0xffffffffu, h[i].x, o);
            h[i].y += __shfl_xor_sync(0xffffffffu, h[i].y, o);
        }
#pragma unroll
    for (int i = 0; i < kSapMaxM; i++) {
        if (i > j) continue;
        const float2* Vi = w.V + (long)i * w.vec + off;
        const float2 hf = from_d<float2>(h[i]);
#pragma unroll
        for (int q = 0; q < EPL; q++) {
            const int e = lane + 32 * q;
            if (e < t.NE) wl[q] = wl[q] - cmul(hf, __ldg(Vi + e));
        }
    }
    double ww = 0.0;
#pragma unroll
    for (int q = 0; q < EPL; q++) ww += (double)cnorm2(wl[q]);
    const double hn = sqrt(warp_sum(ww));
    if (hn > 0) {
        float2* Vn = w.V + (long)(j + 1) * w.vec + off;
        const float inv = (float)(1.0 / hn);
#pragma unroll
        for (int q = 0; q < EPL; q++) {
            const int e = lane + 32 * q;
            if (e < t.NE) Vn[e] = inv * wl[q];
        }
    }
    if (lane != 0) return;
    double2* H = w.H + (long)task * (m + 1) * m;
    double2* cn = w.cn + (long)task * m;
    double2* sn = w.sn + (long)task * m;
    double2* gm = w.gm + (long)task * (m + 1);
#pragma unroll
    for (int i = 0; i < kSapMaxM; i++)
        if (i <= j) H[i * m + j] = h[i];
    H[(j + 1) * m + j] = make_double2(hn, 0.0);
    for (int i = 0; i < j; i++) {
        const double2 hij = H[i * m + j], hi1 = H[(i + 1) * m + j];
        const double2 tmp = cmulc(cn[i], hij) + cmulc(sn[i], hi1);
        H[(i + 1) * m + j] = cmul(cn[i], hi1) - cmul(sn[i], hij);
        H[i * m + j] = tmp;
    }
    const double2 hjj = H[j * m + j], hj1 = H[(j + 1) * m + j];
    const double den = sqrt(cnorm2(hjj) + cnorm2(hj1));
    sn[j] = make_double2(hj1.x / den, hj1.y / den);
    cn[j] = make_double2(hjj.x / den, hjj.y / den);
    H[j * m + j] = cmulc(cn[j], hjj) + cmulc(sn[j], hj1);
    H[(j + 1) * m + j] = make_double2(0.0, 0.0);
    gm[j + 1] = -cmul(sn[j], gm[j]);
    gm[j] = cmulc(cn[j], gm[j]);
    if (sqrt(cnorm2(gm[j + 1])) < tol * w.normb[task]) {
        w.maxit[task] = j + 1;  // not reset at the next restart (src/fgmres.cpp:14,56)
        w.arn[task] = 0;
    }
}

// solve_upper_triangular (src/fgmres.cpp:118-128) and x += sum_jj eta_jj V_jj
__global__ void tcs_update_kernel(TaskGeom t, TcSapWork w, int m) {
    __shared__ double2 eta_s[8][kSapMaxM];
    const int wib = threadIdx.x >> 5;
    const int task = blockIdx.x * (blockDim.x >> 5) + wib, lane = threadIdx.x & 31;
    if (task >= t.NB * t.R) return;
    if (w.fin[task]) return;
    const int mi = w.maxit[task];
    double2* eta = eta_s[wib];
    if (lane == 0) {
        const double2* H = w.H + (long)task * (m + 1) * m;
        const double2* gm = w.gm + (long)task * (m + 1);
        for (int i = mi - 1; i >= 0; i--) {
            double2 e = gm[i];
            for (int jj = i + 1; jj < mi; jj++) e = e - cmul(H[i * m + jj], eta[jj]);
            eta[i] = cdiv(e, H[i * m + i]);
        }
    }
    __syncwarp();
    const long off = (long)task * t.NE;
    for (int e = lane; e < t.NE; e += 32) {
        float2 a = w.x[off + e];
        for (int jj = 0; jj < mi; jj++) a = cfma(from_d<float2>(eta[jj]), w.V[(long)jj * w.vec + off + e], a);
        w.x[off + e] = a;
    }
}

// x_B += e  (src/sap.cpp:106-113)
__global__ void tcs_scatter_kernel(TaskGeom t, TcSapWork w, const int* __restrict__ blocks, float2* __restrict__ xg) {
    const int task = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (task >= t.NB * t.R) return;
    if (!w.act[task] || w.normb[task] == 0.0) return;
    const int kb = task / t.R, r = task - kb * t.R;
    const int blk = blocks[kb];
    const float2* xv = w.x + (long)task * t.NE;
    for (int e = lane; e < t.NE; e += 32) {
        float2* o = xg + (long)r * t.size + level_index(t, blk, e);
        *o = *o + xv[e];
    }
}

namespace {
struct SweepCtx {
    cudaStream_t s;
    const Geom& g;
    const TcSapWork& w;
    const SapArgs& a;
    int nrhs, S;
    void apply(int shape, const float2* src, const float2* bsub, const int* flag, int invert) const {
        const CUtensorMap vmap = vector_map(src, g.dof, S, (long)a.nblocks * nrhs, kShapes[shape].rg);
        ApplyArgs aa{w.tiles, w.w, bsub, flag, invert, a.blocks, nrhs, S, g.sel_x, g.sel_t, g.Nt, g.sap_t,
                     g.dof, (2 * g.dof + 7) / 8, (float)a.m0 + 2.f, w.status};
        launch_apply(shape, s, vmap, aa, a.nblocks);
    }
    TaskGeom task_geom() const { return TaskGeom{nrhs, a.nblocks, S, g.dof, S * g.dof, g.sel_x, g.sel_t, g.Nt, g.sap_t, g.size()}; }
};
}  // namespace

int tc_sweep_shapes() { return kNumShapes; }
void tc_sweep_shape(int idx, int* rg, int* stages, int* chains) {
    *rg = kShapes[idx].rg;
    *stages = kShapes[idx].na;
    *chains = kShapes[idx].nch;
}

// Times one block-operator application per admissible tile shape on the sweep's own data (gathered
// from r first) and returns the fastest; us[i] gets the time of shape i (negative: not admissible).
// Synchronises the stream: run it outside graph capture.
int tune_sap_tc(cudaStream_t s, const Geom& g, const TcSapWork& w, const float2* r, const SapArgs& a, int nrhs,
                double* us) {
    const int S = g.sel_x * g.sel_t;
    SweepCtx c{s, g, w, a, nrhs, S};
    const TaskGeom t = c.task_geom();
    DDAMG_LAUNCH(tcs_gather_kernel, ceil_div(a.nblocks * nrhs, 8), 256, 0, s, t, w, a.blocks, r, a.done);
    cudaEvent_t e0, e1;
    DDAMG_CUDA_TRY(cudaEventCreate(&e0));
    DDAMG_CUDA_TRY(cudaEventCreate(&e1));
    int best = -1;
    for (int i = 0; i < kNumShapes; i++) {
        us[i] = -1.0;
        if (!shape_fits(i, g.sel_t) || kShapes[i].rg / 2 >= nrhs * 2) continue;  // at most 4x padding
        c.apply(i, w.x, w.b, w.act, 0);  // warm-up
        DDAMG_CUDA_TRY(cudaEventRecord(e0, s));
        for (int k = 0; k < 3; k++) c.apply(i, w.x, w.b, w.act, 0);
        DDAMG_CUDA_TRY(cudaEventRecord(e1, s));
        DDAMG_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        DDAMG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        us[i] = 1e3 * ms / 3;
        if (best < 0 || us[i] < us[best]) best = i;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best >= 0 ? best : default_shape(nrhs, g.sel_t);
}

void launch_sap_sweep_tc(cudaStream_t s, const Geom& g, const TcSapWork& w, const float2* r, float2* x,
                         const SapArgs& a, int nrhs, int shape) {
    if (a.m > kSapMaxM) throw ParamFailure{"SAP block GMRES restart length above 8 is not supported"};
    const int S = g.sel_x * g.sel_t;
    SweepCtx c{s, g, w, a, nrhs, S};
    const TaskGeom t = c.task_geom();
    const int tgrid = ceil_div(a.nblocks * nrhs, 8);
    if (shape < 0 || shape >= kNumShapes || !shape_fits(shape, g.sel_t)) shape = default_shape(nrhs, g.sel_t);
    auto arnoldi = [&](int j) {
        const int epl = (t.NE + 31) / 32;
        if (epl <= 8) DDAMG_LAUNCH(tcs_arnoldi_kernel<8>, tgrid, 256, 0, s, t, w, j, a.m, a.tol);
        else if (epl <= 16) DDAMG_LAUNCH(tcs_arnoldi_kernel<16>, tgrid, 256, 0, s, t, w, j, a.m, a.tol);
        else DDAMG_LAUNCH(tcs_arnoldi_kernel<32>, tgrid, 256, 0, s, t, w, j, a.m, a.tol);
    };
    DDAMG_LAUNCH(tcs_gather_kernel, tgrid, 256, 0, s, t, w, a.blocks, r, a.done);
    c.apply(shape, w.x, w.b, w.act, 0);  // r = b - D_B x0 with x0 = b
    DDAMG_LAUNCH(tcs_prep_kernel, tgrid, 256, 0, s, t, w, 1, a.m, a.tol);
    for (int k = 0; k < a.restarts; k++) {
        for (int j = 0; j < a.m; j++) {
            c.apply(shape, w.V + (long)j * w.vec, nullptr, w.arn, 0);  // w = D_B V_j
            arnoldi(j);
        }
        DDAMG_LAUNCH(tcs_update_kernel, tgrid, 256, 0, s, t, w, a.m);
        c.apply(shape, w.x, w.b, w.fin, 1);  // r = b - D_B x for every rhs not yet converged
        DDAMG_LAUNCH(tcs_prep_kernel, tgrid, 256, 0, s, t, w, 0, a.m, a.tol);
    }
    DDAMG_LAUNCH(tcs_scatter_kernel, tgrid, 256, 0, s, t, w, a.blocks, x);
}

}  // namespace ddamg
