// Device helpers and launch parameters shared by the SAP colour-sweep kernels (kernels_sap.cu,
// kernels_sap2.cu).
#pragma once
#include "internal.h"

namespace ddamg {

// warp sums of N values with one interleaved butterfly (N independent shuffle chains)
template <int N> __device__ __forceinline__ void warp_sum_n(double2 (&v)[N]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int g = 0; g < N; g++) {
            v[g].x += __shfl_xor_sync(0xffffffffu, v[g].x, o);
            v[g].y += __shfl_xor_sync(0xffffffffu, v[g].y, o);
        }
}

struct SapKParams {
    int m, restarts;
    double tol, m0;
    const int* blocks;
    int nblocks;
    const int* done;
    int nrhs;     // vectors in the sweep
    int ngroups;  // CTAs per Schwarz block: ceil(nrhs / RB)
    // non-null: the sweep forms each block's residual r_B = v_B - (D x)_B itself from the SAP right-hand
    // side v (this pointer, the sweep's vector type) and the iterate, instead of reading r
    const void* vres = nullptr;
};

// the latency-trimmed coarse sweep (kernels_sap2.cu): blocks of at most 512 unknowns at restart length 5
// with 1, 2 or 4 right-hand sides per CTA where its shared memory fits
bool sap2_fits(int rb, int m, int NE, size_t vbytes);
template <typename V, int RB>
void launch_sap2(cudaStream_t s, const Geom& g, const V* L, const V* r, V* x, SapKParams p);

}  // namespace ddamg
