// Interface of the tcgen05 split-bf16 product kernel (tc_gemm.cu).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include <vector>

namespace ptb {
namespace tc {

enum : int { EPI_FULL = 0, EPI_SP2 = 1 };

// Tensor maps of the two A-role and two B-role bf16 planes (64-byte aligned).
struct TmaPlanes {
    CUtensorMap a[2];
    CUtensorMap b[2];
};

// Which (A plane, B plane) pairs are accumulated per K step.
struct ProdList {
    int n;
    int a[4];
    int b[4];
};

struct EpiParams {
    const int* active;        // device flag; 0 -> the launch does nothing (may be null)
    const int* sq_flag;       // EPI_SP2: 1 -> X' = X^2, 0 -> X' = 2X - X^2
    int* err;                 // device error word (bounded waits)
    long long ld;             // leading dimension of every plane / matrix (multiple of 256)
    const float* xcur;        // EPI_SP2: current iterate (FP32)
    float* out;               // EPI_FULL: C;  EPI_SP2: next iterate (FP32)
    __nv_bfloat16* hi;        // EPI_SP2: next iterate, bf16 hi plane
    __nv_bfloat16* lo;        // EPI_SP2: next iterate, bf16 lo plane
    double* stats;            // EPI_SP2: per-tile {trace, sum of squares}
};

int tile_n();
std::vector<int2> make_tiles(long long ld, bool upper_only);
void launch_product(cudaStream_t s, int epi, long long ld, const void* a0, const void* a1, const void* b0,
                    const void* b1, const ProdList& prods, const int2* tiles_dev, int ntiles,
                    const EpiParams& ep);

}  // namespace tc
}  // namespace ptb
