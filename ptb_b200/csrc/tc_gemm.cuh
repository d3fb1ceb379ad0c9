// Interface of the tcgen05 split-bf16 product kernels (tc_gemm.cu).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include <vector>

namespace ptb {
namespace tc {

enum : int { EPI_FULL = 0, EPI_SP2 = 1 };

// Kernel choice codes: K block 64 or 32 for the one-CTA kernel, and
// kPairKernel + K block for the CTA-pair (cta_group::2, 256 x 256) kernel.
constexpr int kPairKernel = 1000;

// Tensor maps of up to three A-role and three B-role bf16 planes (64-byte aligned).
struct TmaPlanes {
    CUtensorMap a[3];
    CUtensorMap b[3];
};

// Which (A plane, B plane) pairs are accumulated per K step.
struct ProdList {
    int n;
    int a[6];
    int b[6];
};

struct EpiParams {
    const int* active;        // device flag(s); 0 -> the tile does nothing (may be null)
    const int* sq_flag;       // EPI_SP2: 1 -> X' = X^2, 0 -> X' = 2X - X^2
    // stacked != 0: the planes hold systems of ld x ld stacked along the rows
    // (row-major, ld columns); tiles carry global row blocks, output columns
    // are local to the tile's system, and active / sq_flag are per system
    int stacked;
    int* err;                 // device error word (bounded waits)
    long long ld;             // leading dimension of every plane / matrix (multiple of 256)
    const float* xcur;        // EPI_SP2: current iterate (FP32)
    float* out;               // EPI_FULL: C;  EPI_SP2: next iterate (FP32)
    __nv_bfloat16* hi;        // EPI_SP2: next iterate, bf16 hi plane
    __nv_bfloat16* lo;        // EPI_SP2: next iterate, bf16 mid plane  (x - hi)
    __nv_bfloat16* lo2;       // EPI_SP2: next iterate, bf16 lo plane   (x - hi - mid); null: not written
    double* stats;            // EPI_SP2: per-CTA {trace, sum of squares}
};

// Two-plane products run on 128 x 256 tiles (one CTA) or 256 x 256 tiles (a
// CTA pair), three-plane products on 128 x 128.
int tile_n();
std::vector<int2> make_tiles(long long ld, bool upper_only, int bn);
std::vector<int2> make_pair_tiles(long long ld, bool upper_only);
// kblock: 64 / 32 (one CTA), kPairKernel + 64 / + 32 (CTA pair, needs two
// planes and pairs_dev), or 0 = the autotuned choice for this shape (every
// candidate is timed on its first launch).  Returns the number of per-CTA
// stats partials written (EPI_SP2 reduces that many).
// rows: rows of every plane (0 = ld; a multiple of ld for stacked systems).
int launch_product(cudaStream_t s, int epi, int np, long long ld, const void* const* a, const void* const* b,
                   const ProdList& prods, const int2* tiles_dev, int ntiles, const EpiParams& ep, int kblock = 0,
                   const int2* pairs_dev = nullptr, int npairs = 0, long long rows = 0);
int tuned_kblock(int epi, int np, long long ld, long long rows = 0);   // 0 until the shape has been tuned

}  // namespace tc
}  // namespace ptb
