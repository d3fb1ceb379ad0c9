// Interface of the int8 tensor-core FP64 product (oz_gemm.cu).
//
// An FP64 matrix is cut into S int8 "slices" per row (Ozaki scheme): with e_i
// the exponent of row i's largest magnitude, M(i,k) = 2^e_i * sum_p s_p(i,k) *
// 2^(-7(p+1)) + r(i,k), |s_p| <= 127, |r| < 2^(e_i - 7S).  A product of two
// sliced operands is the sum over slice pairs (p, q) with p + q <= S - 1 of
// exact int8 x int8 -> int32 tensor-core products; pairs of equal p + q share
// an int32 accumulator in tensor memory, and the epilogue combines the S
// accumulators in FP64.  With S = 7 the result carries about 49 bits relative
// to the largest magnitudes of the row and column involved.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace ptb {
namespace oz {

constexpr int BM = 128;   // output rows per tile
constexpr int BN = 64;    // output columns per tile (S accumulators of BN int32 columns each)

// Row slices of an n x n FP64 matrix.  Plane p holds s_p row-major (K
// contiguous) in ldp x ldp bytes; the planes are stacked (plane p at row
// p * ldp) so that one tensor map covers them all.
struct Operand {
    int8_t* planes = nullptr;
    int* exps = nullptr;   // ldp row exponents (0 for zero and padding rows)
    int64_t ldp = 0;       // padded dimension, a multiple of 128
    int S = 0;             // slices
};

// Which part of a triangular operand is kept (the rest is read as zero).
enum Tri : int { TRI_NONE = 0, TRI_LOWER = 1 /* k <= i */, TRI_UPPER = 2 /* k >= i */ };

enum Epi : int {
    OZ_OUT = 0,   // every listed tile: out[r * ors + c * ocs] = alpha * C(r, c)
    OZ_SYM = 1,   // upper tiles of a symmetric result: for c >= r, v = alpha * C(r, c) (or with xin:
                  // v = C on `square`, 2 X(r,c) - C otherwise), written to (r,c) and (c,r) of the
                  // column-major `out` (leading dimension ors), per-tile {trace, sum of squares}
};

struct OzEpi {
    int* err = nullptr;            // device error word (bounded waits)
    int64_t n = 0;                 // logical dimension (rows/cols >= n are not written)
    int64_t ldp = 0;               // padded dimension of the operands
    double alpha = 1.0;
    double* out = nullptr;
    int64_t ors = 0, ocs = 0;      // output strides (OZ_SYM: column-major, leading dimension ors)
    const double* xin = nullptr;   // OZ_SYM: current SP2 iterate X (column-major, ld ors) or null
    int square = 1;                // OZ_SYM with xin: 1 -> X' = X^2, 0 -> X' = 2X - X^2
    double* stats = nullptr;       // OZ_SYM: 2 doubles per tile (may be null)
};

// Largest K range whose int32 accumulators cannot overflow with S slices.
int64_t max_k(int S);
bool supported(int64_t n, int S);
int64_t padded(int64_t n);   // round_up(n, 128)

// Slices of M(i,k) = M[i * rs + k * cs] (rs == 1 or cs == 1), i,k < n, masked by
// `tri`.  `rowmax` is device scratch of ldp 64-bit words.
void slice(cudaStream_t s, const double* M, int64_t rs, int64_t cs, int64_t n, int tri, const Operand& op,
           unsigned long long* rowmax);

// Kernel variants: A slices re-read from shared memory by every MMA (64-column
// tiles), or copied once per K step into tensor memory (48-column tiles for 7
// or 8 slices, 64 for fewer), or the shared-memory variant on a CTA pair
// (cta_group::2: 256-row tiles, each SM loads half of the 64 B rows), or
// 128-column tiles whose accumulator groups are summed in two passes over K
// (32-byte K blocks only), or those on a CTA pair (256 x 128 tiles).  All give
// bit-identical results.
enum Variant : int { V_DEFAULT = 0, V_SMEM_A = 1, V_TMEM_A = 2, V_PAIR = 3, V_WIDE = 4, V_WPAIR = 5 };
// The variant V_DEFAULT stands for with S slices and rb-byte K blocks (0 = the
// variant's default); the functions below take resolved variants only.
int resolve_variant(int variant, int S, int rb);
int tile_n(int S, int variant);   // output columns per tile

// Tiles {bi, bj, k0, k1}: 128-row blocks of ldp by bn-column blocks (the last
// may overhang), all or only those touching the upper triangle; the K range of
// each tile is cut to the nonzero part (whole 128-blocks) of a triangular A
// (rows of A) or B (rows of B).  Longest K ranges first.
std::vector<int4> make_tiles(int64_t ldp, bool upper, int a_tri, int b_tri, int bn);

// CTA-pair tiles {pair row block p (rows 256p..256p+255), bj (bn columns), k0,
// k1}: pairs with a half that touches the upper triangle (when `upper`), K
// range = the union of the ranges of those halves (the extra blocks of a
// triangular operand are zero slices).  Longest K ranges first.
std::vector<int4> make_pair_tiles(int64_t ldp, bool upper, int a_tri, int b_tri, int bn);

// The tile list `product` expects for `variant`, the CTAs it launches for it
// (one per tile entry, two per pair entry; OZ_SYM writes one stats pair per
// CTA), and the int8 multiply-adds x 2 the tiles execute.
std::vector<int4> build_tiles(int64_t ldp, bool upper, int a_tri, int b_tri, int S, int variant);
int grid_ctas(int ntiles, int variant);
double tile_ops(const std::vector<int4>& tiles, int S, int variant);

// C(i,j) = sum_k A(i,k) B(j,k) over the listed tiles, which must be built by
// build_tiles for the same (resolved) variant.  rb: K bytes per stage, 64 (64B
// swizzle) or 32 (32B swizzle); 0 = the variant's default.
void product(cudaStream_t s, int epi, const Operand& a, const Operand& b, const int4* tiles_dev, int ntiles,
             const OzEpi& ep, int rb, int variant);

}  // namespace oz
}  // namespace ptb
