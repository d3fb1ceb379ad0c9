// FP64 products on the int8 tensor cores (tcgen05 kind::i8, int32 in tensor
// memory): Ozaki-scheme slicing of the operands and the product kernel.
//
// Product kernel, one CTA per 128 x 64 output tile (cta_group::1):
//   warp 0      TMA producer: per K block of RB bytes, the S A-slices (128 x RB)
//               and the S B-slices (64 x RB) into a ring of stages (64B or 32B
//               swizzle), completion on a "full" mbarrier with a byte count;
//   warp 1      MMA issuer: for every K32 step, the S(S+1)/2 slice pairs
//               (p, q), p + q <= S - 1, as UMMA 128x64x32 int8 into
//               accumulator p + q (tensor-memory columns (p + q) * 64 ..);
//               tcgen05.commit frees the stage;
//   warp 2      allocates / frees 512 tensor-memory columns;
//   warps 4..7  epilogue: per row, sum_g 2^(-7(g+2)) G_g in FP64 (smallest
//               group first), times 2^(e_i + f_j), then the fused output.
// The int32 sums are exact: a group has at most S pairs of |s| <= 127 terms, so
// K <= (2^31 - 1) / (S * 127^2) (19020 for S = 7) never overflows.
//
// Every mbarrier wait is bounded (2 s); on expiry the CTA records an error
// site, drains its copies and frees its tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <mutex>

#include "common.cuh"
#include "oz_gemm.cuh"
#include "tc_ptx.cuh"

namespace ptb {
namespace oz {

namespace {

using namespace tc::ptx;

constexpr int THREADS = 256;
constexpr int kSmemBudget = 196608;
constexpr int kTmemCols = 512;
// Dynamic shared memory that keeps a kernel at one resident CTA per SM (more
// than half of the 227 KB a block may use).  The CTA-pair kernels hold all 512
// TMEM columns of both SMs of a pair: two pair CTAs resident on the same SMs
// could each hold one SM's columns while their peers wait in tcgen05.alloc for
// the other's, and neither pair would finish.
constexpr int kSmemMax = 232448;
constexpr int kOneCtaPerSm = kSmemMax / 2 + 1024;

template <int S, int RB>
struct OzCfg {
    static constexpr int A_TILE = BM * RB;
    static constexpr int B_TILE = BN * RB;
    static constexpr int STAGE = S * (A_TILE + B_TILE);
    static constexpr int STAGES = (kSmemBudget / STAGE) > 4 ? 4 : (kSmemBudget / STAGE);
    static constexpr int SMEM = STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
    static constexpr uint32_t LAYOUT = RB == 64 ? 4u : 6u;   // SWIZZLE_64B / SWIZZLE_32B
    static constexpr uint32_t SBO = 8u * RB;                  // bytes between 8-row groups
    // kind::i8: D s32 (2), A and B signed int8 (1), both K-major, N = 64, M = 128
    static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                      ((uint32_t)(BM >> 4) << 24);
    static_assert(RB == 64 || RB == 32, "64- or 32-byte K blocks");
    static_assert(S >= 2 && S * BN <= kTmemCols, "S accumulators of 64 columns fit in tensor memory");
    static_assert(STAGES >= 2, "at least two pipeline stages");
    static_assert(A_TILE % 1024 == 0 && B_TILE % 1024 == 0, "tiles keep the swizzle atoms aligned");
};

// 2^e as a double for -1022 <= e <= 1023 (IEEE-754 exponent field).
__device__ __forceinline__ double pow2i(int e) {
    return __longlong_as_double((long long)(e + 1023) << 52);
}
// x * 2^e for |e| <= 2044, exact while the result is a normal number
__device__ __forceinline__ double scale2(double x, int e) {
    const int h = e / 2;
    return x * pow2i(h) * pow2i(e - h);
}

// ---- slicing ---------------------------------------------------------------
__device__ __forceinline__ bool tri_keep(int tri, int64_t i, int64_t k) {
    return tri == TRI_NONE || (tri == TRI_LOWER ? k <= i : k >= i);
}

// Row maxima of |M(i,k)| over a 32-row x 128-column tile, merged with
// atomicMax on the bit patterns (order-preserving for non-negative doubles).
__global__ void k_oz_rowmax(const double* __restrict__ M, int64_t rs, int64_t cs, int64_t n, int tri,
                            unsigned long long* __restrict__ rowmax) {
    const int64_t i0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 128;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (cs == 1) {
        // rows contiguous: each warp takes 4 rows, lanes run along k
        for (int rr = 0; rr < 4; ++rr) {
            const int64_t i = i0 + w * 4 + rr;
            double m = 0.0;
            if (i < n) {
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int64_t k = k0 + lane + 32 * t;
                    if (k < n && tri_keep(tri, i, k)) m = fmax(m, fabs(M[i * rs + k]));
                }
            }
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0 && i < n && m > 0.0) atomicMax(&rowmax[i], (unsigned long long)__double_as_longlong(m));
        }
    } else {
        // columns contiguous: lanes run along i, warps along k
        __shared__ double red[8][33];
        const int64_t i = i0 + lane;
        double m = 0.0;
        if (i < n) {
            for (int t = 0; t < 16; ++t) {
                const int64_t k = k0 + w + 8 * t;
                if (k < n && tri_keep(tri, i, k)) m = fmax(m, fabs(M[i + k * cs]));
            }
        }
        red[w][lane] = m;
        __syncthreads();
        if (w == 0) {
            for (int t = 1; t < 8; ++t) m = fmax(m, red[t][lane]);
            if (i < n && m > 0.0) atomicMax(&rowmax[i], (unsigned long long)__double_as_longlong(m));
        }
    }
}

// Slices of a 32-row x 64-column tile; rows/columns beyond n (the padding up
// to ldp) are written as zero.  e_i: |M(i,k)| < 2^e_i, taken from the
// exponent field of the row maximum.
template <int S>
__global__ void k_oz_slice(const double* __restrict__ M, int64_t rs, int64_t cs, int64_t n, int tri,
                           const unsigned long long* __restrict__ rowmax, int8_t* __restrict__ planes,
                           int* __restrict__ exps, int64_t ldp) {
    __shared__ double t[32][65];
    const int64_t i0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 64;
    if (cs == 1) {
        for (int e = threadIdx.x; e < 32 * 64; e += THREADS) {
            const int r = e >> 6, kk = e & 63;
            const int64_t i = i0 + r, k = k0 + kk;
            t[r][kk] = (i < n && k < n && tri_keep(tri, i, k)) ? M[i * rs + k] : 0.0;
        }
    } else {
        for (int e = threadIdx.x; e < 32 * 64; e += THREADS) {
            const int r = e & 31, kk = e >> 5;
            const int64_t i = i0 + r, k = k0 + kk;
            t[r][kk] = (i < n && k < n && tri_keep(tri, i, k)) ? M[i + k * cs] : 0.0;
        }
    }
    __syncthreads();
    const int r = threadIdx.x >> 3, kq = (threadIdx.x & 7) * 8;
    const int64_t i = i0 + r;
    int e = 0;
    if (i < n) {
        const unsigned long long b = rowmax[i];
        if (b != 0ull) {
            const int fld = (int)((b >> 52) & 0x7FF);
            e = fld == 0 ? -1022 : fld - 1022;   // max = m 2^e, 0.5 <= m < 1 (subnormal: max < 2^-1022)
        }
    }
    if (blockIdx.x == 0 && (threadIdx.x & 7) == 0) exps[i] = e;
    const double sc = pow2i(-e);
    uint32_t w[S][2];
#pragma unroll
    for (int p = 0; p < S; ++p) w[p][0] = w[p][1] = 0u;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        double x = t[r][kq + j] * sc;   // |x| < 1
#pragma unroll
        for (int p = 0; p < S; ++p) {
            x *= 128.0;
            const double q = trunc(x);   // |q| <= 127
            x -= q;                      // exact: the fraction of x
            const uint32_t byte = (uint32_t)(uint8_t)(int8_t)(int)q;
            w[p][j >> 2] |= byte << (8 * (j & 3));
        }
    }
#pragma unroll
    for (int p = 0; p < S; ++p)
        *reinterpret_cast<uint2*>(planes + ((int64_t)p * ldp + i) * ldp + k0 + kq) = make_uint2(w[p][0], w[p][1]);
}

// ---- product ---------------------------------------------------------------
struct OzMaps {
    CUtensorMap a;    // S stacked A planes
    CUtensorMap b;    // S stacked B planes
    CUtensorMap a2;   // the same planes with 64-byte K boxes (second pass of the 128-column kernel)
    CUtensorMap b2;
};

template <int W>
__device__ __forceinline__ void tmem_ldw(uint32_t taddr, uint32_t (&v)[W]) {
    if constexpr (W == 32) tmem_ld32(taddr, v);
    else tmem_ld16(taddr, v);
}

template <int EPI, int W>
__device__ __forceinline__ void oz_write(const OzEpi& ep, int64_t r, int64_t cb, const double (&acc)[W], int er,
                                         const int* __restrict__ eb, double& tr, double& ss);

// W columns [c0, c0 + W) of the tile: combine the S group accumulators
// (columns g * NT + c0 ..) in FP64, smallest group first, rescale by
// 2^(e_r + f_c) and write the fused output.
template <int EPI, int S, int NT, int W>
__device__ __forceinline__ void oz_epilogue_chunk(const OzEpi& ep, uint32_t tmem, int bi, int bj, int q4, int lane,
                                                  int c0, bool empty_k, int er, const int* __restrict__ eb,
                                                  double& tr, double& ss) {
    const int64_t r = (int64_t)bi * BM + q4 * 32 + lane;
    double acc[W];
#pragma unroll
    for (int j = 0; j < W; ++j) acc[j] = 0.0;
#pragma unroll 1
    for (int g = S - 1; g >= 0; --g) {
        uint32_t v[W];
        __syncwarp();
        tmem_ldw<W>(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(g * NT + c0), v);
        const double w = pow2i(-7 * (g + 2));
#pragma unroll
        for (int j = 0; j < W; ++j) acc[j] += (double)(int)v[j] * w;
    }
    if (empty_k) {
#pragma unroll
        for (int j = 0; j < W; ++j) acc[j] = 0.0;
    }
    oz_write<EPI, W>(ep, r, (int64_t)bj * NT + c0, acc, er, eb, tr, ss);
}

// Fused output of W finished FP64 sums of row r, columns cb.. (the caller has
// combined the groups): rescale by 2^(e_r + f_c), general strides (OZ_OUT) or
// the upper triangle mirrored with the optional SP2 update and the trace /
// sum-of-squares partials (OZ_SYM).
template <int EPI, int W>
__device__ __forceinline__ void oz_write(const OzEpi& ep, int64_t r, int64_t cb, const double (&acc)[W], int er,
                                         const int* __restrict__ eb, double& tr, double& ss) {
    const int64_t n = ep.n;
    if (r >= n) return;
    if (EPI == OZ_OUT) {
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const int64_t c = cb + j;
            if (c < n) ep.out[r * ep.ors + c * ep.ocs] = ep.alpha * scale2(acc[j], er + eb[c]);
        }
    } else {
        if (cb + W - 1 < r) return;   // chunk entirely below the diagonal
        const int64_t ld = ep.ors;
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const int64_t c = cb + j;
            if (c < r || c >= n) continue;
            double val = ep.alpha * scale2(acc[j], er + eb[c]);
            if (ep.xin && !ep.square) val = 2.0 * ep.xin[r + c * ld] - val;
            ep.out[r + c * ld] = val;
            if (c == r) {
                tr += val;
                ss += val * val;
            } else {
                ss += 2.0 * val * val;
                ep.out[c + r * ld] = val;
            }
        }
    }
}

// Epilogue warps 4..7 (q4 = TMEM lane quarter): wait for the accumulators
// (bounded), drain them chunk by chunk, reduce the per-tile trace / sum of
// squares of a symmetric result in a fixed order.
template <int EPI, int S, int NT>
__device__ __forceinline__ void oz_epilogue(const OzEpi& ep, uint32_t tmem, uint32_t accum_bar, int* abort_flag,
                                            double* red, int bi, int bj, int q4, int lane, int nk,
                                            const int* __restrict__ ea, const int* __restrict__ eb) {
    static_assert(NT == 64 || NT == 48, "tile widths of 64 or 48 columns");
    const int64_t r = (int64_t)bi * BM + q4 * 32 + lane;
    double tr = 0.0, ss = 0.0;
    const bool ok = __all_sync(0xffffffffu, mbar_wait(accum_bar, 0));
    if (!ok && lane == 0) {
        set_err(ep.err, 131);
        *(volatile int*)abort_flag = 1;
    }
    const int aborted = __shfl_sync(0xffffffffu, *(volatile int*)abort_flag, 0);
    tc_fence_after();
    if (ok && !aborted) {
        const int er = r < ep.n ? ea[r] : 0;
        oz_epilogue_chunk<EPI, S, NT, 32>(ep, tmem, bi, bj, q4, lane, 0, nk == 0, er, eb, tr, ss);
        if constexpr (NT == 64)
            oz_epilogue_chunk<EPI, S, NT, 32>(ep, tmem, bi, bj, q4, lane, 32, nk == 0, er, eb, tr, ss);
        else
            oz_epilogue_chunk<EPI, S, NT, 16>(ep, tmem, bi, bj, q4, lane, 32, nk == 0, er, eb, tr, ss);
    }
    if (EPI == OZ_SYM && ep.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            tr += __shfl_xor_sync(0xffffffffu, tr, o);
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
        }
        if (lane == 0) {
            red[2 * q4] = tr;
            red[2 * q4 + 1] = ss;
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");   // epilogue warps only
        if (q4 == 0 && lane == 0) {
            ep.stats[2 * blockIdx.x] = red[0] + red[2] + red[4] + red[6];
            ep.stats[2 * blockIdx.x + 1] = red[1] + red[3] + red[5] + red[7];
        }
    }
}

template <int EPI, int S, int RB>
__global__ void __launch_bounds__(THREADS, 1)
    k_oz_product(const __grid_constant__ OzMaps maps, const int4* __restrict__ tiles, const int* __restrict__ ea,
                 const int* __restrict__ eb, OzEpi ep) {
    using C = OzCfg<S, RB>;
    constexpr int STAGE = C::STAGE;
    constexpr int STAGES = C::STAGES;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - base_raw);
    const uint32_t bar0 = base + STAGES * STAGE;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
    const uint32_t accum_bar = bar0 + 8u * (2 * STAGES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE + 8 * (2 * STAGES + 1));
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(gbase + STAGES * STAGE + 128);   // 8 doubles

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int4 tile = tiles[blockIdx.x];
    const int bi = tile.x, bj = tile.y;
    const int kb0 = tile.z / RB;
    const int nk = (tile.w - tile.z) / RB;

    auto a_tile = [&](int s, int p) { return base + s * STAGE + p * C::A_TILE; };
    auto b_tile = [&](int s, int q) { return base + s * STAGE + S * C::A_TILE + q * C::B_TILE; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(accum_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"((uint32_t)kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer ----------------
        int issued_phase[STAGES];
        for (int s = 0; s < STAGES; ++s) issued_phase[s] = -1;
        for (int it = 0; it < nk; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (round > 0 && !mbar_wait(empty_bar(s), (round - 1) & 1)) {
                set_err(ep.err, 111);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            mbar_expect_tx(full_bar(s), STAGE);
            const int kx = (kb0 + it) * RB;
            for (int p = 0; p < S; ++p)
                tma_load_2d(a_tile(s, p), &maps.a, full_bar(s), kx, (int)(p * ep.ldp) + bi * BM);
            for (int q = 0; q < S; ++q)
                tma_load_2d(b_tile(s, q), &maps.b, full_bar(s), kx, (int)(q * ep.ldp) + bj * BN);
            issued_phase[s] = round & 1;
        }
        for (int s = 0; s < STAGES; ++s)
            if (issued_phase[s] >= 0 && !mbar_wait(full_bar(s), (uint32_t)issued_phase[s])) set_err(ep.err, 112);
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        bool ok = true;
        for (int it = 0; it < nk; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (!mbar_wait(full_bar(s), round & 1)) {
                set_err(ep.err, 121);
                *(volatile int*)abort_flag = 1;
                ok = false;
                break;
            }
            if (*(volatile int*)abort_flag) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < RB / 32; ++k) {
#pragma unroll
                for (int p = 0; p < S; ++p) {
                    const uint64_t ad = sdesc(a_tile(s, p) + k * 32, C::SBO, C::LAYOUT);
#pragma unroll
                    for (int q = 0; q < S - p; ++q) {
                        const uint64_t bd = sdesc(b_tile(s, q) + k * 32, C::SBO, C::LAYOUT);
                        // p = 0 opens every accumulator on the first K step; the rest add
                        umma_i8(tmem + (uint32_t)((p + q) * BN), ad, bd, C::IDESC, (it | k | p) != 0);
                    }
                }
            }
            umma_commit(empty_bar(s));
        }
        umma_commit(accum_bar);
        if (!ok) mbar_wait(accum_bar, 0);
    } else if (warp >= 4) {
        oz_epilogue<EPI, S, BN>(ep, tmem, accum_bar, abort_flag, red, bi, bj, warp - 4, lane, nk, ea, eb);
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols));
    }
}

// Same product with the A slices in tensor memory: per K32 step, tcgen05.cp
// copies the S A-slices (128 rows x 32 bytes each) from the stage into one of
// two TMEM buffers (columns 384.. and 448..), and the S(S+1)/2 MMAs read A from
// there and only the B slice from shared memory, which removes the A re-reads
// that bound the kernel above (each A slice feeds S - p MMAs).  The
// accumulators are NT columns wide (48 for 7 or 8 slices, 64 for fewer) so
// that S * NT <= 384.  A buffer is rewritten only after the MMAs that read it
// have completed (tcgen05.commit to a per-buffer mbarrier, bounded wait).
template <int EPI, int S, int RB, int NT>
__global__ void __launch_bounds__(THREADS, 1)
    k_oz_product_ta(const __grid_constant__ OzMaps maps, const int4* __restrict__ tiles, const int* __restrict__ ea,
                    const int* __restrict__ eb, OzEpi ep) {
    constexpr int A_TILE = BM * RB;
    constexpr int B_TILE = NT * RB;
    constexpr int STAGE = S * (A_TILE + B_TILE);
    constexpr int STAGES = (kSmemBudget / STAGE) > 4 ? 4 : (kSmemBudget / STAGE);
    constexpr uint32_t LAYOUT = RB == 64 ? 4u : 6u;
    constexpr uint32_t SBO = 8u * RB;
    constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                               ((uint32_t)(BM >> 4) << 24);
    constexpr uint32_t TA = 384;   // first TMEM column of the A buffers (2 x 8 S columns)
    static_assert(S * NT <= (int)TA && TA + 16 * S <= (uint32_t)kTmemCols, "TMEM budget");
    static_assert(NT % 16 == 0 && STAGES >= 2, "tile shape");
    static_assert(A_TILE % (8 * RB) == 0 && B_TILE % (8 * RB) == 0, "tiles keep the swizzle atoms aligned");

    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - base_raw);
    const uint32_t bar0 = base + STAGES * STAGE;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
    const uint32_t accum_bar = bar0 + 8u * (2 * STAGES);
    const uint32_t abuf_bar0 = bar0 + 8u * (2 * STAGES + 1);   // two: one per A buffer
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE + 8 * (2 * STAGES + 3));
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(gbase + STAGES * STAGE + 128);   // 8 doubles

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int4 tile = tiles[blockIdx.x];
    const int bi = tile.x, bj = tile.y;
    const int kb0 = tile.z / RB;
    const int nk = (tile.w - tile.z) / RB;

    auto a_tile = [&](int s, int p) { return base + s * STAGE + p * A_TILE; };
    auto b_tile = [&](int s, int q) { return base + s * STAGE + S * A_TILE + q * B_TILE; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(accum_bar, 1);
        mbar_init(abuf_bar0, 1);
        mbar_init(abuf_bar0 + 8u, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"((uint32_t)kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer ----------------
        int issued_phase[STAGES];
        for (int s = 0; s < STAGES; ++s) issued_phase[s] = -1;
        for (int it = 0; it < nk; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (round > 0 && !mbar_wait(empty_bar(s), (round - 1) & 1)) {
                set_err(ep.err, 141);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            mbar_expect_tx(full_bar(s), STAGE);
            const int kx = (kb0 + it) * RB;
            for (int p = 0; p < S; ++p)
                tma_load_2d(a_tile(s, p), &maps.a, full_bar(s), kx, (int)(p * ep.ldp) + bi * BM);
            for (int q = 0; q < S; ++q)
                tma_load_2d(b_tile(s, q), &maps.b, full_bar(s), kx, (int)(q * ep.ldp) + bj * NT);
            issued_phase[s] = round & 1;
        }
        for (int s = 0; s < STAGES; ++s)
            if (issued_phase[s] >= 0 && !mbar_wait(full_bar(s), (uint32_t)issued_phase[s])) set_err(ep.err, 142);
    } else if (warp == 1 && lane == 0) {
        // ---------------- copy + MMA issuer ----------------
        bool ok = true;
        int t = 0;   // K32 step counter over the tile
        for (int it = 0; it < nk && ok; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (!mbar_wait(full_bar(s), round & 1)) {
                set_err(ep.err, 151);
                *(volatile int*)abort_flag = 1;
                ok = false;
                break;
            }
            if (*(volatile int*)abort_flag) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < RB / 32; ++k, ++t) {
                const int b = t & 1;
                if (t >= 2 && !mbar_wait(abuf_bar0 + 8u * b, (uint32_t)(((t - 2) >> 1) & 1))) {
                    set_err(ep.err, 152);
                    *(volatile int*)abort_flag = 1;
                    ok = false;
                    break;
                }
                const uint32_t ta = tmem + TA + (uint32_t)(b * 8 * S);
#pragma unroll
                for (int p = 0; p < S; ++p)
                    tmem_cp_128x256b(ta + 8u * p, sdesc(a_tile(s, p) + k * 32, SBO, LAYOUT));
#pragma unroll
                for (int p = 0; p < S; ++p) {
#pragma unroll
                    for (int q = 0; q < S - p; ++q) {
                        const uint64_t bd = sdesc(b_tile(s, q) + k * 32, SBO, LAYOUT);
                        umma_i8_ta(tmem + (uint32_t)((p + q) * NT), ta + 8u * p, bd, IDESC, (t | p) != 0);
                    }
                }
                umma_commit(abuf_bar0 + 8u * b);
            }
            umma_commit(empty_bar(s));
        }
        umma_commit(accum_bar);
        if (!ok) mbar_wait(accum_bar, 0);
    } else if (warp >= 4) {
        oz_epilogue<EPI, S, NT>(ep, tmem, accum_bar, abort_flag, red, bi, bj, warp - 4, lane, nk, ea, eb);
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols));
    }
}

// CTA-pair variant (cta_group::2, cluster of two): one 256 x 64 tile per pair,
// UMMA 256x64x32 int8 issued by the leader CTA.  CTA r holds rows 128r..128r+127
// of the A slices and of the accumulators, and rows 32r..32r+31 of the 64 B
// rows, so each SM reads its A slice and half the B slice per MMA (5 KB instead
// of 6 KB of shared memory for 32 tensor cycles of the SM).  Both CTAs' TMA
// loads count on the leader's "full" mbarrier, which the leader arms with both
// CTAs' bytes; the leader's commits arrive on the "empty" and accumulator
// barriers of both CTAs (tcgen05.commit multicast; no multicast loads).  The
// epilogue is the one-CTA epilogue on each CTA's own 128 rows.  Tiles
// {pair row block, bj, k0, k1}: the K range covers both halves.
template <int S, int RB>
struct OzPairCfg {
    static constexpr int A_TILE = BM * RB;
    static constexpr int B_TILE = (BN / 2) * RB;
    static constexpr int STAGE = S * (A_TILE + B_TILE);
    static constexpr int STAGES = (kSmemBudget / STAGE) > 4 ? 4 : (kSmemBudget / STAGE);
    static constexpr int SMEM = STAGES * STAGE + 1024 + 256 > kOneCtaPerSm ? STAGES * STAGE + 1024 + 256
                                                                          : kOneCtaPerSm;
    static constexpr uint32_t LAYOUT = RB == 64 ? 4u : 6u;
    static constexpr uint32_t SBO = 8u * RB;
    // kind::i8: D s32, A and B s8, K-major, N = 64, M = 256 (the pair)
    static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                      ((uint32_t)(256 >> 4) << 24);
    static_assert(RB == 64 || RB == 32, "64- or 32-byte K blocks");
    static_assert(S >= 2 && S * BN <= kTmemCols, "S accumulators of 64 columns fit in tensor memory");
    static_assert(STAGES >= 2, "at least two pipeline stages");
    static_assert(A_TILE % 1024 == 0 && B_TILE % 1024 == 0, "tiles keep the swizzle atoms aligned");
    static_assert(SMEM >= kOneCtaPerSm && SMEM <= kSmemMax, "one resident CTA per SM");
};

template <int EPI, int S, int RB>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
    k_oz_product_pair(const __grid_constant__ OzMaps maps, const int4* __restrict__ pairs,
                      const int* __restrict__ ea, const int* __restrict__ eb, OzEpi ep) {
    using C = OzPairCfg<S, RB>;
    constexpr int STAGE = C::STAGE;
    constexpr int STAGES = C::STAGES;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - base_raw);
    const uint32_t bar0 = base + STAGES * STAGE;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
    const uint32_t accum_bar = bar0 + 8u * (2 * STAGES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE + 8 * (2 * STAGES + 1));
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(gbase + STAGES * STAGE + 128);   // 8 doubles

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int4 pt = pairs[blockIdx.x >> 1];
    const int bi = 2 * pt.x + (int)rank, bj = pt.y;
    const int kb0 = pt.z / RB;
    const int nk = (pt.w - pt.z) / RB;
    // an odd row-block count leaves the second half of the last pair past the
    // operand: it loads the first half's rows again and writes nothing
    const int nbi = (int)(ep.ldp / BM);
    const int abi = bi < nbi ? bi : nbi - 1;

    auto a_tile = [&](int s, int p) { return base + s * STAGE + p * C::A_TILE; };
    auto b_tile = [&](int s, int q) { return base + s * STAGE + S * C::A_TILE + q * C::B_TILE; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(accum_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"((uint32_t)kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();   // both CTAs' barriers are initialised before any remote arrive
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        int issued_phase[STAGES];
        for (int s = 0; s < STAGES; ++s) issued_phase[s] = -1;
        for (int it = 0; it < nk; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (round > 0 && !mbar_wait(empty_bar(s), (round - 1) & 1)) {
                set_err(ep.err, 141);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            if (rank == 0) mbar_expect_tx(full_bar(s), 2 * STAGE);   // both CTAs' bytes
            const uint32_t fb = mapa_shared(full_bar(s), 0);
            const int kx = (kb0 + it) * RB;
            for (int p = 0; p < S; ++p)
                tma_load_2d_pair(a_tile(s, p), &maps.a, fb, kx, (int)(p * ep.ldp) + abi * BM);
            for (int q = 0; q < S; ++q)
                tma_load_2d_pair(b_tile(s, q), &maps.b, fb, kx, (int)(q * ep.ldp) + bj * BN + (int)rank * (BN / 2));
            issued_phase[s] = round & 1;
        }
        // drain: the leader sees every copy of the pair land on its full barriers;
        // the peer's copies have landed once the leader's MMAs consumed them,
        // which its accumulator barrier (waited by the epilogue) certifies
        if (rank == 0)
            for (int s = 0; s < STAGES; ++s)
                if (issued_phase[s] >= 0 && !mbar_wait(full_bar(s), (uint32_t)issued_phase[s])) set_err(ep.err, 142);
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // ---------------- MMA issuer (leader CTA) ----------------
        bool ok = true;
        for (int it = 0; it < nk; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (!mbar_wait(full_bar(s), round & 1)) {
                set_err(ep.err, 151);
                *(volatile int*)abort_flag = 1;
                ok = false;
                break;
            }
            if (*(volatile int*)abort_flag) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < RB / 32; ++k) {
#pragma unroll
                for (int p = 0; p < S; ++p) {
                    const uint64_t ad = sdesc(a_tile(s, p) + k * 32, C::SBO, C::LAYOUT);
#pragma unroll
                    for (int q = 0; q < S - p; ++q) {
                        const uint64_t bd = sdesc(b_tile(s, q) + k * 32, C::SBO, C::LAYOUT);
                        umma_i8_pair(tmem + (uint32_t)((p + q) * BN), ad, bd, C::IDESC, (it | k | p) != 0);
                    }
                }
            }
            umma_commit_pair(empty_bar(s), (uint16_t)0x3);
        }
        umma_commit_pair(accum_bar, (uint16_t)0x3);   // also on abort so both epilogues' waits end
        if (!ok) mbar_wait(accum_bar, 0);
    } else if (warp >= 4) {
        oz_epilogue<EPI, S, BN>(ep, tmem, accum_bar, abort_flag, red, bi, bj, warp - 4, lane, nk, ea, eb);
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    cluster_sync();   // the leader's MMAs have finished reading the peer's shared memory
    tc_fence_after();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols));
    }
}

// Wide variant: one CTA per 128 x 128 tile, UMMA 128x128x32 int8.  Every
// tcgen05.mma instruction costs the tensor pipe a fixed ~17 cycles besides its
// math (32 cycles at N = 64, 64 at N = 128: measured as tensor-pipe activity of
// 51 % against 80 % for the issuing pipe in the 64-column kernels), so N = 128
// halves that overhead per flop.  Eight 128-column int32 accumulators do not
// fit the 512 TMEM columns, so the groups are split over two passes over K:
// pass 1 sums the slice pairs of groups GS..S-1 (GS = S - 4, the low-weight
// groups) and its epilogue combines them in FP64, smallest group first, and
// parks the partial sum in the output's own storage (OZ_OUT: the element
// itself; OZ_SYM: the mirrored lower-triangle element, which nothing reads,
// and a register for the diagonal); pass 2 sums groups 0..GS-1 into the freed
// columns and the epilogue continues the same FP64 sum from the parked value.
// The result is bit-identical to the 64-column kernel.  Pass 2 loads only the
// slices 0..GS-1; its loads overlap the pass-1 epilogue.  Pass 1 takes K
// blocks of 32 bytes (32B swizzle: a stage holds S A slices and S B slices of
// 4 KB each), pass 2 blocks of 64 bytes (64B swizzle, GS slices of 8 KB each in
// the same stage buffers), so that its few MMAs per K byte still see two K32
// steps of work per stage.
template <int S>
struct OzWideCfg {
    static constexpr int NT = 128;
    static constexpr int RB = 32;
    static constexpr int GS = S > 4 ? S - 4 : 0;   // first group of pass 1 (0: one pass)
    static constexpr int A_TILE = BM * RB;
    static constexpr int B_TILE = NT * RB;
    static constexpr int STAGE = S * (A_TILE + B_TILE);
    static constexpr int STAGES = (kSmemBudget / STAGE) > 4 ? 4 : (kSmemBudget / STAGE);
    static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
    static constexpr uint32_t LAYOUT = 6u;   // SWIZZLE_32B
    static constexpr uint32_t SBO = 8u * RB;
    static constexpr int RB2 = 64;          // pass 2
    static constexpr int A2_TILE = BM * RB2;
    static constexpr int B2_TILE = NT * RB2;
    static constexpr uint32_t LAYOUT2 = 4u;   // SWIZZLE_64B
    static constexpr uint32_t SBO2 = 8u * RB2;
    // kind::i8: D s32, A and B s8, K-major, N = 128, M = 128
    static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                                      ((uint32_t)(BM >> 4) << 24);
    static_assert((S - GS) * NT <= kTmemCols, "one pass's accumulators fit in tensor memory");
    static_assert(STAGES >= 2, "at least two pipeline stages");
    static_assert(A_TILE % 1024 == 0 && B_TILE % 1024 == 0, "tiles keep the swizzle atoms aligned");
    static_assert(GS * (A2_TILE + B2_TILE) <= STAGE, "pass-2 slices fit a stage");
    // one resident CTA per SM (all 512 TMEM columns: a second CTA would only wait in tcgen05.alloc)
    static_assert(SMEM >= kOneCtaPerSm && SMEM <= kSmemMax, "shared memory keeps the kernel at one CTA per SM");
};

// Bounded wait that also ends when the abort flag is raised; true when the phase completed.
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, const int* abort_flag) {
    const uint64_t t0 = gtimer();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*(volatile const int*)abort_flag) return false;
        if (gtimer() - t0 > kTimeoutNs) return false;
    }
}

// Sum of groups g = g_hi down to g_lo (accumulator of g at column (g - gc) * 128)
// of 32 columns [c0, c0 + 32) into acc, smallest group first.
__device__ __forceinline__ void oz_wide_groups(uint32_t tmem, int q4, int c0, int g_hi, int g_lo, int gc,
                                               double (&acc)[32]) {
#pragma unroll 1
    for (int g = g_hi; g >= g_lo; --g) {
        uint32_t v[32];
        __syncwarp();
        tmem_ld32(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)((g - gc) * 128 + c0), v);
        const double w = pow2i(-7 * (g + 2));
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] += (double)(int)v[j] * w;
    }
}

// Epilogue warps 4..7 of the 128-column kernels (q4 = TMEM lane quarter): pass 1
// drain into the parked partial sums, one arrival per warp on the "free" barrier
// (of the leader CTA, a shared::cluster address, when CLUSTER_ARRIVE), pass 2
// drain continuing the parked sums, fused output and per-CTA stats.
template <int EPI, int S, bool CLUSTER_ARRIVE>
__device__ __forceinline__ void oz_wide_epilogue(const OzEpi& ep, uint32_t tmem, uint32_t accum_bar, uint32_t free_bar,
                                                 int* abort_flag, double* red, int bi, int bj, int q4, int lane,
                                                 int nk, const int* __restrict__ ea, const int* __restrict__ eb) {
    constexpr int GS = OzWideCfg<S>::GS;
    constexpr int NT = OzWideCfg<S>::NT;
    const int64_t n = ep.n, r = (int64_t)bi * BM + q4 * 32 + lane;
    const int64_t ld = ep.ors;
    double tr = 0.0, ss = 0.0, dlo = 0.0;
    bool live = true;
    if constexpr (GS > 0) {
        const bool ok = __all_sync(0xffffffffu, mbar_wait_or_abort(accum_bar, 0, abort_flag));
        const int aborted = __shfl_sync(0xffffffffu, *(volatile int*)abort_flag, 0);
        tc_fence_after();
        if (!ok && !aborted && lane == 0) set_err(ep.err, 180);
        live = ok && !aborted;
        if (live) {
#pragma unroll 1
            for (int c0 = 0; c0 < NT; c0 += 32) {
                double acc[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) acc[j] = 0.0;
                oz_wide_groups(tmem, q4, c0, S - 1, GS, GS, acc);
                const int64_t cb = (int64_t)bj * NT + c0;
                if (r < n) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int64_t c = cb + j;
                        if (c >= n) continue;
                        if (EPI == OZ_OUT) ep.out[r * ep.ors + c * ep.ocs] = acc[j];
                        else if (c > r) ep.out[c + r * ld] = acc[j];
                        else if (c == r) dlo = acc[j];
                    }
                }
            }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
            if constexpr (CLUSTER_ARRIVE)
                asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(free_bar) : "memory");
            else
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(free_bar) : "memory");
        }
    }
    if (live) {
        const uint32_t par = GS > 0 ? 1u : 0u;
        const bool ok = __all_sync(0xffffffffu, mbar_wait_or_abort(accum_bar, par, abort_flag));
        const int aborted = __shfl_sync(0xffffffffu, *(volatile int*)abort_flag, 0);
        tc_fence_after();
        if (!ok && !aborted && lane == 0) set_err(ep.err, 181);
        if (ok && !aborted) {
            const int er = r < n ? ea[r] : 0;
#pragma unroll 1
            for (int c0 = 0; c0 < NT; c0 += 32) {
                double acc[32];
                const int64_t cb = (int64_t)bj * NT + c0;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int64_t c = cb + j;
                    double v = 0.0;
                    if (GS > 0 && r < n && c < n) {
                        if (EPI == OZ_OUT) v = ep.out[r * ep.ors + c * ep.ocs];
                        else if (c > r) v = ep.out[c + r * ld];
                        else if (c == r) v = dlo;
                    }
                    acc[j] = v;
                }
                if (GS > 0) oz_wide_groups(tmem, q4, c0, GS - 1, 0, 0, acc);
                else oz_wide_groups(tmem, q4, c0, S - 1, 0, 0, acc);
                if (nk == 0) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[j] = 0.0;
                }
                oz_write<EPI, 32>(ep, r, cb, acc, er, eb, tr, ss);
            }
        }
    }
    if (EPI == OZ_SYM && ep.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            tr += __shfl_xor_sync(0xffffffffu, tr, o);
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
        }
        if (lane == 0) {
            red[2 * q4] = tr;
            red[2 * q4 + 1] = ss;
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");   // epilogue warps only
        if (q4 == 0 && lane == 0) {
            ep.stats[2 * blockIdx.x] = red[0] + red[2] + red[4] + red[6];
            ep.stats[2 * blockIdx.x + 1] = red[1] + red[3] + red[5] + red[7];
        }
    }
}

template <int EPI, int S>
__global__ void __launch_bounds__(THREADS, 1)
    k_oz_product_w(const __grid_constant__ OzMaps maps, const int4* __restrict__ tiles, const int* __restrict__ ea,
                   const int* __restrict__ eb, OzEpi ep) {
    using C = OzWideCfg<S>;
    constexpr int STAGE = C::STAGE;
    constexpr int STAGES = C::STAGES;
    constexpr int GS = C::GS;
    constexpr int NT = C::NT;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - base_raw);
    const uint32_t bar0 = base + STAGES * STAGE;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
    const uint32_t accum_bar = bar0 + 8u * (2 * STAGES);
    const uint32_t free_bar = bar0 + 8u * (2 * STAGES + 1);   // pass-1 accumulators drained
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE + 8 * (2 * STAGES + 2));
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(gbase + STAGES * STAGE + 128);   // 8 doubles

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int4 tile = tiles[blockIdx.x];
    const int bi = tile.x, bj = tile.y;
    const int nk = (tile.w - tile.z) / C::RB;                  // K steps of pass 1
    const int nk2 = GS > 0 ? (tile.w - tile.z) / C::RB2 : 0;   // K steps of pass 2
    const int ntot = nk + nk2;

    auto a_tile = [&](int s, int p) { return base + s * STAGE + p * C::A_TILE; };
    auto b_tile = [&](int s, int q) { return base + s * STAGE + S * C::A_TILE + q * C::B_TILE; };
    auto a2_tile = [&](int s, int p) { return base + s * STAGE + p * C::A2_TILE; };
    auto b2_tile = [&](int s, int q) { return base + s * STAGE + GS * C::A2_TILE + q * C::B2_TILE; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(accum_bar, 1);
        mbar_init(free_bar, 4);   // one arrival per epilogue warp
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"((uint32_t)kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer: pass 1 (all S slices), pass 2 (slices 0..GS-1) ----------------
        int issued_phase[STAGES];
        for (int s = 0; s < STAGES; ++s) issued_phase[s] = -1;
        for (int it = 0; it < ntot; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (round > 0 && !mbar_wait(empty_bar(s), (round - 1) & 1)) {
                set_err(ep.err, 161);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            if (it < nk) {
                mbar_expect_tx(full_bar(s), (uint32_t)(S * (C::A_TILE + C::B_TILE)));
                const int kx = tile.z + it * C::RB;
                for (int p = 0; p < S; ++p)
                    tma_load_2d(a_tile(s, p), &maps.a, full_bar(s), kx, (int)(p * ep.ldp) + bi * BM);
                for (int q = 0; q < S; ++q)
                    tma_load_2d(b_tile(s, q), &maps.b, full_bar(s), kx, (int)(q * ep.ldp) + bj * NT);
            } else {
                mbar_expect_tx(full_bar(s), (uint32_t)(GS * (C::A2_TILE + C::B2_TILE)));
                const int kx = tile.z + (it - nk) * C::RB2;
                for (int p = 0; p < GS; ++p)
                    tma_load_2d(a2_tile(s, p), &maps.a2, full_bar(s), kx, (int)(p * ep.ldp) + bi * BM);
                for (int q = 0; q < GS; ++q)
                    tma_load_2d(b2_tile(s, q), &maps.b2, full_bar(s), kx, (int)(q * ep.ldp) + bj * NT);
            }
            issued_phase[s] = round & 1;
        }
        for (int s = 0; s < STAGES; ++s)
            if (issued_phase[s] >= 0 && !mbar_wait(full_bar(s), (uint32_t)issued_phase[s])) set_err(ep.err, 162);
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        int commits = 0;
        for (int it = 0; it < ntot; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            const bool pass2 = GS > 0 && it >= nk;
            if (GS > 0 && it == nk) {
                // end of pass 1: hand the accumulators to the epilogue, wait until drained
                umma_commit(accum_bar);
                ++commits;
                if (!mbar_wait_or_abort(free_bar, 0, abort_flag)) {
                    set_err(ep.err, 173);
                    *(volatile int*)abort_flag = 1;
                    break;
                }
                tc_fence_after();
            }
            if (!mbar_wait(full_bar(s), round & 1)) {
                set_err(ep.err, 171);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            tc_fence_after();
            const int itp = pass2 ? it - nk : it;
            if (!pass2) {
#pragma unroll
                for (int p = 0; p < S; ++p) {
                    const uint64_t ad = sdesc(a_tile(s, p), C::SBO, C::LAYOUT);
#pragma unroll
                    for (int q = (GS - p > 0 ? GS - p : 0); q < S - p; ++q) {
                        const uint64_t bd = sdesc(b_tile(s, q), C::SBO, C::LAYOUT);
                        // p = 0 opens every accumulator of the pass on its first K step
                        umma_i8(tmem + (uint32_t)((p + q - GS) * NT), ad, bd, C::IDESC, (itp | p) != 0);
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < C::RB2 / 32; ++k) {
#pragma unroll
                    for (int p = 0; p < GS; ++p) {
                        const uint64_t ad = sdesc(a2_tile(s, p) + k * 32, C::SBO2, C::LAYOUT2);
#pragma unroll
                        for (int q = 0; q < GS - p; ++q) {
                            const uint64_t bd = sdesc(b2_tile(s, q) + k * 32, C::SBO2, C::LAYOUT2);
                            umma_i8(tmem + (uint32_t)((p + q) * NT), ad, bd, C::IDESC, (itp | k | p) != 0);
                        }
                    }
                }
            }
            umma_commit(empty_bar(s));
        }
        if (GS > 0 && nk == 0) {   // empty K range: both epilogue phases still complete
            umma_commit(accum_bar);
            ++commits;
            if (!mbar_wait_or_abort(free_bar, 0, abort_flag)) set_err(ep.err, 174);
        }
        umma_commit(accum_bar);
        ++commits;
        // every MMA of the tile has completed before the block tears down
        if (!mbar_wait(accum_bar, (uint32_t)((commits - 1) & 1))) set_err(ep.err, 175);
    } else if (warp >= 4) {
        oz_wide_epilogue<EPI, S, false>(ep, tmem, accum_bar, free_bar, abort_flag, red, bi, bj, warp - 4, lane, nk, ea,
                                        eb);
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols));
    }
}

// The 128-column two-pass kernel on a CTA pair (cta_group::2, cluster of two):
// one 256 x 128 tile per pair, UMMA 256x128x32 int8 issued by the leader CTA.
// CTA r holds rows 128r..128r+127 of the A slices and of the accumulators and
// rows 64r..64r+63 of the 128 B rows, so each SM loads its A slices and half
// the B slices: 6 KB instead of 8 KB per slice pair and K32 step, which the
// one-CTA form draws from L2 at up to ~60 % of its throughput.  Both CTAs' TMA
// loads count on the leader's "full" barrier (armed with both CTAs' bytes), the
// leader's commits arrive on both CTAs' "empty" and accumulator barriers, and
// both CTAs' epilogue warps arrive on the leader's "free" barrier after the
// pass-1 drain (8 arrivals) before the leader starts pass 2.  Same passes,
// parking and FP64 order as the one-CTA form: bit-identical results.
template <int S>
struct OzWidePairCfg {
    static constexpr int NT = 128;
    static constexpr int RB = 32, RB2 = 64;
    static constexpr int GS = OzWideCfg<S>::GS;
    static constexpr int A_TILE = BM * RB;
    static constexpr int B_TILE = (NT / 2) * RB;
    static constexpr int A2_TILE = BM * RB2;
    static constexpr int B2_TILE = (NT / 2) * RB2;
    static constexpr int STAGE = S * (A_TILE + B_TILE);
    static constexpr int STAGES = (kSmemBudget / STAGE) > 4 ? 4 : (kSmemBudget / STAGE);
    static constexpr int SMEM = STAGES * STAGE + 1024 + 256 > kOneCtaPerSm ? STAGES * STAGE + 1024 + 256
                                                                          : kOneCtaPerSm;
    static constexpr uint32_t LAYOUT = 6u, SBO = 8u * RB;      // SWIZZLE_32B
    static constexpr uint32_t LAYOUT2 = 4u, SBO2 = 8u * RB2;   // SWIZZLE_64B
    // kind::i8: D s32, A and B s8, K-major, N = 128, M = 256 (the pair)
    static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                                      ((uint32_t)(256 >> 4) << 24);
    static_assert((S - GS) * NT <= kTmemCols, "one pass's accumulators fit in tensor memory");
    static_assert(STAGES >= 2, "at least two pipeline stages");
    static_assert(A_TILE % 1024 == 0 && B_TILE % 1024 == 0 && B2_TILE % 1024 == 0, "swizzle atoms aligned");
    static_assert(GS * (A2_TILE + B2_TILE) <= STAGE, "pass-2 slices fit a stage");
    static_assert(SMEM >= kOneCtaPerSm && SMEM <= kSmemMax, "one resident CTA per SM");
};

template <int EPI, int S>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
    k_oz_product_wp(const __grid_constant__ OzMaps maps, const int4* __restrict__ pairs,
                    const int* __restrict__ ea, const int* __restrict__ eb, OzEpi ep) {
    using C = OzWidePairCfg<S>;
    constexpr int STAGE = C::STAGE;
    constexpr int STAGES = C::STAGES;
    constexpr int GS = C::GS;
    constexpr int NT = C::NT;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - base_raw);
    const uint32_t bar0 = base + STAGES * STAGE;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
    const uint32_t accum_bar = bar0 + 8u * (2 * STAGES);
    const uint32_t free_bar = bar0 + 8u * (2 * STAGES + 1);   // the leader's: pass-1 accumulators drained
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE + 8 * (2 * STAGES + 2));
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(gbase + STAGES * STAGE + 128);   // 8 doubles

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int4 pt = pairs[blockIdx.x >> 1];
    const int bi = 2 * pt.x + (int)rank, bj = pt.y;
    // an odd row-block count leaves the second half of the last pair past the
    // operand: it loads the first half's rows again and writes nothing
    const int nbi = (int)(ep.ldp / BM);
    const int abi = bi < nbi ? bi : nbi - 1;
    const int nk = (pt.w - pt.z) / C::RB;                  // K steps of pass 1
    const int nk2 = GS > 0 ? (pt.w - pt.z) / C::RB2 : 0;   // K steps of pass 2
    const int ntot = nk + nk2;

    auto a_tile = [&](int s, int p) { return base + s * STAGE + p * C::A_TILE; };
    auto b_tile = [&](int s, int q) { return base + s * STAGE + S * C::A_TILE + q * C::B_TILE; };
    auto a2_tile = [&](int s, int p) { return base + s * STAGE + p * C::A2_TILE; };
    auto b2_tile = [&](int s, int q) { return base + s * STAGE + GS * C::A2_TILE + q * C::B2_TILE; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(accum_bar, 1);
        mbar_init(free_bar, 8);   // four epilogue warps of each CTA (the leader's barrier is used)
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"((uint32_t)kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();   // both CTAs' barriers are initialised before any remote arrive
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        int issued_phase[STAGES];
        for (int s = 0; s < STAGES; ++s) issued_phase[s] = -1;
        for (int it = 0; it < ntot; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            if (round > 0 && !mbar_wait(empty_bar(s), (round - 1) & 1)) {
                set_err(ep.err, 191);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            const uint32_t fb = mapa_shared(full_bar(s), 0);
            if (it < nk) {
                if (rank == 0) mbar_expect_tx(full_bar(s), (uint32_t)(2 * S * (C::A_TILE + C::B_TILE)));
                const int kx = pt.z + it * C::RB;
                for (int p = 0; p < S; ++p)
                    tma_load_2d_pair(a_tile(s, p), &maps.a, fb, kx, (int)(p * ep.ldp) + abi * BM);
                for (int q = 0; q < S; ++q)
                    tma_load_2d_pair(b_tile(s, q), &maps.b, fb, kx,
                                     (int)(q * ep.ldp) + bj * NT + (int)rank * (NT / 2));
            } else {
                if (rank == 0) mbar_expect_tx(full_bar(s), (uint32_t)(2 * GS * (C::A2_TILE + C::B2_TILE)));
                const int kx = pt.z + (it - nk) * C::RB2;
                for (int p = 0; p < GS; ++p)
                    tma_load_2d_pair(a2_tile(s, p), &maps.a2, fb, kx, (int)(p * ep.ldp) + abi * BM);
                for (int q = 0; q < GS; ++q)
                    tma_load_2d_pair(b2_tile(s, q), &maps.b2, fb, kx,
                                     (int)(q * ep.ldp) + bj * NT + (int)rank * (NT / 2));
            }
            issued_phase[s] = round & 1;
        }
        // drain: the leader sees every copy of the pair land on its full barriers;
        // the peer's copies have landed once the leader's MMAs consumed them,
        // which its accumulator barrier (waited by the epilogue) certifies
        if (rank == 0)
            for (int s = 0; s < STAGES; ++s)
                if (issued_phase[s] >= 0 && !mbar_wait(full_bar(s), (uint32_t)issued_phase[s])) set_err(ep.err, 192);
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // ---------------- MMA issuer (leader CTA) ----------------
        int commits = 0;
        for (int it = 0; it < ntot; ++it) {
            const int s = it % STAGES, round = it / STAGES;
            const bool pass2 = GS > 0 && it >= nk;
            if (GS > 0 && it == nk) {
                // end of pass 1: hand the accumulators to both epilogues, wait until both drained
                umma_commit_pair(accum_bar, (uint16_t)0x3);
                ++commits;
                if (!mbar_wait_or_abort(free_bar, 0, abort_flag)) {
                    set_err(ep.err, 203);
                    *(volatile int*)abort_flag = 1;
                    break;
                }
                tc_fence_after();
            }
            if (!mbar_wait(full_bar(s), round & 1)) {
                set_err(ep.err, 201);
                *(volatile int*)abort_flag = 1;
                break;
            }
            if (*(volatile int*)abort_flag) break;
            tc_fence_after();
            const int itp = pass2 ? it - nk : it;
            if (!pass2) {
#pragma unroll
                for (int p = 0; p < S; ++p) {
                    const uint64_t ad = sdesc(a_tile(s, p), C::SBO, C::LAYOUT);
#pragma unroll
                    for (int q = (GS - p > 0 ? GS - p : 0); q < S - p; ++q) {
                        const uint64_t bd = sdesc(b_tile(s, q), C::SBO, C::LAYOUT);
                        umma_i8_pair(tmem + (uint32_t)((p + q - GS) * NT), ad, bd, C::IDESC, (itp | p) != 0);
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < C::RB2 / 32; ++k) {
#pragma unroll
                    for (int p = 0; p < GS; ++p) {
                        const uint64_t ad = sdesc(a2_tile(s, p) + k * 32, C::SBO2, C::LAYOUT2);
#pragma unroll
                        for (int q = 0; q < GS - p; ++q) {
                            const uint64_t bd = sdesc(b2_tile(s, q) + k * 32, C::SBO2, C::LAYOUT2);
                            umma_i8_pair(tmem + (uint32_t)((p + q) * NT), ad, bd, C::IDESC, (itp | k | p) != 0);
                        }
                    }
                }
            }
            umma_commit_pair(empty_bar(s), (uint16_t)0x3);
        }
        if (GS > 0 && nk == 0) {   // empty K range: both epilogue phases still complete
            umma_commit_pair(accum_bar, (uint16_t)0x3);
            ++commits;
            if (!mbar_wait_or_abort(free_bar, 0, abort_flag)) set_err(ep.err, 204);
        }
        umma_commit_pair(accum_bar, (uint16_t)0x3);
        ++commits;
        // every MMA of the pair has completed before either CTA tears down
        if (!mbar_wait(accum_bar, (uint32_t)((commits - 1) & 1))) set_err(ep.err, 205);
    } else if (warp >= 4) {
        oz_wide_epilogue<EPI, S, true>(ep, tmem, accum_bar, mapa_shared(free_bar, 0), abort_flag, red, bi, bj,
                                       warp - 4, lane, nk, ea, eb);
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    cluster_sync();   // the leader's MMAs have finished with the peer's shared and tensor memory
    tc_fence_after();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols));
    }
}

// ---- host side ---------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    PTB_CHECK(fn != nullptr, PTBGPU_ECUDA, "cuTensorMapEncodeTiled unavailable");
    return fn;
}

void encode_planes(CUtensorMap* map, const Operand& op, int box_rows, int rb) {
    PTB_CHECK(((uintptr_t)op.planes & 15) == 0, PTBGPU_EINVAL, "slice planes not 16-byte aligned");
    PTB_CHECK(op.ldp % BM == 0, PTBGPU_EINVAL, "slice leading dimension must be a multiple of 128");
    cuuint64_t dims[2] = {(cuuint64_t)op.ldp, (cuuint64_t)op.ldp * (cuuint64_t)op.S};
    cuuint64_t strides[1] = {(cuuint64_t)op.ldp};
    cuuint32_t box[2] = {(cuuint32_t)rb, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapSwizzle sw = rb == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    CUresult r = get_encode()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, op.planes, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    PTB_CHECK(r == CUDA_SUCCESS, PTBGPU_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
}

template <int EPI, int S, int RB>
void launch_t(cudaStream_t s, const OzMaps& maps, const int4* tiles, int ntiles, const Operand& a,
              const Operand& b, const OzEpi& ep) {
    using C = OzCfg<S, RB>;
    static const bool attr = [] {   // thread-safe one-time setup
        PTB_CUDA(cudaFuncSetAttribute(k_oz_product<EPI, S, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      C::SMEM));
        return true;
    }();
    (void)attr;
    k_oz_product<EPI, S, RB><<<ntiles, THREADS, C::SMEM, s>>>(maps, tiles, a.exps, b.exps, ep);
    count_launch();
}

template <int EPI, int S, int RB>
void launch_p(cudaStream_t s, const OzMaps& maps, const int4* pairs, int npairs, const Operand& a,
              const Operand& b, const OzEpi& ep) {
    using C = OzPairCfg<S, RB>;
    static const bool attr = [] {   // thread-safe one-time setup
        PTB_CUDA(cudaFuncSetAttribute(k_oz_product_pair<EPI, S, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      C::SMEM));
        return true;
    }();
    (void)attr;
    k_oz_product_pair<EPI, S, RB><<<2 * npairs, THREADS, C::SMEM, s>>>(maps, pairs, a.exps, b.exps, ep);
    count_launch();
}

template <int EPI, int S>
void launch_w(cudaStream_t s, const OzMaps& maps, const int4* tiles, int ntiles, const Operand& a,
              const Operand& b, const OzEpi& ep) {
    using C = OzWideCfg<S>;
    static const bool attr = [] {   // thread-safe one-time setup
        PTB_CUDA(cudaFuncSetAttribute(k_oz_product_w<EPI, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
        return true;
    }();
    (void)attr;
    k_oz_product_w<EPI, S><<<ntiles, THREADS, C::SMEM, s>>>(maps, tiles, a.exps, b.exps, ep);
    count_launch();
}

template <int EPI, int S>
void launch_wp(cudaStream_t s, const OzMaps& maps, const int4* pairs, int npairs, const Operand& a,
               const Operand& b, const OzEpi& ep) {
    using C = OzWidePairCfg<S>;
    static const bool attr = [] {   // thread-safe one-time setup
        PTB_CUDA(cudaFuncSetAttribute(k_oz_product_wp<EPI, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
        return true;
    }();
    (void)attr;
    k_oz_product_wp<EPI, S><<<2 * npairs, THREADS, C::SMEM, s>>>(maps, pairs, a.exps, b.exps, ep);
    count_launch();
}

constexpr int ta_tile_n(int S) { return S >= 7 ? 48 : 64; }

template <int EPI, int S, int RB>
void launch_ta(cudaStream_t s, const OzMaps& maps, const int4* tiles, int ntiles, const Operand& a,
               const Operand& b, const OzEpi& ep) {
    constexpr int NT = ta_tile_n(S);
    constexpr int STAGE = S * (BM * RB + NT * RB);
    constexpr int STAGES = (kSmemBudget / STAGE) > 4 ? 4 : (kSmemBudget / STAGE);
    constexpr int SMEM = STAGES * STAGE + 1024 + 256;
    static const bool attr = [] {   // thread-safe one-time setup
        PTB_CUDA(cudaFuncSetAttribute(k_oz_product_ta<EPI, S, RB, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      SMEM));
        return true;
    }();
    (void)attr;
    k_oz_product_ta<EPI, S, RB, NT><<<ntiles, THREADS, SMEM, s>>>(maps, tiles, a.exps, b.exps, ep);
    count_launch();
}

template <int EPI, int S>
void launch_s(cudaStream_t s, int rb, int variant, const OzMaps& maps, const int4* tiles, int ntiles,
              const Operand& a, const Operand& b, const OzEpi& ep) {
    if (variant == V_TMEM_A) {
        if (rb == 64) launch_ta<EPI, S, 64>(s, maps, tiles, ntiles, a, b, ep);
        else launch_ta<EPI, S, 32>(s, maps, tiles, ntiles, a, b, ep);
    } else if (variant == V_PAIR) {
        if (rb == 64) launch_p<EPI, S, 64>(s, maps, tiles, ntiles, a, b, ep);
        else launch_p<EPI, S, 32>(s, maps, tiles, ntiles, a, b, ep);
    } else if (variant == V_WIDE) {
        launch_w<EPI, S>(s, maps, tiles, ntiles, a, b, ep);
    } else if (variant == V_WPAIR) {
        launch_wp<EPI, S>(s, maps, tiles, ntiles, a, b, ep);
    } else {
        if (rb == 64) launch_t<EPI, S, 64>(s, maps, tiles, ntiles, a, b, ep);
        else launch_t<EPI, S, 32>(s, maps, tiles, ntiles, a, b, ep);
    }
}

template <int EPI>
void launch_e(cudaStream_t s, int S, int rb, int variant, const OzMaps& maps, const int4* tiles, int ntiles,
              const Operand& a, const Operand& b, const OzEpi& ep) {
    switch (S) {
        case 4: launch_s<EPI, 4>(s, rb, variant, maps, tiles, ntiles, a, b, ep); break;
        case 6: launch_s<EPI, 6>(s, rb, variant, maps, tiles, ntiles, a, b, ep); break;
        case 7: launch_s<EPI, 7>(s, rb, variant, maps, tiles, ntiles, a, b, ep); break;
        case 8: launch_s<EPI, 8>(s, rb, variant, maps, tiles, ntiles, a, b, ep); break;
        default: PTB_CHECK(false, PTBGPU_EINVAL, "unsupported slice count %d (4, 6, 7 or 8)", S);
    }
}

}  // namespace

int64_t max_k(int S) { return (int64_t)2147483647 / ((int64_t)S * 127 * 127); }
int64_t padded(int64_t n) { return round_up(n, BM); }
bool supported(int64_t n, int S) { return (S == 4 || (S >= 6 && S <= 8)) && padded(n) <= max_k(S); }

void slice(cudaStream_t s, const double* M, int64_t rs, int64_t cs, int64_t n, int tri, const Operand& op,
           unsigned long long* rowmax) {
    PTB_CHECK(rs == 1 || cs == 1, PTBGPU_EINVAL, "slicing needs rows or columns contiguous");
    PTB_CHECK(op.ldp >= n && op.ldp % BM == 0, PTBGPU_EINVAL, "bad slice leading dimension");
    PTB_CUDA(cudaMemsetAsync(rowmax, 0, sizeof(unsigned long long) * (size_t)op.ldp, s));
    const dim3 g1((unsigned)((n + 127) / 128), (unsigned)((n + 31) / 32));
    k_oz_rowmax<<<g1, THREADS, 0, s>>>(M, rs, cs, n, tri, rowmax);
    count_launch();
    const dim3 g2((unsigned)(op.ldp / 64), (unsigned)(op.ldp / 32));
    switch (op.S) {
        case 4: k_oz_slice<4><<<g2, THREADS, 0, s>>>(M, rs, cs, n, tri, rowmax, op.planes, op.exps, op.ldp); break;
        case 6: k_oz_slice<6><<<g2, THREADS, 0, s>>>(M, rs, cs, n, tri, rowmax, op.planes, op.exps, op.ldp); break;
        case 7: k_oz_slice<7><<<g2, THREADS, 0, s>>>(M, rs, cs, n, tri, rowmax, op.planes, op.exps, op.ldp); break;
        case 8: k_oz_slice<8><<<g2, THREADS, 0, s>>>(M, rs, cs, n, tri, rowmax, op.planes, op.exps, op.ldp); break;
        default: PTB_CHECK(false, PTBGPU_EINVAL, "unsupported slice count %d (4, 6, 7 or 8)", op.S);
    }
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

int resolve_variant(int variant, int S, int rb) {
    if (variant != V_DEFAULT) return variant;
    // 128-column tiles on a CTA pair measured x1.21-1.29 faster than 128 x 64 tiles
    // with 6, 7 or 8 slices at ndim 4096-11776 (N = 128 MMAs: x1.09-1.22 on one CTA;
    // the pair halves the B loads per SM); they take 32-byte K blocks only
    return S >= 6 && rb != 64 ? V_WPAIR : V_SMEM_A;
}

int tile_n(int S, int variant) {
    PTB_CHECK(variant != V_DEFAULT, PTBGPU_EINVAL, "kernel variant not resolved");
    return variant == V_TMEM_A ? ta_tile_n(S) : (variant == V_WIDE || variant == V_WPAIR) ? 128 : BN;
}

std::vector<int4> make_tiles(int64_t ldp, bool upper, int a_tri, int b_tri, int bn) {
    PTB_CHECK(bn == 128 || bn == 64 || bn == 48, PTBGPU_EINVAL, "tile width must be 128, 64 or 48");
    // column tiles may overhang ldp (the operand rows there are padding or the
    // next plane; those columns are never written)
    const int nbi = (int)(ldp / BM), nbj = (int)((ldp + bn - 1) / bn);
    std::vector<int4> t;
    const int G = 16;
    for (int g0 = 0; g0 < nbi; g0 += G)
        for (int bj = 0; bj < nbj; ++bj)
            for (int bi = g0; bi < std::min(nbi, g0 + G); ++bi) {
                if (upper && (int64_t)bj * bn + bn - 1 < (int64_t)bi * BM) continue;
                int64_t k0 = 0, k1 = ldp;
                // K ranges in whole 128-blocks: the masked triangle reads as zero beyond
                if (a_tri == TRI_LOWER) k1 = std::min<int64_t>(k1, (int64_t)(bi + 1) * BM);
                if (a_tri == TRI_UPPER) k0 = std::max<int64_t>(k0, (int64_t)bi * BM);
                if (b_tri == TRI_LOWER) k1 = std::min<int64_t>(k1, round_up((int64_t)(bj + 1) * bn, BM));
                if (b_tri == TRI_UPPER) k0 = std::max<int64_t>(k0, (int64_t)bj * bn / BM * BM);
                PTB_CHECK(k1 > k0, PTBGPU_EINVAL, "empty K range in a tile");
                t.push_back(make_int4(bi, bj, (int)k0, (int)k1));
            }
    std::stable_sort(t.begin(), t.end(), [](const int4& x, const int4& y) { return x.w - x.z > y.w - y.z; });
    return t;
}

std::vector<int4> make_pair_tiles(int64_t ldp, bool upper, int a_tri, int b_tri, int bn) {
    PTB_CHECK(bn == 64 || bn == 128, PTBGPU_EINVAL, "pair tiles are 64 or 128 columns wide");
    const std::vector<int4> one = make_tiles(ldp, upper, a_tri, b_tri, bn);
    const int nbi = (int)(ldp / BM), nbj = (int)(ldp / bn), np = (nbi + 1) / 2;
    // K range of each (pair, bj) over the halves make_tiles keeps; k1 = 0: none kept
    std::vector<int2> kr((size_t)np * nbj, make_int2(INT_MAX, 0));
    for (const int4& x : one) {
        int2& r = kr[(size_t)(x.x / 2) * nbj + x.y];
        r.x = std::min(r.x, x.z);
        r.y = std::max(r.y, x.w);
    }
    std::vector<int4> t;
    const int G = 8;   // pair blocks per column sweep (16 row blocks, as make_tiles)
    for (int g0 = 0; g0 < np; g0 += G)
        for (int bj = 0; bj < nbj; ++bj)
            for (int p = g0; p < std::min(np, g0 + G); ++p) {
                const int2 r = kr[(size_t)p * nbj + bj];
                if (r.y > 0) t.push_back(make_int4(p, bj, r.x, r.y));
            }
    std::stable_sort(t.begin(), t.end(), [](const int4& x, const int4& y) { return x.w - x.z > y.w - y.z; });
    return t;
}

std::vector<int4> build_tiles(int64_t ldp, bool upper, int a_tri, int b_tri, int S, int variant) {
    return (variant == V_PAIR || variant == V_WPAIR) ? make_pair_tiles(ldp, upper, a_tri, b_tri, tile_n(S, variant))
                                                     : make_tiles(ldp, upper, a_tri, b_tri, tile_n(S, variant));
}

int grid_ctas(int ntiles, int variant) { return (variant == V_PAIR || variant == V_WPAIR) ? 2 * ntiles : ntiles; }

double tile_ops(const std::vector<int4>& tiles, int S, int variant) {
    double kk = 0.0;
    for (const int4& x : tiles) kk += (double)(x.w - x.z);
    const int rows = (variant == V_PAIR || variant == V_WPAIR) ? 2 * BM : BM;
    return 2.0 * rows * tile_n(S, variant) * kk * (double)(S * (S + 1) / 2);
}

void product(cudaStream_t s, int epi, const Operand& a, const Operand& b, const int4* tiles_dev, int ntiles,
             const OzEpi& ep, int rb, int variant) {
    PTB_CHECK(variant == V_SMEM_A || variant == V_TMEM_A || variant == V_PAIR || variant == V_WIDE ||
                  variant == V_WPAIR,
              PTBGPU_EINVAL, "bad kernel variant %d", variant);
    if (variant == V_WIDE || variant == V_WPAIR) {
        PTB_CHECK(rb == 0 || rb == 32, PTBGPU_EINVAL, "the 128-column kernel takes 32-byte K blocks");
        rb = 32;
    }
    if (rb == 0) rb = 64;   // measured faster than 32 at ndim 11776 (S = 7 and 8)
    PTB_CHECK(rb == 32 || rb == 64, PTBGPU_EINVAL, "K block must be 32 or 64 bytes");
    PTB_CHECK(a.S == b.S && a.ldp == b.ldp && a.ldp == ep.ldp, PTBGPU_EINVAL, "operands do not match");
    PTB_CHECK(a.ldp <= max_k(a.S), PTBGPU_EINVAL, "dimension %lld too large for exact int32 sums with %d slices",
              (long long)a.ldp, a.S);
    PTB_CHECK(epi == OZ_OUT || epi == OZ_SYM, PTBGPU_EINVAL, "bad epilogue");
    if (ntiles == 0) return;
    OzMaps maps{};
    encode_planes(&maps.a, a, BM, rb);
    // a CTA pair splits the B rows of a tile between its two CTAs
    const bool pair = variant == V_PAIR || variant == V_WPAIR;
    const int brows = pair ? tile_n(a.S, variant) / 2 : tile_n(a.S, variant);
    encode_planes(&maps.b, b, brows, rb);
    if (variant == V_WIDE || variant == V_WPAIR) {   // the second pass takes 64-byte K blocks
        encode_planes(&maps.a2, a, BM, 64);
        encode_planes(&maps.b2, b, brows, 64);
    }
    if (epi == OZ_OUT) launch_e<OZ_OUT>(s, a.S, rb, variant, maps, tiles_dev, ntiles, a, b, ep);
    else launch_e<OZ_SYM>(s, a.S, rb, variant, maps, tiles_dev, ntiles, a, b, ep);
    PTB_CUDA(cudaGetLastError());
}

}  // namespace oz
}  // namespace ptb
