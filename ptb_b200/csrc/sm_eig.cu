// Batched FP64 generalized eigensolver of the submatrix method, one CTA per
// submatrix.
//
// The reference solves H_k U = S_k U diag(e) with LAPACK dsygvd per submatrix
// (la_sygvd, source/sm.f90:296-299), forms S_k U for the electron-count
// weights fe (source/sm.f90:305-310) and, at the final chemical potential,
// P_k = U occ U^T of which only the owned columns are kept
// (source/sm.f90:343-362).  Only these quantities leave the solver, and all of
// them are reached without forming U:
//
//   S_k = L L^T                      Cholesky, blocked (k_eig_potrf)
//   C   = L^-1 H_k L^-T              two blocked triangular solves
//   C   = Q T Q^T                    Householder tridiagonalisation, lower,
//                                    Q = H_0 H_1 ... H_{m-3} (k_eig_sytrd)
//   T   = Z diag(e) Z^T              divide and conquer (k_eig_dc)
//   U   = L^-T Q Z                   never formed:
//     rows c of U    = (L^-T)[c,:] Q Z,  rows c of S U = L[c,:] Q Z  for the
//     owned columns c (k_eig_rows), so fe_j = sum_c (SU)[c,j] U[c,j];
//     P_k[:,c] = U (occ o U[c,:]^T) = L^-T (Q (Z w)) (k_eig_final).
//
// Each step's quantities are summed in a fixed order, so results do not depend
// on scheduling.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "sm_eig.cuh"

namespace ptb {

namespace cg = cooperative_groups;

namespace {

constexpr int kT = 512;           // threads of the per-problem CTAs (16 warps)
constexpr int NB = 32;            // panel width of the blocked stages
constexpr int TS = 64;            // output tile of the blocked updates
constexpr int kQlMaxIter = 30;    // QL sweeps per eigenvalue of a leaf before giving up (as LAPACK's dsteqr)

// Status words per problem.
constexpr int kStOk = 0;
constexpr int kStNoConv = -1;     // a leaf's QL sweeps exhausted
// > 0: leading minor of that order of S_k is not positive definite

struct EigProb {
    int k, m, nown;
    int kind;             // 0: H U = S U e; 1: standard problem (S not read, L = I)
    int mode;             // 0: eigenvalues, fe, owned rows; 2: density 2 U_occ U_occ^T (m x m at boff)
    int nocc;             // mode 2: occupied eigenvectors (the lowest)
    int64_t moff, eoff, o0;
    int64_t gbase, gld;   // the problem's H / S: element (i, j) at gbase + map(i) + map(j) gld
    int64_t poff;         // dense output of the owned columns of P (m x nown, column-major)
    int64_t aoff;     // C, L, Z and merge-workspace arenas (m x m, column-major, ld = m)
    int64_t voff;     // d, e, tau, eigenvalue arenas (m)
    int64_t boff;     // owned-row arena (4 nown x m)
    int64_t xoff;     // cluster solver scratch (orders above kEigBatchMax)
    int64_t koff;     // T of the compact WY panels (t_panels(m) x NB^2)
};

// ---------------------------------------------------------------------------
// Tile products on the FP64 tensor cores: one TS x TS output tile per CTA, the
// K range staged through shared memory in NB-deep chunks (the next chunk's
// loads in flight in registers while the current one is multiplied), each of
// the 16 warps owning a 16 x 16 block of the tile as 2 x 2 fragments of
// mma.m8n8k4.f64 (A fragment: lane holds A[g][t4]; B fragment: B[t4][g];
// accumulator: C[g][2 t4 + h], g = lane / 4, t4 = lane % 4).
//   A(i, k) = AT ? A[kg + (r0+i) lda] : A[(r0+i) + kg lda],   kg = kx ? kx[k] : k
//   B(k, j) = BT ? B[(c0+j) + kg ldb] : B[kg + (c0+j) ldb],   kg = kxb ? kxb[k] : k
//   MMA_SET: C[crow + r0 + i, col] = sum_k A(i,k) B(k,j); MMA_SUB: C[...] -= sum;
//   col = ccol ? ccol[c0+j] : c0+j; LOWER: only r0+i >= c0+j is written.
// Staged layouts keep both the stores (contiguous global runs) and the
// fragment reads free of bank conflicts: the operand whose global run is along
// the tile edge is stored k-major with row stride 68, the other edge-major with
// stride 36 (both = 4 mod 16 doubles).
constexpr int kStageOp = 2304;   // doubles of one staged operand chunk (max of 32 x 68 and 64 x 36)
enum { MMA_SET = 0, MMA_SUB = 1 };

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}
template <bool AT>
__device__ __forceinline__ int sa_idx(int i, int k) {
    return AT ? i * 36 + k : k * 68 + i;
}
template <bool BT>
__device__ __forceinline__ int sb_idx(int k, int j) {
    return BT ? k * 68 + j : j * 36 + k;
}

// AREF / BREF: the operand is a panel of Householder reflectors stored as
// below, read with its implicit structure (1 where the row equals the
// reflector's index, the stored value below it, 0 above): A(i, k) is reflector
// r0+i at row k when AT, row r0+i of reflector k otherwise; B(k, j) is row k of
// reflector c0+j.
template <bool AT, bool BT, int MODE, bool LOWER, bool AREF = false, bool BREF = false>
__device__ void tile_mma(double* __restrict__ C, int64_t ldc, int crow, const int* ccol, int r0, int c0, int mr,
                         int nc, const double* __restrict__ A, int64_t lda, const int* kx,
                         const double* __restrict__ B, int64_t ldb, const int* kxb, int K, double* sA, double* sB) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int wr = (warp & 3) * 16, wc = (warp >> 2) * 16;
    double acc[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    constexpr int kPer = TS * NB / kT;   // staged elements of A (and of B) per thread
    double ra[kPer], rb[kPer];
    auto fetch = [&](int k0) {
        const int kk = min(NB, K - k0);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int t = tid + q * kT;
            const int i = AT ? t / NB : t % TS, k = AT ? t % NB : t / TS;
            double v = 0.0;
            if (i < mr && k < kk) {
                const int64_t kg = kx ? kx[k0 + k] : (k0 + k);
                if (AREF) {
                    const int64_t ig = r0 + i;   // AT: reflector ig at row kg; else row ig of reflector kg
                    const int64_t row = AT ? kg : ig, refl = AT ? ig : kg;
                    v = (row == refl) ? 1.0 : (row > refl ? A[row + refl * lda] : 0.0);
                } else {
                    v = AT ? A[kg + (int64_t)(r0 + i) * lda] : A[(int64_t)(r0 + i) + kg * lda];
                }
            }
            ra[q] = v;
            const int j = BT ? t % TS : t / NB, kb = BT ? t / TS : t % NB;
            double w = 0.0;
            if (j < nc && kb < kk) {
                const int64_t kg = kxb ? kxb[k0 + kb] : (k0 + kb);
                if (BREF) {
                    const int64_t refl = c0 + j;
                    w = (kg == refl) ? 1.0 : (kg > refl ? B[kg + refl * ldb] : 0.0);
                } else {
                    w = BT ? B[(int64_t)(c0 + j) + kg * ldb] : B[kg + (int64_t)(c0 + j) * ldb];
                }
            }
            rb[q] = w;
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int t = tid + q * kT;
            const int i = AT ? t / NB : t % TS, k = AT ? t % NB : t / TS;
            sA[sa_idx<AT>(i, k)] = ra[q];
            const int j = BT ? t % TS : t / NB, kb = BT ? t / TS : t % NB;
            sB[sb_idx<BT>(kb, j)] = rb[q];
        }
    };
    fetch(0);
    stash();
    __syncthreads();
    for (int k0 = 0; k0 < K; k0 += NB) {
        const bool more = k0 + NB < K;
        if (more) fetch(k0 + NB);
        const int ksteps = (min(NB, K - k0) + 3) >> 2;
        for (int ks = 0; ks < ksteps; ++ks) {
            const int k = ks * 4 + t4;
            const double a0 = sA[sa_idx<AT>(wr + g, k)], a1 = sA[sa_idx<AT>(wr + 8 + g, k)];
            const double b0 = sB[sb_idx<BT>(k, wc + g)], b1 = sB[sb_idx<BT>(k, wc + 8 + g)];
            dmma(acc[0][0][0], acc[0][0][1], a0, b0);
            dmma(acc[0][1][0], acc[0][1][1], a0, b1);
            dmma(acc[1][0][0], acc[1][0][1], a1, b0);
            dmma(acc[1][1][0], acc[1][1][1], a1, b1);
        }
        __syncthreads();
        if (more) {
            stash();
            __syncthreads();
        }
    }
    // accumulator acc[a][b][h] is C(wr + 8a + g, wc + 8b + 2 t4 + h); for a
    // read-modify-write every load is issued before any store
    double cv[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = wr + 8 * a + g, j = wc + 8 * b + 2 * t4 + h;
                const bool ok = i < mr && j < nc && !(LOWER && r0 + i < c0 + j);
                cv[a][b][h] = 0.0;
                if (MODE == MMA_SUB && ok) {
                    const int64_t col = ccol ? ccol[c0 + j] : (c0 + j);
                    cv[a][b][h] = C[(int64_t)(crow + r0 + i) + col * ldc];
                }
            }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = wr + 8 * a + g, j = wc + 8 * b + 2 * t4 + h;
                const bool ok = i < mr && j < nc && !(LOWER && r0 + i < c0 + j);
                if (ok) {
                    const int64_t col = ccol ? ccol[c0 + j] : (c0 + j);
                    C[(int64_t)(crow + r0 + i) + col * ldc] =
                        (MODE == MMA_SUB) ? cv[a][b][h] - acc[a][b][h] : acc[a][b][h];
                }
            }
    __syncthreads();
}

// C[r0+i, c0+j] -= sum_{k < kk} A(i,k) B(k,j) on one TS x TS tile (mr x nc
// valid):  A(i,k) = A[(r0+i) + k lda],  B(k,j) = BT ? B[(c0+j) + k ldb] : B[k + (c0+j) ldb].
// LOWER: only elements on or below the diagonal of C are written.
template <bool BT, bool LOWER>
__device__ void tile_update(double* __restrict__ C, int ldc, int r0, int c0, int mr, int nc,
                            const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb, int kk,
                            double* sA, double* sB) {
    tile_mma<false, BT, MMA_SUB, LOWER>(C, ldc, 0, nullptr, r0, c0, mr, nc, A, lda, nullptr, B, ldb, nullptr, kk,
                                        sA, sB);
}

// Fixed-order sum over the CTA (every thread gets the result).
__device__ double cta_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
    __syncthreads();
    return s;
}

__device__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// Shared memory of the stages, carved from one dynamic buffer: the tile
// staging (sA, sB), the diagonal block of the blocked factorisations (sD), a
// union region (the tridiagonalisation's vectors or the divide and conquer's
// per-element arrays, M = the largest order of the batch) and a few scalars.
struct StageSmem {
    double *sA, *sB, *sD;
    unsigned char* uni;
    int* ints;      // 16
    double* dsc;    // 2 + kT / 32
    int M;
};

// ---------------------------------------------------------------------------
// Gather H_k, S_k (source/sm.f90:240-246) into the C and L arenas.
__device__ void stage_gather(const EigProb& p, const int* __restrict__ maps, const double* __restrict__ H,
                             const double* __restrict__ S, double* __restrict__ Ca, double* __restrict__ La) {
    const int m = p.m;
    const int* mp = maps + p.moff;
    double* C = Ca + p.aoff;
    double* L = La + p.aoff;
    for (int j = 0; j < m; ++j) {
        const int64_t gj = p.gbase + (int64_t)mp[j] * p.gld;
        for (int i = threadIdx.x; i < m; i += kT) {
            const int64_t g = (int64_t)mp[i] + gj;
            C[i + (int64_t)j * m] = H[g];
            L[i + (int64_t)j * m] = S[g];
        }
    }
}

// ---------------------------------------------------------------------------
// S_k = L L^T in place (lower), right-looking with 32-wide panels; the strict
// upper triangle is zeroed.  Returns the order of the first non-positive
// pivot (0: positive definite).
__device__ int stage_potrf(const EigProb& p, double* __restrict__ La, const StageSmem& sh) {
    double* sA = sh.sA;
    double* sB = sh.sB;
    double* sD = sh.sD;   // sD[i + j*(NB+1)]
    int& fail = sh.ints[0];
    const int m = p.m;
    double* L = La + p.aoff;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail = 0;
    __syncthreads();
    for (int kb = 0; kb < m; kb += NB) {
        const int nb = min(NB, m - kb);
        for (int t = tid; t < NB * NB; t += kT) {
            const int i = t % NB, j = t / NB;
            sD[i + j * (NB + 1)] = (i < nb && j < nb) ? L[(int64_t)(kb + i) + (int64_t)(kb + j) * m] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int jj = 0; jj < nb; ++jj) {
                if (lane == jj) {
                    const double piv = sD[jj + jj * (NB + 1)];
                    if (!(piv > 0.0)) fail = kb + jj + 1;
                    else sD[jj + jj * (NB + 1)] = sqrt(piv);
                }
                __syncwarp();
                if (fail) break;
                const double djj = sD[jj + jj * (NB + 1)];
                if (lane > jj && lane < nb) sD[lane + jj * (NB + 1)] /= djj;
                __syncwarp();
                if (lane > jj && lane < nb) {
                    const double lij = sD[lane + jj * (NB + 1)];
                    for (int k = jj + 1; k <= lane; ++k) sD[lane + k * (NB + 1)] -= lij * sD[k + jj * (NB + 1)];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        if (fail) break;
        for (int t = tid; t < nb * nb; t += kT) {
            const int i = t % nb, j = t / nb;
            if (i >= j) L[(int64_t)(kb + i) + (int64_t)(kb + j) * m] = sD[i + j * (NB + 1)];
        }
        // panel: rows below solve x L11^T = a
        for (int r = kb + nb + tid; r < m; r += kT) {
            double x[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) x[j] = (j < nb) ? L[(int64_t)r + (int64_t)(kb + j) * m] : 0.0;
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (j < nb) {
                    double v = x[j];
                    for (int k = 0; k < j; ++k) v -= x[k] * sD[j + k * (NB + 1)];
                    x[j] = v / sD[j + j * (NB + 1)];
                }
            }
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) L[(int64_t)r + (int64_t)(kb + j) * m] = x[j];
        }
        __syncthreads();
        // trailing update of the lower triangle: A22 -= L21 L21^T
        const int t0 = kb + nb;
        for (int c0 = t0; c0 < m; c0 += TS)
            for (int r0 = c0; r0 < m; r0 += TS)
                tile_update<true, true>(L, m, r0, c0, min(TS, m - r0), min(TS, m - c0), L + (int64_t)kb * m, m,
                                        L + (int64_t)kb * m, m, nb, sA, sB);
    }
    __syncthreads();
    const int f = fail;
    __syncthreads();
    if (f) return f;
    for (int j = 1; j < m; ++j)
        for (int i = tid; i < j; i += kT) L[(int64_t)i + (int64_t)j * m] = 0.0;
    return 0;
}

// X <- L^-1 X (L lower, m x m; X m x m), blocked by 32 rows.
__device__ void trsm_left_lower(const double* __restrict__ L, double* __restrict__ X, int m, double* sA, double* sB,
                                double* sD) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i0 = 0; i0 < m; i0 += NB) {
        const int nb = min(NB, m - i0), i1 = i0 + nb;
        for (int t = tid; t < NB * NB; t += kT) {
            const int i = t % NB, j = t / NB;
            sD[i + j * (NB + 1)] = (i < nb && j < nb) ? L[(int64_t)(i0 + i) + (int64_t)(i0 + j) * m] : 0.0;
        }
        __syncthreads();
        // diagonal block: warp per column of X, lanes over its rows
        for (int j = warp; j < m; j += kT / 32) {
            double x = (lane < nb) ? X[(int64_t)(i0 + lane) + (int64_t)j * m] : 0.0;
            for (int k = 0; k < nb; ++k) {
                if (lane == k) x /= sD[k + k * (NB + 1)];
                const double xk = __shfl_sync(0xffffffffu, x, k);
                if (lane > k && lane < nb) x -= sD[lane + k * (NB + 1)] * xk;
            }
            if (lane < nb) X[(int64_t)(i0 + lane) + (int64_t)j * m] = x;
        }
        __syncthreads();
        for (int c0 = 0; c0 < m; c0 += TS)
            for (int r0 = i1; r0 < m; r0 += TS)
                tile_update<false, false>(X, m, r0, c0, min(TS, m - r0), min(TS, m - c0), L + (int64_t)i0 * m, m,
                                          X + i0, m, nb, sA, sB);
    }
}

// C <- L^-1 H_k L^-T: C <- L^-1 C, transpose, C <- L^-1 C, then the lower
// triangle copied to the upper one (exactly symmetric).
__device__ void stage_reduce(const EigProb& p, const double* __restrict__ La, double* __restrict__ Ca,
                             const StageSmem& sh) {
    double* sA = sh.sA;
    double* sB = sh.sB;
    double* sD = sh.sD;
    const int m = p.m;
    const double* L = La + p.aoff;
    double* C = Ca + p.aoff;
    trsm_left_lower(L, C, m, sA, sB, sD);
    __syncthreads();
    for (int64_t t = threadIdx.x; t < (int64_t)m * m; t += kT) {
        const int i = (int)(t % m), j = (int)(t / m);
        if (i > j) {
            const double a = C[i + (int64_t)j * m], b = C[j + (int64_t)i * m];
            C[i + (int64_t)j * m] = b;
            C[j + (int64_t)i * m] = a;
        }
    }
    __syncthreads();
    trsm_left_lower(L, C, m, sA, sB, sD);
    __syncthreads();
    for (int64_t t = threadIdx.x; t < (int64_t)m * m; t += kT) {
        const int i = (int)(t % m), j = (int)(t / m);
        if (i > j) C[j + (int64_t)i * m] = C[i + (int64_t)j * m];
    }
}

// ---------------------------------------------------------------------------
// Householder tridiagonalisation of C (lower).  Iteration j applies the
// previous reflector's rank-2 update to column j, forms reflector j from it
// (LAPACK's dlarfg convention: beta = -sign(alpha) |x|, tau = (beta - alpha) /
// beta, v = x / (alpha - beta) with v_{j+1} = 1), and in one pass over the
// trailing block applies the previous update and accumulates p = A v for the
// new reflector; w = tau p - (tau^2/2)(p.v) v.  The trailing block is read and
// written once per column.  Output: d (m), e (m-1), tau, and v_j in C's column
// j below the subdiagonal.
constexpr int kSyRows = (kEigBatchMax + kT - 1) / kT;   // rows per thread
constexpr int kSyChunk = 8;                              // columns per batch of loads

__device__ void stage_sytrd(const EigProb& p, double* __restrict__ Ca, double* __restrict__ Da,
                            double* __restrict__ Ea, double* __restrict__ Ta, const StageSmem& sh) {
    double* vc = reinterpret_cast<double*>(sh.uni);
    double* wc = vc + sh.M;
    double* vn = wc + sh.M;
    double* red = sh.dsc + 2;
    double& sh_tau = sh.dsc[0];
    double& sh_alpha = sh.dsc[1];
    const int m = p.m;
    double* A = Ca + p.aoff;
    double* d = Da + p.voff;
    double* e = Ea + p.voff;
    double* tau = Ta + p.voff;
    const int tid = threadIdx.x;
    if (m == 1) {
        if (tid == 0) {
            d[0] = A[0];
            tau[0] = 0.0;
        }
        return;
    }
    for (int r = tid; r < m; r += kT) {
        vc[r] = 0.0;
        wc[r] = 0.0;
    }
    __syncthreads();
    for (int j = 0; j <= m - 2; ++j) {
        // (1) column j (rows >= j) gets the previous reflector's update
        const double vj = vc[j], wj = wc[j];
        for (int r = j + tid; r < m; r += kT) {
            double a = A[r + (int64_t)j * m];
            a -= vc[r] * wj + wc[r] * vj;
            A[r + (int64_t)j * m] = a;
            vn[r] = a;
        }
        __syncthreads();
        if (j == m - 2) {
            if (tid == 0) {
                d[m - 2] = vn[m - 2];
                e[m - 2] = vn[m - 1];
                double a = A[(m - 1) + (int64_t)(m - 1) * m];
                a -= 2.0 * vc[m - 1] * wc[m - 1];
                A[(m - 1) + (int64_t)(m - 1) * m] = a;
                d[m - 1] = a;
                tau[m - 2] = 0.0;
                tau[m - 1] = 0.0;
            }
            break;
        }
        // (2) reflector of x = column j, rows j+1..m-1
        double part = 0.0;
        for (int r = j + 2 + tid; r < m; r += kT) part += vn[r] * vn[r];
        const double xn2 = cta_sum(part, red);
        if (tid == 0) {
            const double alpha = vn[j + 1];
            d[j] = vn[j];
            double t, beta;
            if (xn2 == 0.0) {
                t = 0.0;
                beta = alpha;
            } else {
                beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                t = (beta - alpha) / beta;
            }
            e[j] = beta;
            tau[j] = t;
            sh_tau = t;
            sh_alpha = (t == 0.0) ? 0.0 : 1.0 / (alpha - beta);
            A[(j + 1) + (int64_t)j * m] = beta;
        }
        __syncthreads();
        const double t = sh_tau, sc = sh_alpha;
        for (int r = j + 1 + tid; r < m; r += kT) {
            double v;
            if (r == j + 1) v = 1.0;
            else v = (t == 0.0) ? 0.0 : vn[r] * sc;
            vn[r] = v;
            if (r >= j + 2) A[r + (int64_t)j * m] = v;
        }
        __syncthreads();
        // (3) trailing block [j+1, m)^2: previous update + p = A v
        const int r0 = j + 1;
        double acc[kSyRows], vr[kSyRows], wr[kSyRows];
#pragma unroll
        for (int q = 0; q < kSyRows; ++q) {
            const int r = r0 + tid + q * kT;
            acc[q] = 0.0;
            vr[q] = (r < m) ? vc[r] : 0.0;
            wr[q] = (r < m) ? wc[r] : 0.0;
        }
        // columns in chunks of kSyChunk: every load of a chunk is issued before
        // its stores, so the pass streams instead of waiting on each element;
        // threads without a row in the trailing block skip the pass, and while
        // the block has at most kT rows each thread carries one row only
        const bool has_row = r0 + tid < m;
        if (m - r0 <= kT) {
            double* colbase = A + r0 + tid;
            for (int k0 = has_row ? r0 : m; k0 < m; k0 += kSyChunk) {
                double a1[kSyChunk];
#pragma unroll
                for (int u = 0; u < kSyChunk; ++u) {
                    const int k = k0 + u;
                    a1[u] = (k < m) ? colbase[(int64_t)k * m] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kSyChunk; ++u) {
                    const int k = k0 + u;
                    if (k < m) {
                        const double x = a1[u] - (vr[0] * wc[k] + wr[0] * vc[k]);
                        colbase[(int64_t)k * m] = x;
                        acc[0] = fma(x, vn[k], acc[0]);
                    }
                }
            }
        } else
        for (int k0 = has_row ? r0 : m; k0 < m; k0 += kSyChunk) {
            double a[kSyChunk][kSyRows];
#pragma unroll
            for (int u = 0; u < kSyChunk; ++u) {
                const int k = k0 + u;
#pragma unroll
                for (int q = 0; q < kSyRows; ++q) {
                    const int r = r0 + tid + q * kT;
                    a[u][q] = (k < m && r < m) ? A[r + (int64_t)k * m] : 0.0;
                }
            }
#pragma unroll
            for (int u = 0; u < kSyChunk; ++u) {
                const int k = k0 + u;
                if (k < m) {
                    const double vk = vc[k], wk = wc[k], nk = vn[k];
#pragma unroll
                    for (int q = 0; q < kSyRows; ++q) {
                        const int r = r0 + tid + q * kT;
                        if (r < m) {
                            const double x = a[u][q] - (vr[q] * wk + wr[q] * vk);
                            A[r + (int64_t)k * m] = x;
                            acc[q] = fma(x, nk, acc[q]);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // (4) w = tau p - (tau/2)(tau p . v) v
        double pv = 0.0;
#pragma unroll
        for (int q = 0; q < kSyRows; ++q) {
            const int r = r0 + tid + q * kT;
            if (r < m) {
                acc[q] *= t;
                pv += acc[q] * vn[r];
            }
        }
        const double ptv = cta_sum(pv, red);
        const double half = 0.5 * t * ptv;
#pragma unroll
        for (int q = 0; q < kSyRows; ++q) {
            const int r = r0 + tid + q * kT;
            if (r < m) {
                wc[r] = acc[q] - half * vn[r];
                vc[r] = vn[r];
            }
        }
        if (tid == 0) {
            vc[j] = 0.0;
            wc[j] = 0.0;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// C[crow + r0 + i, col(c0 + j)] = sum_k A(i, kx(k)) B(kxb(k), j) on one TS x TS
// output tile (tile_mma, MMA_SET).
template <bool AT, bool BT = false>
__device__ void tile_gemm(double* __restrict__ C, int64_t ldc, int crow, const int* ccol, int r0, int c0, int mr,
                          int nc, const double* __restrict__ A, int64_t lda, const int* kx,
                          const double* __restrict__ B, int64_t ldb, const int* kxb, int K, double* sA, double* sB) {
    tile_mma<AT, BT, MMA_SET, false>(C, ldc, crow, ccol, r0, c0, mr, nc, A, lda, kx, B, ldb, kxb, K, sA, sB);
}

// ---------------------------------------------------------------------------
// Divide and conquer for the tridiagonal eigenproblem T = Z diag(w) Z^T
// (Cuppen's split T = diag(T1, T2) + |beta| u u^T, u = e_last + sign(beta)
// e_first; Gu and Eisenstat's recomputed z for orthogonal eigenvectors), one
// CTA per problem.  Leaves of at most 32 rows are solved by a warp with the
// implicit QL iteration (every lane runs the same scalar iteration and applies
// each rotation to its own row of the leaf's Z); the merges run bottom-up over
// a balanced tree, one at a time with the whole CTA:
//   z = [last row of Z1, sign(beta) first row of Z2] / sqrt 2, rho = 2|beta|;
//   sort the block eigenvalues (merge of two sorted lists);
//   deflate: rho |z_j| <= tol -> eigenpair (d_j, q_j); two close d's -> a Givens
//   rotation zeroes one z entry (LAPACK's dlaed2 rules, tol = 8 eps max(|d|, rho));
//   secular roots lambda_i = d_org + tau in (d_i, d_i+1), each step modelling the
//   left and right sums by one pole each;
//   zhat_j^2 = (lambda_j - d_j) prod_{i != j} (lambda_i - d_j)/(d_i - d_j) / rho;
//   v_i = (zhat_j / (d_j - lambda_i))_j normalised; Z_new = Q v in two GEMMs
//   (rows of block 1 against the columns that touch it, rows of block 2 likewise).
// Output: w ascending, Z in the Z arena (column-major, ld m).
constexpr int kDcLeaf = 32;

struct DcSmem {
    // per-element arrays of the merge (kEigBatchMax each)
    double *D, *Ds, *zs, *dk, *zk, *tau, *zh, *val;
    int *perm, *org, *sec, *dl, *rank, *cls, *ktop, *kbot;
    int2* rpair;
    double2* rcs;
};

// Per-element arrays of capacity M (a multiple of 2, so every block stays
// 16-byte aligned).
__device__ DcSmem dc_smem(unsigned char* base, int M) {
    DcSmem s;
    double* d = reinterpret_cast<double*>(base);
    s.D = d;
    s.Ds = d + M;
    s.zs = d + 2 * M;
    s.dk = d + 3 * M;
    s.zk = d + 4 * M;
    s.tau = d + 5 * M;
    s.zh = d + 6 * M;
    s.val = d + 7 * M;
    s.rcs = reinterpret_cast<double2*>(d + 8 * M);
    int* ip = reinterpret_cast<int*>(s.rcs + M);
    s.perm = ip;
    s.org = ip + M;
    s.sec = ip + 2 * M;
    s.dl = ip + 3 * M;
    s.rank = ip + 4 * M;
    s.cls = ip + 5 * M;
    s.ktop = ip + 6 * M;
    s.kbot = ip + 7 * M;
    s.rpair = reinterpret_cast<int2*>(ip + 8 * M);
    return s;
}
__host__ __device__ constexpr size_t dc_smem_bytes(int M) {
    return (sizeof(double) * 8 + sizeof(double2) + sizeof(int) * 8 + sizeof(int2)) * (size_t)M;
}

// Leaf: implicit QL on d[0..s), e[0..s-1) with Z = I accumulated.  Every
// lane runs the same scalar iteration on its own copies of d and e and rotates
// its own row z of Z (lane r holds row r), so no lane reads another's data.
__device__ bool dc_leaf(int s, double* d, double* e, double* z, int lane) {
    const double eps = 2.220446049250313e-16;
    for (int c = 0; c < kDcLeaf; ++c) z[c] = (c == lane) ? 1.0 : 0.0;
    for (int l = 0; l < s; ++l) {
        int iter = 0;
        for (;;) {
            int mm = l;
            for (; mm < s - 1; ++mm)
                if (fabs(e[mm]) <= eps * (fabs(d[mm]) + fabs(d[mm + 1]))) break;
            if (mm == l) break;
            if (++iter > kQlMaxIter) return false;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + copysign(r, g));
            double sn = 1.0, c = 1.0, pp = 0.0;
            bool underflow = false;
            for (int i = mm - 1; i >= l; --i) {
                const double f = sn * e[i], b = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= pp;
                    e[mm] = 0.0;
                    underflow = true;
                    break;
                }
                sn = f / r;
                c = g / r;
                g = d[i + 1] - pp;
                r = (d[i] - g) * sn + 2.0 * c * b;
                pp = sn * r;
                d[i + 1] = g + pp;
                g = c * r - b;
                const double zi = z[i], zi1 = z[i + 1];
                z[i + 1] = sn * zi + c * zi1;
                z[i] = c * zi - sn * zi1;
            }
            if (underflow) continue;
            d[l] -= pp;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    return true;
}

// Root i of 1 + rho sum_t z_t^2 / (dk_t - lambda) = 0 (dk ascending, k roots):
// returns tau with lambda = dk[*org] + tau.
__device__ double dc_secular(int k, const double* dk, const double* zk, double rho, int i, int* org_out) {
    const double eps = 2.220446049250313e-16;
    int org;
    double lo, hi;
    if (i < k - 1) {
        const double mid = 0.5 * (dk[i + 1] - dk[i]);
        double f = 1.0;
        for (int t = 0; t < k; ++t) f += rho * zk[t] * zk[t] / ((dk[t] - dk[i]) - mid);
        if (f >= 0.0) {
            org = i;
            lo = 0.0;
            hi = mid;
        } else {
            org = i + 1;
            lo = -mid;
            hi = 0.0;
        }
    } else {
        double z2 = 0.0;
        for (int t = 0; t < k; ++t) z2 += zk[t] * zk[t];
        org = i;
        lo = 0.0;
        hi = rho * z2;
    }
    const double dorg = dk[org];
    const double a = dk[i] - dorg;
    const double b = (i < k - 1) ? dk[i + 1] - dorg : 0.0;
    double tau = 0.5 * (lo + hi);
    for (int it = 0; it < 100; ++it) {
        double psi = 0.0, phi = 0.0, dpsi = 0.0, dphi = 0.0;
        for (int t = 0; t < k; ++t) {
            const double den = (dk[t] - dorg) - tau;
            const double q = rho * zk[t] * zk[t] / den;
            if (t <= i) {
                psi += q;
                dpsi += q / den;
            } else {
                phi += q;
                dphi += q / den;
            }
        }
        const double f = 1.0 + psi + phi;
        if (f > 0.0) hi = tau;
        else if (f < 0.0) lo = tau;
        else break;
        if (fabs(f) <= 16.0 * eps * (1.0 + fabs(psi) + fabs(phi))) break;
        const double B = dpsi * (a - tau) * (a - tau);
        const double A = psi - B / (a - tau);
        double nt;
        if (i < k - 1) {
            const double E = dphi * (b - tau) * (b - tau);
            const double Cc = phi - E / (b - tau);
            const double c0 = 1.0 + A + Cc;
            const double qb = -(c0 * (a + b) + B + E);
            const double qc = c0 * a * b + B * b + E * a;
            if (c0 == 0.0) {
                nt = -qc / qb;
            } else {
                const double disc = fmax(qb * qb - 4.0 * c0 * qc, 0.0);
                const double r1 = (-qb - copysign(sqrt(disc), qb)) / (2.0 * c0);
                const double r2 = (r1 != 0.0) ? qc / (c0 * r1) : r1;
                nt = (lo < r1 && r1 < hi) ? r1 : r2;
            }
        } else {
            const double c0 = 1.0 + A + phi;
            nt = (c0 != 0.0) ? a + B / c0 : 0.5 * (lo + hi);
        }
        if (!(lo < nt && nt < hi)) nt = 0.5 * (lo + hi);
        if (fabs(nt - tau) <= 2.0 * eps * fabs(nt)) {
            tau = nt;
            break;
        }
        tau = nt;
    }
    *org_out = org;
    return tau;
}

__device__ bool stage_dc(const EigProb& p, const double* __restrict__ Da, const double* __restrict__ Ea,
                         double* __restrict__ Wa, double* __restrict__ Za, double* __restrict__ Qa,
                         double* __restrict__ Va, const StageSmem& sh) {
    double* sA = sh.sA;
    double* sB = sh.sB;
    int& s_k = sh.ints[1];
    int& s_nd = sh.ints[2];
    int& s_nrot = sh.ints[3];
    int& s_ntop = sh.ints[4];
    int& s_nbot = sh.ints[5];
    int& s_fail = sh.ints[6];
    const int m = p.m;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* Z = Za + p.aoff;
    double* Qp = Qa + p.aoff;
    double* V = Va + p.aoff;
    const double* eo = Ea + p.voff;
    DcSmem S = dc_smem(sh.uni, sh.M);
    int L = 0;
    while (((m + (1 << L) - 1) >> L) > kDcLeaf) ++L;
    const int nleaf = 1 << L;
    for (int i = tid; i < m; i += kT) S.D[i] = Da[p.voff + i];
    if (tid == 0) s_fail = 0;
    __syncthreads();
    if (tid == 0)
        for (int q = 1; q < nleaf; ++q) {
            const int pos = (int)(((int64_t)q * m) >> L);
            const double ab = fabs(eo[pos - 1]);
            S.D[pos - 1] -= ab;
            S.D[pos] -= ab;
        }
    __syncthreads();
    // leaves: a warp each
    for (int q = warp; q < nleaf; q += kT / 32) {
        const int lo = (int)(((int64_t)q * m) >> L), hi = (int)(((int64_t)(q + 1) * m) >> L), s = hi - lo;
        double dl[kDcLeaf], el[kDcLeaf], zl[kDcLeaf];
        for (int i = 0; i < kDcLeaf; ++i) {
            dl[i] = (i < s) ? S.D[lo + i] : 0.0;
            el[i] = (i < s - 1) ? eo[lo + i] : 0.0;
        }
        const bool ok = dc_leaf(s, dl, el, zl, lane);
        if (!ok && lane == 0) s_fail = 1;
        // eigenvalues ascending (ties by index) and the columns in that order
        int rk = 0;
        if (lane < s) {
            const double x = dl[lane];
            for (int c = 0; c < s; ++c) rk += (dl[c] < x || (dl[c] == x && c < lane)) ? 1 : 0;
        }
        for (int c = 0; c < s; ++c) {
            const int rc = __shfl_sync(0xffffffffu, rk, c);
            if (lane < s) Z[(int64_t)(lo + lane) + (int64_t)(lo + rc) * m] = zl[c];
        }
        __syncwarp();
        if (lane < s) S.D[lo + rk] = dl[lane];
        __syncwarp();
    }
    __syncthreads();
    if (s_fail) return false;
    const double eps = 2.220446049250313e-16;
    for (int lev = L - 1; lev >= 0; --lev) {
        for (int q = 0; q < (1 << lev); ++q) {
            const int lo = (int)(((int64_t)q * m) >> lev), hi = (int)(((int64_t)(q + 1) * m) >> lev);
            const int mid = (int)(((int64_t)(2 * q + 1) * m) >> (lev + 1));
            const int n1 = mid - lo, n2 = hi - mid, n = n1 + n2;
            const double beta = eo[mid - 1];
            const double rho = 2.0 * fabs(beta);
            const double sgn = beta >= 0.0 ? 1.0 : -1.0;
            const double rs2 = 0.70710678118654752440;
            // (a) merged order of the two sorted blocks
            for (int j = tid; j < n; j += kT) {
                int r;
                if (j < n1) {
                    const double x = S.D[lo + j];
                    int a = 0, b = n2;
                    while (a < b) {
                        const int c = (a + b) >> 1;
                        if (S.D[mid + c] < x) a = c + 1;
                        else b = c;
                    }
                    r = j + a;
                } else {
                    const double x = S.D[mid + j - n1];
                    int a = 0, b = n1;
                    while (a < b) {
                        const int c = (a + b) >> 1;
                        if (S.D[lo + c] <= x) a = c + 1;
                        else b = c;
                    }
                    r = (j - n1) + a;
                }
                S.perm[r] = j;
            }
            __syncthreads();
            // (b) sorted d, z and column classes; (c) Q with the block columns in that order
            for (int r = tid; r < n; r += kT) {
                const int j = S.perm[r];
                if (j < n1) {
                    S.Ds[r] = S.D[lo + j];
                    S.zs[r] = Z[(int64_t)(mid - 1) + (int64_t)(lo + j) * m] * rs2;
                    S.cls[r] = 1;
                } else {
                    S.Ds[r] = S.D[mid + j - n1];
                    S.zs[r] = sgn * Z[(int64_t)mid + (int64_t)(mid + j - n1) * m] * rs2;
                    S.cls[r] = 2;
                }
            }
            for (int64_t t = tid; t < (int64_t)n * n; t += kT) {
                const int i = (int)(t % n), r = (int)(t / n);
                const int j = S.perm[r];
                double v = 0.0;
                if (j < n1) {
                    if (i < n1) v = Z[(int64_t)(lo + i) + (int64_t)(lo + j) * m];
                } else if (i >= n1) {
                    v = Z[(int64_t)(lo + i) + (int64_t)(mid + j - n1) * m];
                }
                Qp[t] = v;
            }
            __syncthreads();
            // (d) deflation (one thread, in sorted order)
            if (tid == 0) {
                double dmax = 0.0;
                for (int r = 0; r < n; ++r) dmax = fmax(dmax, fabs(S.Ds[r]));
                const double tol = 8.0 * eps * fmax(dmax, rho);
                int k = 0, nd = 0, nrot = 0, pj = -1;
                for (int r = 0; r < n; ++r) {
                    if (rho * fabs(S.zs[r]) <= tol) {
                        S.dl[nd++] = r;
                        continue;
                    }
                    if (pj < 0) {
                        pj = r;
                        continue;
                    }
                    double sn = S.zs[pj], c = S.zs[r];
                    const double t = hypot(c, sn);
                    const double dd = S.Ds[r] - S.Ds[pj];
                    c /= t;
                    sn = -sn / t;
                    if (fabs(dd * c * sn) <= tol) {
                        S.zs[r] = t;
                        S.zs[pj] = 0.0;
                        S.rpair[nrot] = make_int2(pj, r);
                        S.rcs[nrot] = make_double2(c, sn);
                        ++nrot;
                        const double t2 = S.Ds[pj] * c * c + S.Ds[r] * sn * sn;
                        S.Ds[r] = S.Ds[pj] * sn * sn + S.Ds[r] * c * c;
                        S.Ds[pj] = t2;
                        S.cls[r] |= S.cls[pj];
                        S.dl[nd++] = pj;
                        pj = r;
                    } else {
                        S.sec[k++] = pj;
                        pj = r;
                    }
                }
                if (pj >= 0) S.sec[k++] = pj;
                // secular columns that touch block 1 / block 2 (the K lists of the two GEMMs)
                int nt = 0, nb = 0;
                for (int t = 0; t < k; ++t) {
                    const int c = S.cls[S.sec[t]];
                    if (c & 1) S.ktop[nt++] = t;
                    if (c & 2) S.kbot[nb++] = t;
                }
                s_k = k;
                s_nd = nd;
                s_nrot = nrot;
                s_ntop = nt;
                s_nbot = nb;
            }
            __syncthreads();
            const int k = s_k, nd = s_nd, nrot = s_nrot;
            // (e) deflation rotations on the columns of Q (thread per row)
            if (nrot > 0)
                for (int i = tid; i < n; i += kT)
                    for (int q2 = 0; q2 < nrot; ++q2) {
                        const int2 pr = S.rpair[q2];
                        const double2 cs = S.rcs[q2];
                        const double a = Qp[i + (int64_t)pr.x * n], b = Qp[i + (int64_t)pr.y * n];
                        Qp[i + (int64_t)pr.x * n] = cs.x * a + cs.y * b;
                        Qp[i + (int64_t)pr.y * n] = -cs.y * a + cs.x * b;
                    }
            for (int t = tid; t < k; t += kT) {
                S.dk[t] = S.Ds[S.sec[t]];
                S.zk[t] = S.zs[S.sec[t]];
            }
            __syncthreads();
            // (f) secular roots
            for (int i = tid; i < k; i += kT) S.tau[i] = dc_secular(k, S.dk, S.zk, rho, i, &S.org[i]);
            __syncthreads();
            // (g) recomputed z
            for (int j = tid; j < k; j += kT) {
                const double dj = S.dk[j];
                double w = (S.dk[S.org[j]] - dj) + S.tau[j];
                for (int i = 0; i < k; ++i) {
                    if (i == j) continue;
                    w *= ((S.dk[S.org[i]] - dj) + S.tau[i]) / (S.dk[i] - dj);
                }
                S.zh[j] = copysign(sqrt(fmax(w / rho, 0.0)), S.zk[j]);
            }
            __syncthreads();
            // (h) eigenvectors of the rank-one problem (columns of V, k x k) and the new eigenvalues
            for (int i = tid; i < k; i += kT) {
                const double dorg = S.dk[S.org[i]], ti = S.tau[i];
                double nrm = 0.0;
                for (int j = 0; j < k; ++j) {
                    const double v = S.zh[j] / ((S.dk[j] - dorg) - ti);
                    nrm = fma(v, v, nrm);
                }
                const double sc = 1.0 / sqrt(nrm);
                for (int j = 0; j < k; ++j) V[j + (int64_t)i * k] = sc * (S.zh[j] / ((S.dk[j] - dorg) - ti));
                S.val[i] = dorg + ti;
            }
            for (int q2 = tid; q2 < nd; q2 += kT) S.val[k + q2] = S.Ds[S.dl[q2]];
            __syncthreads();
            // (i) positions of the n new eigenvalues in ascending order
            for (int a = tid; a < n; a += kT) {
                const double x = S.val[a];
                int r = 0;
                for (int b2 = 0; b2 < n; ++b2) r += (S.val[b2] < x || (S.val[b2] == x && b2 < a)) ? 1 : 0;
                S.rank[a] = lo + r;
            }
            __syncthreads();
            // (j) Z block = Q [V | deflated columns]: block-1 rows against the columns
            // touching block 1, block-2 rows against those touching block 2
            // gathered K lists: columns of Q (sec[ktop[t]]) against rows ktop[t] of V
            for (int t = tid; t < s_ntop; t += kT) S.perm[t] = S.sec[S.ktop[t]];
            __syncthreads();
            // rows of block 1: Z[lo + r, rank[c]] = sum_t Q[r, sec[ktop[t]]] V[ktop[t], c]
            for (int c0 = 0; c0 < k; c0 += TS)
                for (int r0 = 0; r0 < n1; r0 += TS)
                    tile_gemm<false>(Z, m, lo, S.rank, r0, c0, min(TS, n1 - r0), min(TS, k - c0), Qp, n, S.perm, V, k,
                                     S.ktop, s_ntop, sA, sB);
            __syncthreads();
            for (int t = tid; t < s_nbot; t += kT) S.perm[t] = S.sec[S.kbot[t]];
            __syncthreads();
            // rows of block 2 against the columns that touch block 2
            for (int c0 = 0; c0 < k; c0 += TS)
                for (int r0 = n1; r0 < n; r0 += TS)
                    tile_gemm<false>(Z, m, lo, S.rank, r0, c0, min(TS, n - r0), min(TS, k - c0), Qp, n, S.perm, V, k,
                                     S.kbot, s_nbot, sA, sB);
            // deflated columns: copies of Q's columns
            for (int64_t t = tid; t < (int64_t)nd * n; t += kT) {
                const int i = (int)(t % n), q2 = (int)(t / n);
                Z[(int64_t)(lo + i) + (int64_t)S.rank[k + q2] * m] = Qp[i + (int64_t)S.dl[q2] * n];
            }
            for (int a = tid; a < n; a += kT) S.D[S.rank[a]] = S.val[a];
            __syncthreads();
        }
    }
    for (int i = tid; i < m; i += kT) Wa[p.voff + i] = S.D[i];
    return true;
}

// ---------------------------------------------------------------------------
// Q = H_0 H_1 ... H_{m-3} applied to nv vectors x_t of length m (x_t at
// X + t m): trans -> x <- Q^T x (panels of 32 reflectors in order), else
// x <- Q x (panels in reverse).  A panel's reflectors act together as
// I - V T V^T (compact WY: T upper triangular, T_qq = tau_q,
// T[0:q, q] = -tau_q T[0:q, 0:q] V[:, 0:q]^T v_q), so each panel costs three
// small products and a handful of barriers instead of two barriers per
// reflector.  v_j: 1 at j+1, C[r + j m] for r >= j+2, zero above.
struct WySmem {
    double* G;   // NB x (NB+1): Gram V^T V, then T
    double* Xs;  // NB x kWyChunk: V^T x, then T(^T) V^T x
};
constexpr int kWyChunk = 64;
static_assert(TS * NB % kT == 0, "tile staging divides over the CTA");
static_assert(NB * (NB + 1) <= kStageOp && NB * kWyChunk <= kStageOp, "WY scratch fits the tile staging");

__device__ __forceinline__ double wy_v(const double* C, int m, int j, int r) {
    return (r == j + 1) ? 1.0 : (r > j + 1 ? C[r + (int64_t)j * m] : 0.0);
}

__device__ void wy_apply(const double* __restrict__ C, int m, const double* __restrict__ tau, double* X, int nv,
                         bool trans, WySmem sm) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nref = m - 2;   // reflectors 0..m-3
    if (nref <= 0) return;
    const int npan = (nref + NB - 1) / NB;
    for (int pp = 0; pp < npan; ++pp) {
        const int pan = trans ? pp : npan - 1 - pp;
        const int j0 = pan * NB, nb = min(NB, nref - j0);
        // Gram of the panel's vectors (rows j0+1 .. m-1): a warp per pair, lanes
        // over the rows (coalesced), fixed-order sums
        for (int q = warp; q < NB * NB; q += kT / 32) {
            const int a = q % NB, b = q / NB;
            double g = 0.0;
            if (a < nb && b < nb && a <= b) {
                for (int r = j0 + 1 + b + lane; r < m; r += 32)
                    g = fma(wy_v(C, m, j0 + a, r), wy_v(C, m, j0 + b, r), g);
                g = warp_sum(g);
            }
            if (lane == 0) sm.G[a + b * (NB + 1)] = g;
        }
        __syncthreads();
        // T in place of the Gram's upper triangle (one warp, column by column)
        if (warp == 0) {
            for (int b = 0; b < nb; ++b) {
                const double tb = tau[j0 + b];
                // T[a][b] = -tb * sum_{a <= c < b} T[a][c] G[c][b] for a < b (lane a)
                double acc = 0.0;
                if (lane < b)
                    for (int c2 = lane; c2 < b; ++c2) acc = fma(sm.G[lane + c2 * (NB + 1)], sm.G[c2 + b * (NB + 1)], acc);
                __syncwarp();
                if (lane < b) sm.G[lane + b * (NB + 1)] = -tb * acc;
                if (lane == b) sm.G[b + b * (NB + 1)] = tb;
                __syncwarp();
            }
        }
        __syncthreads();
        for (int t0 = 0; t0 < nv; t0 += kWyChunk) {
            const int nc = min(kWyChunk, nv - t0);
            // Xs = V^T x: a warp per (reflector, vector), lanes over the rows
            for (int q = warp; q < NB * nc; q += kT / 32) {
                const int a = q % NB, t = q / NB;
                double g = 0.0;
                if (a < nb) {
                    const double* x = X + (int64_t)(t0 + t) * m;
                    for (int r = j0 + 1 + a + lane; r < m; r += 32) g = fma(wy_v(C, m, j0 + a, r), x[r], g);
                    g = warp_sum(g);
                }
                if (lane == 0) sm.Xs[a + t * NB] = g;
            }
            __syncthreads();
            // Xs <- T Xs or T^T Xs (thread per column t, in registers)
            for (int t = tid; t < nc; t += kT) {
                double xv[NB], yv[NB];
                for (int a = 0; a < NB; ++a) xv[a] = sm.Xs[a + t * NB];
                for (int a = 0; a < NB; ++a) {
                    double y = 0.0;
                    if (a < nb) {
                        if (trans) {   // (T^T x)_a = sum_{c <= a} T[c][a] x_c
                            for (int c2 = 0; c2 <= a; ++c2) y = fma(sm.G[c2 + a * (NB + 1)], xv[c2], y);
                        } else {       // (T x)_a = sum_{c >= a} T[a][c] x_c
                            for (int c2 = a; c2 < nb; ++c2) y = fma(sm.G[a + c2 * (NB + 1)], xv[c2], y);
                        }
                    }
                    yv[a] = y;
                }
                for (int a = 0; a < NB; ++a) sm.Xs[a + t * NB] = yv[a];
            }
            __syncthreads();
            // x <- x - V Xs
            for (int64_t q = tid; q < (int64_t)nc * (m - j0 - 1); q += kT) {
                const int t = (int)(q / (m - j0 - 1)), r = j0 + 1 + (int)(q % (m - j0 - 1));
                double s = 0.0;
                for (int a = 0; a < nb; ++a) s = fma(wy_v(C, m, j0 + a, r), sm.Xs[a + t * NB], s);
                X[(int64_t)(t0 + t) * m + r] -= s;
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
constexpr int kWyMmaMin = 64;   // orders from which the reflectors are applied as tile products

__host__ __device__ constexpr int64_t t_panels(int m) { return m > 2 ? (m - 2 + NB - 1) / NB : 0; }

// T of the compact WY form I - V T V^T of every panel of NB reflectors of
// Q = H_0 ... H_{m-3} (panels p = first, first + step, ...): the panel's
// Gram V^T V as one tile product reading the reflectors in place, then T
// column by column (T_bb = tau_b, T[0:b, b] = -tau_b T[0:b, 0:b] G[0:b, b])
// by one warp.  Tall + p NB^2 holds panel p's T (NB x NB, column-major, zero
// outside the panel's nb x nb upper triangle).  Gg: NB^2 global scratch;
// T: NB x (NB+1) shared.
__device__ void build_T(const double* __restrict__ C, int m, const double* __restrict__ tau, double* __restrict__ Tall,
                        int first, int step, double* Gg, double* T, double* sA, double* sB) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nref = m - 2;
    const int npan = (int)t_panels(m);
    for (int pan = first; pan < npan; pan += step) {
        const int j0 = pan * NB, nb = min(NB, nref - j0), r0 = j0 + 1, len = m - r0;
        const double* Vb = C + r0 + (int64_t)j0 * m;
        tile_mma<true, false, MMA_SET, false, true, true>(Gg, NB, 0, nullptr, 0, 0, nb, nb, Vb, m, nullptr, Vb, m,
                                                          nullptr, len, sA, sB);
        for (int q = tid; q < NB * NB; q += kT) {
            const int a = q % NB, b = q / NB;
            T[a + b * (NB + 1)] = (a <= b && b < nb) ? Gg[a + b * NB] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int b = 0; b < nb; ++b) {
                const double tb = tau[j0 + b];
                double acc = 0.0;
                if (lane < b)
                    for (int c2 = lane; c2 < b; ++c2) acc = fma(T[lane + c2 * (NB + 1)], T[c2 + b * (NB + 1)], acc);
                __syncwarp();
                if (lane < b) T[lane + b * (NB + 1)] = -tb * acc;
                if (lane == b) T[b + b * (NB + 1)] = tb;
                __syncwarp();
            }
        }
        __syncthreads();
        double* Tp = Tall + (int64_t)pan * NB * NB;
        for (int q = tid; q < NB * NB; q += kT) {
            const int a = q % NB, b = q / NB;
            Tp[q] = (a < nb && b < nb) ? T[a + b * (NB + 1)] : 0.0;
        }
        __syncthreads();
    }
}

// Q = H_0 ... H_{m-3} applied to nv vectors (X, ld m) on the FP64 tensor
// cores, a panel of NB reflectors at a time as I - V T V^T with the panels' T
// from build_T: Y = V^T X, Y2 = T^T Y (trans: panels in order) or T Y (panels
// in reverse), X -= V Y2, the reflectors read in place from C.  Y and Y2 are
// NB x nv global scratch each.
__device__ void wy_apply_t(const double* __restrict__ C, int m, const double* __restrict__ Tall, double* X, int nv,
                           bool trans, double* Y, double* Y2, double* sA, double* sB) {
    const int tid = threadIdx.x;
    const int nref = m - 2;
    const int npan = (int)t_panels(m);
    if (npan == 0 || nv <= 0) return;
    for (int pp = 0; pp < npan; ++pp) {
        const int pan = trans ? pp : npan - 1 - pp;
        const int j0 = pan * NB, nb = min(NB, nref - j0), r0 = j0 + 1, len = m - r0;
        const double* Vb = C + r0 + (int64_t)j0 * m;
        const double* Tp = Tall + (int64_t)pan * NB * NB;
        for (int c0 = 0; c0 < nv; c0 += TS)
            tile_mma<true, false, MMA_SET, false, true, false>(Y, NB, 0, nullptr, 0, c0, nb, min(TS, nv - c0), Vb, m,
                                                               nullptr, X + r0, m, nullptr, len, sA, sB);
        for (int64_t q = tid; q < (int64_t)NB * nv; q += kT) {
            const int a = (int)(q % NB), t = (int)(q / NB);
            const double* yc = Y + (int64_t)t * NB;
            double y = 0.0;
            if (a < nb) {
                if (trans) {
                    for (int c2 = 0; c2 <= a; ++c2) y = fma(Tp[c2 + a * NB], yc[c2], y);
                } else {
                    for (int c2 = a; c2 < nb; ++c2) y = fma(Tp[a + c2 * NB], yc[c2], y);
                }
            }
            Y2[q] = y;
        }
        __syncthreads();
        for (int c0 = 0; c0 < nv; c0 += TS)
            for (int i0 = 0; i0 < len; i0 += TS)
                tile_mma<false, false, MMA_SUB, false, true, false>(X + r0, m, 0, nullptr, i0, c0, min(TS, len - i0),
                                                                    min(TS, nv - c0), Vb, m, nullptr, Y2, NB, nullptr,
                                                                    nb, sA, sB);
    }
}

// X <- L^-1 X (lower = true) or X <- L^-T X (lower = false) for the columns
// [c_begin, c_end) of X (ld ldx), L lower (ld m): over 64-row blocks (from the
// top, or from the bottom for L^-T), the earlier blocks' contribution as one
// tile product per 64-column block, then the diagonal block's substitution
// (warp per column, two rows per lane).  One CTA; sD holds TS x (TS+1).
__device__ void trsm_cols(bool lower, const double* __restrict__ L, int m, double* X, int64_t ldx, int c_begin,
                          int c_end, double* sD, double* sA, double* sB) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nrb = (m + TS - 1) / TS;
    for (int c0 = c_begin; c0 < c_end; c0 += TS) {
        const int nc = min(TS, c_end - c0);
        for (int q = 0; q < nrb; ++q) {
            const int rb = lower ? q : nrb - 1 - q;
            const int i0 = rb * TS, mr = min(TS, m - i0), i1 = i0 + mr;
            if (lower) {
                if (i0 > 0)
                    tile_mma<false, false, MMA_SUB, false>(X, ldx, 0, nullptr, i0, c0, mr, nc, L, m, nullptr, X, ldx,
                                                           nullptr, i0, sA, sB);
            } else if (i1 < m) {
                // (L^T)[i, k] = L[k, i] for k >= i1
                tile_mma<true, false, MMA_SUB, false>(X, ldx, 0, nullptr, i0, c0, mr, nc, L + i1, m, nullptr, X + i1,
                                                      ldx, nullptr, m - i1, sA, sB);
            }
            for (int t = tid; t < TS * TS; t += kT) {
                const int i = t % TS, j = t / TS;
                sD[i + j * (TS + 1)] = (i < mr && j < mr && i >= j) ? L[(int64_t)(i0 + i) + (int64_t)(i0 + j) * m] : 0.0;
            }
            __syncthreads();
            for (int jc = warp; jc < nc; jc += kT / 32) {
                double* x = X + (int64_t)(c0 + jc) * ldx + i0;
                double x0 = lane < mr ? x[lane] : 0.0, x1 = lane + 32 < mr ? x[lane + 32] : 0.0;
                if (lower) {
                    for (int k = 0; k < mr; ++k) {
                        double xk;
                        if (k < 32) {
                            if (lane == k) x0 /= sD[k + k * (TS + 1)];
                            xk = __shfl_sync(0xffffffffu, x0, k);
                        } else {
                            if (lane == k - 32) x1 /= sD[k + k * (TS + 1)];
                            xk = __shfl_sync(0xffffffffu, x1, k - 32);
                        }
                        if (lane > k && lane < mr) x0 -= sD[lane + k * (TS + 1)] * xk;
                        if (lane + 32 > k && lane + 32 < mr) x1 -= sD[lane + 32 + k * (TS + 1)] * xk;
                    }
                } else {
                    // L_bb^T x = b: back substitution, (L^T)[i, k] = sD[k + i (TS+1)] for k > i
                    for (int k = mr - 1; k >= 0; --k) {
                        double xk;
                        if (k < 32) {
                            if (lane == k) x0 /= sD[k + k * (TS + 1)];
                            xk = __shfl_sync(0xffffffffu, x0, k);
                        } else {
                            if (lane == k - 32) x1 /= sD[k + k * (TS + 1)];
                            xk = __shfl_sync(0xffffffffu, x1, k - 32);
                        }
                        if (lane < k) x0 -= sD[k + lane * (TS + 1)] * xk;
                        if (lane + 32 < k) x1 -= sD[k + (lane + 32) * (TS + 1)] * xk;
                    }
                }
                if (lane < mr) x[lane] = x0;
                if (lane + 32 < mr) x[lane + 32] = x1;
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Owned rows of S U and U, fe and the eigenpairs.  R holds 2 nown rows of
// length m (row-major, i.e. the column-major m x 2nown matrix R^T): rows
// t < nown are L[c_t,:] -> (S U)[c_t,:], rows nown + t are (L^-T)[c_t,:] ->
// U[c_t,:].  The final product with Z goes into the third block G (R Z).
__device__ void stage_rows(const EigProb& p, const double* __restrict__ Ca, const double* __restrict__ La,
                           const double* __restrict__ Ta, const double* __restrict__ Wa,
                           const double* __restrict__ Za, const int* __restrict__ own_cols,
                           const int* __restrict__ ipos, double* __restrict__ Ba, double* __restrict__ Qa,
                           double* __restrict__ Va, const double* __restrict__ Ka, double* __restrict__ e_out,
                           double* __restrict__ fe_out, const StageSmem& sh) {
    double* sA = sh.sA;
    double* sB = sh.sB;
    const int m = p.m, no = p.nown, nb2 = 2 * no;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* Z = Za + p.aoff;
    const double* tau = Ta + p.voff;
    double* R = Ba + p.boff;                     // 2 nown rows
    double* R2 = R + (int64_t)no * m;
    double* G = R + (int64_t)nb2 * m;            // 2 nown rows of R Z
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kT / 32;
    for (int t = 0; t < no; ++t) {
        const int ct = ipos[own_cols[p.o0 + t]];
        for (int r = tid; r < m; r += kT) {
            R[(int64_t)t * m + r] = (r <= ct) ? L[ct + (int64_t)r * m] : 0.0;
            R2[(int64_t)t * m + r] = (r == ct) ? 1.0 : 0.0;
        }
    }
    __syncthreads();
    // rows of L^-T: x_t = L^-1 e_{c_t}; blocked on the tensor cores when the
    // divide and conquer's (now free) arrays hold a 64 x 65 diagonal block
    if (dc_smem_bytes(sh.M) >= sizeof(double) * TS * (TS + 1)) {
        trsm_cols(true, L, m, R2, m, 0, no, reinterpret_cast<double*>(sh.uni), sA, sB);
    } else {
        for (int i0 = 0; i0 < m; i0 += NB) {
            const int nb = min(NB, m - i0), i1 = i0 + nb;
            for (int t = warp; t < no; t += nwarp) {
                double* x = R2 + (int64_t)t * m;
                double xv = (lane < nb) ? x[i0 + lane] : 0.0;
                for (int k = 0; k < nb; ++k) {
                    if (lane == k) xv /= L[(i0 + k) + (int64_t)(i0 + k) * m];
                    const double xk = __shfl_sync(0xffffffffu, xv, k);
                    if (lane > k && lane < nb) xv -= L[(i0 + lane) + (int64_t)(i0 + k) * m] * xk;
                }
                if (lane < nb) x[i0 + lane] = xv;
            }
            __syncthreads();
            for (int64_t q = tid; q < (int64_t)no * (m - i1); q += kT) {
                const int t = (int)(q / (m - i1)), r = i1 + (int)(q % (m - i1));
                double* x = R2 + (int64_t)t * m;
                double s = 0.0;
                for (int k = 0; k < nb; ++k) s = fma(L[r + (int64_t)(i0 + k) * m], x[i0 + k], s);
                x[r] -= s;
            }
            __syncthreads();
        }
    }
    // R <- R Q: each row x becomes Q^T x (from order 64 as tile products with the
    // panels' T, the divide and conquer's Q and V arenas as scratch)
    if (m >= kWyMmaMin) wy_apply_t(C, m, Ka + p.koff, R, nb2, true, Qa + p.aoff, Va + p.aoff, sA, sB);
    else wy_apply(C, m, tau, R, nb2, true, WySmem{sA, sB});
    __syncthreads();
    // G^T = Z^T R^T (m x 2nown, column-major = G row-major)
    for (int c0 = 0; c0 < nb2; c0 += TS)
        for (int r0 = 0; r0 < m; r0 += TS)
            tile_gemm<true>(G, m, 0, nullptr, r0, c0, min(TS, m - r0), min(TS, nb2 - c0), Z, m, nullptr, R, m, nullptr, m,
                            sA, sB);
    __syncthreads();
    const double* G2 = G + (int64_t)no * m;
    for (int j = tid; j < m; j += kT) {
        double f = 0.0;
        for (int t = 0; t < no; ++t) f = fma(G[(int64_t)t * m + j], G2[(int64_t)t * m + j], f);
        e_out[p.eoff + j] = Wa[p.voff + j];
        fe_out[p.eoff + j] = f;
    }
}

// ---------------------------------------------------------------------------
// Density of one system on one CTA (mode 2): U = L^-T Q Z in place of Z (Q as
// WY tile products, L^-T by blocked back substitution, or one warp per column
// when the divide and conquer's arrays are too small for the 64 x 65 block),
// then the upper tiles of U_occ U_occ^T (K = nocc, the lowest eigenvectors:
// the divide and conquer leaves them ascending) into Ba + boff; the factor 2
// is applied when packing.
__device__ void stage_density(const EigProb& p, const double* __restrict__ Ca, const double* __restrict__ La,
                              const double* __restrict__ Ta, double* __restrict__ Za, double* __restrict__ Qa,
                              double* __restrict__ Va, const double* __restrict__ Ka, double* __restrict__ Ba,
                              const StageSmem& sh) {
    const int m = p.m, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int no = p.nocc;   // only the occupied eigenvectors enter P
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    double* U = Za + p.aoff;
    if (no == 0) return;
    if (m >= kWyMmaMin) wy_apply_t(C, m, Ka + p.koff, U, no, false, Qa + p.aoff, Va + p.aoff, sh.sA, sh.sB);
    else wy_apply(C, m, Ta + p.voff, U, no, false, WySmem{sh.sA, sh.sB});
    __syncthreads();
    if (p.kind == 0) {
        if (dc_smem_bytes(sh.M) >= sizeof(double) * TS * (TS + 1)) {
            trsm_cols(false, L, m, U, m, 0, no, reinterpret_cast<double*>(sh.uni), sh.sA, sh.sB);
        } else {
            for (int t = warp; t < no; t += kT / 32) {
                double* w = U + (int64_t)t * m;
                for (int i = m - 1; i >= 0; --i) {
                    const double* li = L + (int64_t)i * m;
                    double sum = 0.0;
                    for (int k = i + 1 + lane; k < m; k += 32) sum = fma(li[k], w[k], sum);
                    sum = warp_sum(sum);
                    if (lane == 0) w[i] = (w[i] - sum) / li[i];
                    __syncwarp();
                }
            }
        }
    }
    __syncthreads();
    double* P = Ba + p.boff;
    const int nt = (m + TS - 1) / TS;
    for (int cb = 0; cb < nt; ++cb)
        for (int rb = 0; rb <= cb; ++rb)
            tile_mma<false, true, MMA_SET, false>(P, m, 0, nullptr, rb * TS, cb * TS, min(TS, m - rb * TS),
                                                  min(TS, m - cb * TS), U, m, nullptr, U, m, nullptr, p.nocc, sh.sA,
                                                  sh.sB);
}

// ---------------------------------------------------------------------------
// One persistent launch for every submatrix of the step: each CTA takes the
// next submatrix (largest first) from a device counter and runs all stages on
// it - gather, Cholesky, reduction, tridiagonalisation, divide and conquer,
// owned rows and fe - so the uneven sizes balance over the SMs without a
// launch per stage or per size bucket.  status[pi]: 0, the order of a
// non-positive pivot of S_k, or kStNoConv.
__host__ __device__ constexpr size_t stage_smem_bytes(int M) {
    return sizeof(double) * (2 * kStageOp + NB * (NB + 1)) + dc_smem_bytes(M) + sizeof(int) * 16 +
           sizeof(double) * (2 + kT / 32) + 16;
}

__device__ StageSmem stage_smem(unsigned char* base, int M) {
    StageSmem sh;
    double* d = reinterpret_cast<double*>(base);
    sh.sA = d;
    sh.sB = d + kStageOp;
    sh.sD = d + 2 * kStageOp;
    sh.uni = reinterpret_cast<unsigned char*>(d + 2 * kStageOp + NB * (NB + 1));
    sh.ints = reinterpret_cast<int*>(sh.uni + dc_smem_bytes(M));
    sh.dsc = reinterpret_cast<double*>(sh.ints + 16);
    sh.M = M;
    return sh;
}

__global__ void __launch_bounds__(kT, 1) k_eig_fused(
    const EigProb* __restrict__ probs, const int* __restrict__ order, int np, int* __restrict__ counter, int M,
    const int* __restrict__ maps, const double* __restrict__ H, const double* __restrict__ S,
    double* __restrict__ Ca, double* __restrict__ La, double* __restrict__ Za, double* __restrict__ Qa,
    double* __restrict__ Va, double* __restrict__ Da, double* __restrict__ Ea, double* __restrict__ Ta,
    double* __restrict__ Wa, double* __restrict__ Ba, double* __restrict__ Ka, const int* __restrict__ own_cols,
    const int* __restrict__ ipos, double* __restrict__ e_out, double* __restrict__ fe_out,
    int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const StageSmem sh = stage_smem(smraw, M);
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) sh.ints[15] = atomicAdd(counter, 1);
        __syncthreads();
        const int q = sh.ints[15];
        __syncthreads();
        if (q >= np) break;
        const int pi = order[q];
        const EigProb p = probs[pi];
        stage_gather(p, maps, H, S, Ca, La);
        __syncthreads();
        int st = stage_potrf(p, La, sh);
        __syncthreads();
        if (st == kStOk) {
            stage_reduce(p, La, Ca, sh);
            __syncthreads();
            stage_sytrd(p, Ca, Da, Ea, Ta, sh);
            __syncthreads();
            if (!stage_dc(p, Da, Ea, Wa, Za, Qa, Va, sh)) st = kStNoConv;
            __syncthreads();
            if (st == kStOk) {
                if (p.m >= kWyMmaMin)
                    build_T(Ca + p.aoff, p.m, Ta + p.voff, Ka + p.koff, 0, 1, Va + p.aoff, sh.sD, sh.sA, sh.sB);
                if (p.mode == 2) {
                    for (int j = threadIdx.x; j < p.m; j += kT) e_out[p.eoff + j] = Wa[p.voff + j];
                    stage_density(p, Ca, La, Ta, Za, Qa, Va, Ka, Ba, sh);
                } else {
                    stage_rows(p, Ca, La, Ta, Wa, Za, own_cols, ipos, Ba, Qa, Va, Ka, e_out, fe_out, sh);
                }
            }
        }
        if (tid == 0) status[pi] = st;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Owned columns of P_k at mu: w_t = occ o U[c_t,:]^T, w <- Z w, w <- Q w
// (reflectors in reverse), w <- L^-T w; scattered into the packed result,
// rows map(i) <= c_t of column c_t (or written dense).
// Shared memory of the final-column kernels: tile staging, a 64 x 65 diagonal
// block of L and the panel's T.
constexpr size_t kFinalSmem = sizeof(double) * (2 * kStageOp + TS * (TS + 1) + NB * (NB + 1));

__global__ void __launch_bounds__(kT) k_eig_final(const EigProb* __restrict__ probs, const int* __restrict__ order,
                                                  const double* __restrict__ Ca,
                                                  const double* __restrict__ La, const double* __restrict__ Ta,
                                                  const double* __restrict__ Wa, const double* __restrict__ Za,
                                                  double* __restrict__ Qa, double* __restrict__ Va,
                                                  const double* __restrict__ Ka,
                                                  const int* __restrict__ maps, const int* __restrict__ own_cols,
                                                  double* __restrict__ Ba, double mu, double* __restrict__ Ppk,
                                                  double* __restrict__ Pdense) {
    extern __shared__ __align__(16) unsigned char smf[];
    double* sA = reinterpret_cast<double*>(smf);
    double* sB = sA + kStageOp;
    double* sD = sB + kStageOp;
    double* sT = sD + TS * (TS + 1);
    const EigProb p = probs[order[blockIdx.x]];
    const int m = p.m, no = p.nown;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* Z = Za + p.aoff;
    const double* tau = Ta + p.voff;
    const double* ev = Wa + p.voff;
    double* W0 = Ba + p.boff;                       // (S U) rows block: free after the prepare step
    const double* U2 = Ba + p.boff + 3 * (int64_t)no * m;   // U[c_t, :] (second half of G)
    double* W = Ba + p.boff + (int64_t)no * m;      // m x nown, column-major
    const int tid = threadIdx.x;
    for (int64_t q = tid; q < (int64_t)no * m; q += kT) {
        const int j = (int)(q % m);
        const double e = ev[j];
        const double occ = e < mu ? 2.0 : (e == mu ? 1.0 : 0.0);
        W0[q] = occ * U2[q];
    }
    __syncthreads();
    // W = Z W0
    for (int c0 = 0; c0 < no; c0 += TS)
        for (int r0 = 0; r0 < m; r0 += TS)
            tile_gemm<false>(W, m, 0, nullptr, r0, c0, min(TS, m - r0), min(TS, no - c0), Z, m, nullptr, W0, m, nullptr, m,
                             sA, sB);
    __syncthreads();
    // Q W (from order 64 as tile products, the divide and conquer's arenas as scratch)
    if (m >= kWyMmaMin) wy_apply_t(C, m, Ka + p.koff, W, no, false, Qa + p.aoff, Va + p.aoff, sA, sB);
    else wy_apply(C, m, tau, W, no, false, WySmem{sA, sB});
    __syncthreads();
    // L^-T W: blocked back substitution
    trsm_cols(false, L, m, W, m, 0, no, sD, sA, sB);
    if (Pdense) {
        for (int64_t q = tid; q < (int64_t)no * m; q += kT) Pdense[p.poff + q] = W[q];
        return;
    }
    const int* mp = maps + p.moff;
    for (int64_t q = tid; q < (int64_t)no * m; q += kT) {
        const int t = (int)(q / m), i = (int)(q % m);
        const int64_t cgl = own_cols[p.o0 + t];
        const int64_t gi = mp[i];
        if (gi <= cgl) Ppk[cgl * (cgl + 1) / 2 + gi] = W[q];
    }
}


// ===========================================================================
// Submatrices above kEigBatchMax (the k-means columns of large boxes): the
// same stages on a thread-block cluster of G CTAs per submatrix, one cluster
// barrier (barrier.cluster) between dependent steps and every intermediate in
// global memory (L2-resident for the vectors and panels).
//   gather       columns split over the CTAs
//   Cholesky     32-wide panels: the diagonal block factored by every CTA (same
//                data, same arithmetic, same result), panel rows and lower
//                trailing tiles split over the CTAs
//   reduction    C = L^-1 H L^-T: left-looking triangular solves over 64-row
//                blocks, each CTA owning 64-column blocks of C (no barrier
//                inside a solve)
//   tridiag.     blocked Householder with lazy updates (LAPACK's latrd
//                scheme): per column the panel's earlier reflectors update that
//                column, the reflector is formed, and y = A v runs over the
//                lower 64 x 64 tiles of the not yet updated trailing block (each
//                tile read once for both its row and its column contribution),
//                corrected by V (W^T v) + W (V^T v); w = tau (y - tau/2 (y.v) v);
//                after 32 columns the trailing block gets A -= V W^T + W V^T.
//                Rows are owned in 32-row chunks, partial sums go through
//                per-CTA slots summed in CTA order, so results do not depend on
//                scheduling.  Two cluster barriers per column.
//   D&C          leaves and the lower merges one CTA each, merges with fewer
//                problems than CTAs by the whole cluster
//   owned rows   vectors split over the CTAs, then one tiled product with Z
// ===========================================================================
constexpr int kLargeMax = kEigLargeMax;   // largest order the cluster solver takes (its vectors live in shared memory)
constexpr int kRedW = 2 * NB + 4;         // per-CTA partial sums of the tridiagonalisation
constexpr int kRedVAv = 2 * NB + 1;       // slot of the partial v^T A v
constexpr int kLgStages = 6;              // stage timestamps per problem: start, Cholesky, reduction, tridiag., D&C, rows
constexpr int kLgSub = 7;                 // tridiagonalisation phase times per problem (ns, summed over its columns)
constexpr int kLgStride = kLgStages + kLgSub;

// Phase clock of one thread (rank 0, thread 0 of a cluster when stage times are
// requested): lap(q) adds the time since the previous lap to acc[q].
struct PhaseClock {
    unsigned long long* acc;
    unsigned long long t;
    __device__ __forceinline__ static unsigned long long now() {
        unsigned long long v;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
        return v;
    }
    __device__ __forceinline__ void start() {
        if (acc) t = now();
    }
    __device__ __forceinline__ void lap(int q) {
        if (acc) {
            const unsigned long long n = now();
            acc[q] += n - t;
            t = n;
        }
    }
};

// Software barrier over the CTAs of a cooperative launch (all resident):
// bar[0] counts arrivals, bar[1] is the generation.  The wait is bounded: after
// kGridSpin polls the CTA records the failure in *err and goes on, and every
// later barrier returns at once, so a kernel whose barrier gave up still ends
// (its results are then discarded by the host, which reports the timeout).
constexpr long long kGridSpin = 1ll << 24;

__device__ void grid_barrier(unsigned* bar, int nblocks, int* err) {
    __syncthreads();
    if (threadIdx.x == 0 && *(volatile int*)err == 0) {
        volatile unsigned* vb = bar;
        const unsigned gen = vb[1];
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == (unsigned)nblocks - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            long long it = 0;
            while (vb[1] == gen) {
                if (++it > kGridSpin) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// The CTAs that solve one problem together: a thread-block cluster (bar null,
// hardware barrier) or the whole grid of a cooperative launch (software barrier).
struct Grp {
    int rank, size;
    unsigned* bar;
    int* err;
    __device__ __forceinline__ void sync() const {
        if (!bar) cg::this_cluster().sync();
        else grid_barrier(bar, size, err);
    }
};

// Per-problem scratch of a cluster solve (offsets in doubles from p.xoff).
struct LgLayout {
    int64_t rowp, colp, red, V, W, dc, scal, total;
};
constexpr int kSegW = 64;    // columns of one A v work unit of the tridiagonalisation
constexpr int kAvGrp = 8;    // columns whose loads are issued together in the A v units
__host__ __device__ inline LgLayout lg_layout(int m, int G) {
    LgLayout L;
    int64_t o = 0;
    L.rowp = o;   // row sums of the A v units: [segment][m]
    o += (int64_t)((m + kSegW - 1) / kSegW + 1) * m;
    L.colp = o;   // column sums of the A v units: [64-row block][m]
    o += (int64_t)((m + TS - 1) / TS) * m;
    L.red = o;
    o += (int64_t)G * kRedW;
    L.V = o;
    o += (int64_t)m * NB;
    L.W = o;
    o += (int64_t)m * NB;
    o = (o + 1) & ~int64_t(1);
    L.dc = o;
    o += (int64_t)((dc_smem_bytes((m + 1) & ~1) + 15) / 16) * 2;
    L.scal = o;
    o += ((int64_t)m + 64) / 2 + 2;   // 8 ints per merge of the widest level (at most m / 16 merges)
    L.total = (o + 1) & ~int64_t(1);
    return L;
}

struct LgSmem {
    double *sA, *sB;           // tile staging
    double* sD;                // diagonal blocks (TS x (TS+1)), union with the vectors below
    double *v, *y;             // tridiagonalisation: reflector and updated column (M each)
    double *pw, *pv, *wtv, *vtv, *wj, *vj;   // NB each
    double* red;               // kT / 32 + 2
    double* dsc;               // scalars
    int* ints;                 // 16
};
__host__ __device__ constexpr size_t lg_union_doubles(int M) {
    return (size_t)2 * M + 6 * NB + kT / 32 + 2 + 8 > (size_t)TS * (TS + 1) ? (size_t)2 * M + 6 * NB + kT / 32 + 2 + 8
                                                                            : (size_t)TS * (TS + 1);
}
__host__ __device__ constexpr size_t lg_smem_bytes(int M) {
    return sizeof(double) * (2 * kStageOp + lg_union_doubles(M)) + sizeof(int) * 16;
}
static_assert(lg_smem_bytes(kLargeMax) <= 232448, "cluster solver shared memory within the per-CTA limit");
__device__ LgSmem lg_smem(unsigned char* base, int M) {
    LgSmem s;
    double* d = reinterpret_cast<double*>(base);
    s.sA = d;
    s.sB = d + kStageOp;
    double* u = d + 2 * kStageOp;
    s.sD = u;
    s.v = u;
    s.y = u + M;
    s.pw = s.y + M;
    s.pv = s.pw + NB;
    s.wtv = s.pv + NB;
    s.vtv = s.wtv + NB;
    s.wj = s.vtv + NB;
    s.vj = s.wj + NB;
    s.red = s.vj + NB;
    s.dsc = s.red + kT / 32 + 2;
    s.ints = reinterpret_cast<int*>(u + lg_union_doubles(M));
    return s;
}

// Lower-triangle tile index -> (row block, column block), rb >= cb.
__device__ __forceinline__ void tri_decode(int64_t idx, int& rb, int& cb) {
    int r = (int)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while ((int64_t)(r + 1) * (r + 2) / 2 <= idx) ++r;
    while ((int64_t)r * (r + 1) / 2 > idx) --r;
    rb = r;
    cb = (int)(idx - (int64_t)r * (r + 1) / 2);
}

__device__ void lg_gather(const Grp& g, const EigProb& p, const int* __restrict__ maps, const double* __restrict__ H,
                          const double* __restrict__ S, double* __restrict__ Ca, double* __restrict__ La) {
    const int m = p.m;
    const int* mp = maps + p.moff;
    double* C = Ca + p.aoff;
    double* L = La + p.aoff;
    for (int j = g.rank; j < m; j += g.size) {
        const int64_t gj = p.gbase + (int64_t)mp[j] * p.gld;
        for (int i = threadIdx.x; i < m; i += kT) {
            const int64_t q = (int64_t)mp[i] + gj;
            C[i + (int64_t)j * m] = H[q];
            if (p.kind == 0) L[i + (int64_t)j * m] = S[q];
        }
    }
}

// S_k = L L^T (lower) on the cluster; returns the order of the first
// non-positive pivot (0: positive definite), the same on every CTA.
__device__ int lg_potrf(const Grp& g, int m, double* __restrict__ L, const LgSmem& sh) {
    double* sD = sh.sD;   // sD[i + j*(NB+1)]
    int& fail = sh.ints[0];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail = 0;
    __syncthreads();
    for (int kb = 0; kb < m; kb += NB) {
        const int nb = min(NB, m - kb);
        for (int t = tid; t < NB * NB; t += kT) {
            const int i = t % NB, j = t / NB;
            sD[i + j * (NB + 1)] = (i < nb && j < nb) ? L[(int64_t)(kb + i) + (int64_t)(kb + j) * m] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int jj = 0; jj < nb; ++jj) {
                if (lane == jj) {
                    const double piv = sD[jj + jj * (NB + 1)];
                    if (!(piv > 0.0)) fail = kb + jj + 1;
                    else sD[jj + jj * (NB + 1)] = sqrt(piv);
                }
                __syncwarp();
                if (fail) break;
                const double djj = sD[jj + jj * (NB + 1)];
                if (lane > jj && lane < nb) sD[lane + jj * (NB + 1)] /= djj;
                __syncwarp();
                if (lane > jj && lane < nb) {
                    const double lij = sD[lane + jj * (NB + 1)];
                    for (int k = jj + 1; k <= lane; ++k) sD[lane + k * (NB + 1)] -= lij * sD[k + jj * (NB + 1)];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        if (fail) break;   // every CTA factored the same block: the same decision everywhere
        if (g.rank == 0)
            for (int t = tid; t < nb * nb; t += kT) {
                const int i = t % nb, j = t / nb;
                if (i >= j) L[(int64_t)(kb + i) + (int64_t)(kb + j) * m] = sD[i + j * (NB + 1)];
            }
        for (int r = kb + nb + g.rank * kT + tid; r < m; r += g.size * kT) {
            double x[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) x[j] = (j < nb) ? L[(int64_t)r + (int64_t)(kb + j) * m] : 0.0;
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (j < nb) {
                    double v = x[j];
                    for (int k = 0; k < j; ++k) v -= x[k] * sD[j + k * (NB + 1)];
                    x[j] = v / sD[j + j * (NB + 1)];
                }
            }
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) L[(int64_t)r + (int64_t)(kb + j) * m] = x[j];
        }
        g.sync();
        const int t0 = kb + nb;
        const int nt = (m - t0 + TS - 1) / TS;
        const int64_t ntile = (int64_t)nt * (nt + 1) / 2;
        for (int64_t idx = g.rank; idx < ntile; idx += g.size) {
            int rb, cb;
            tri_decode(idx, rb, cb);
            const int r0 = t0 + rb * TS, c0 = t0 + cb * TS;
            tile_update<true, true>(L, m, r0, c0, min(TS, m - r0), min(TS, m - c0), L + (int64_t)kb * m, m,
                                    L + (int64_t)kb * m, m, nb, sh.sA, sh.sB);
        }
        g.sync();
    }
    __syncthreads();
    const int f = fail;
    __syncthreads();
    if (f) return f;
    for (int j = 1 + g.rank; j < m; j += g.size)
        for (int i = tid; i < j; i += kT) L[(int64_t)i + (int64_t)j * m] = 0.0;
    return 0;
}

// X <- L^-1 X for the 64-column blocks cb = rank, rank + G, ... of X (m x m):
// left-looking over 64-row blocks, X_i -= L[i, <i] X[<i] as one tile product,
// then the diagonal block's forward substitution (warp per column, two rows per
// lane).  The column blocks are independent, so no cluster barrier is needed.
__device__ void lg_trsm_cols(const Grp& g, const double* __restrict__ L, double* X, int m, const LgSmem& sh) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* sD = sh.sD;   // sD[i + j*(TS+1)]
    const int ncb = (m + TS - 1) / TS;
    for (int cb = g.rank; cb < ncb; cb += g.size) {
        const int c0 = cb * TS, nc = min(TS, m - c0);
        for (int i0 = 0; i0 < m; i0 += TS) {
            const int mr = min(TS, m - i0);
            if (i0 > 0)
                tile_mma<false, false, MMA_SUB, false>(X, m, 0, nullptr, i0, c0, mr, nc, L, m, nullptr, X, m, nullptr,
                                                       i0, sh.sA, sh.sB);
            for (int t = tid; t < TS * TS; t += kT) {
                const int i = t % TS, j = t / TS;
                sD[i + j * (TS + 1)] = (i < mr && j < mr && i >= j) ? L[(int64_t)(i0 + i) + (int64_t)(i0 + j) * m] : 0.0;
            }
            __syncthreads();
            for (int jc = warp; jc < nc; jc += kT / 32) {
                double* x = X + (int64_t)(c0 + jc) * m + i0;
                double x0 = lane < mr ? x[lane] : 0.0, x1 = lane + 32 < mr ? x[lane + 32] : 0.0;
                for (int k = 0; k < mr; ++k) {
                    double xk;
                    if (k < 32) {
                        if (lane == k) x0 /= sD[k + k * (TS + 1)];
                        xk = __shfl_sync(0xffffffffu, x0, k);
                    } else {
                        if (lane == k - 32) x1 /= sD[k + k * (TS + 1)];
                        xk = __shfl_sync(0xffffffffu, x1, k - 32);
                    }
                    if (lane > k && lane < mr) x0 -= sD[lane + k * (TS + 1)] * xk;
                    if (lane + 32 > k && lane + 32 < mr) x1 -= sD[lane + 32 + k * (TS + 1)] * xk;
                }
                if (lane < mr) x[lane] = x0;
                if (lane + 32 < mr) x[lane + 32] = x1;
            }
            __syncthreads();
        }
    }
}

// C <- L^-1 H_k L^-T: C <- L^-1 C, transpose, C <- L^-1 C (only the lower
// triangle is read afterwards).
__device__ void lg_reduce(const Grp& g, const EigProb& p, const double* __restrict__ La, double* Ca,
                          const LgSmem& sh) {
    const int m = p.m;
    const double* L = La + p.aoff;
    double* C = Ca + p.aoff;
    lg_trsm_cols(g, L, C, m, sh);
    g.sync();
    const int64_t mm = (int64_t)m * m;
    for (int64_t t = (int64_t)g.rank * kT + threadIdx.x; t < mm; t += (int64_t)g.size * kT) {
        const int i = (int)(t % m), j = (int)(t / m);
        if (i > j) {
            const double a = C[i + (int64_t)j * m], b = C[j + (int64_t)i * m];
            C[i + (int64_t)j * m] = b;
            C[j + (int64_t)i * m] = a;
        }
    }
    g.sync();
    lg_trsm_cols(g, L, C, m, sh);
    g.sync();
}

// w of reflector jp (column j - 1 of the panel's first column j0 = j - 1 - jp)
// on this CTA's rows r >= j, from the summed partial products; the reflector
// itself goes into column j - 1 below its leading 1.  Returns w at row j
// (every CTA computes it).
// Units of the A v pass for the trailing block from row/column s: tile rows
// I in [s/64, nT), each cut into kSegW-column segments from column 64 (s/64).
__device__ __forceinline__ int av_nseg(int I, int cstart) {
    return ((I + 1) * TS - cstart + kSegW - 1) / kSegW;
}

// w of column jp of the panel (the column before j) on this CTA's rows, with the
// reflector stored into A's column j-1; w_j itself goes to sh.wj[jp], computed
// by the last warp beside the row loop.  The caller synchronises the CTA.
__device__ void lg_finish_w(const Grp& g, int m, int j, int jp, double* __restrict__ A, double* __restrict__ V,
                            double* __restrict__ W, const double* __restrict__ rowp,
                            const double* __restrict__ colp, const double* __restrict__ red, const LgSmem& sh) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double tp = sh.dsc[0];
    double vAv = 0.0;
    for (int q = 0; q < g.size; ++q) vAv += red[q * kRedW + kRedVAv];
    double vw = 0.0;
    for (int q = 0; q < jp; ++q) vw = fma(sh.vtv[q], sh.wtv[q], vw);
    const double ytv = vAv - 2.0 * vw;
    const double hc = 0.5 * tp * ytv;
    const int cstart = (j / TS) * TS, nT = (m + TS - 1) / TS;
    auto w_at = [&](int r) {
        // y_r = its row sums over the segments of its tile row, then its column
        // sums over the tile rows at and below its own, in that fixed order
        const int Ir = r / TS;
        double y = 0.0;
        const int ns = av_nseg(Ir, cstart);
        for (int q = 0; q < ns; ++q) y += rowp[(int64_t)q * m + r];
        for (int I = Ir; I < nT; ++I) y += colp[(int64_t)I * m + r];
        for (int q = 0; q < jp; ++q) y -= V[r + (int64_t)q * m] * sh.wtv[q] + W[r + (int64_t)q * m] * sh.vtv[q];
        return tp * (y - hc * sh.v[r]);
    };
    if (tid == kT - 32 && j < m) sh.wj[jp] = w_at(j);
    for (int ch = g.rank + g.size * warp; ch * 32 < m; ch += g.size * (kT / 32)) {
        const int r = ch * 32 + lane;
        if (r >= j && r < m) {
            W[r + (int64_t)jp * m] = w_at(r);
            if (r >= j + 1) A[r + (int64_t)(j - 1) * m] = sh.v[r];
        }
    }
}

__device__ void lg_sytrd(const Grp& g, const EigProb& p, double* __restrict__ Ca, double* __restrict__ Da,
                         double* __restrict__ Ea, double* __restrict__ Ta, double* __restrict__ X, const LgSmem& sh,
                         unsigned long long* tsub) {
    const int m = p.m, G = g.size, rk = g.rank;
    PhaseClock pc{(g.rank == 0 && threadIdx.x == 0) ? tsub : nullptr, 0};
    pc.start();
    double* A = Ca + p.aoff;
    double* d = Da + p.voff;
    double* e = Ea + p.voff;
    double* tau = Ta + p.voff;
    const LgLayout lay = lg_layout(m, G);
    double* rowp = X + lay.rowp;
    double* colp = X + lay.colp;
    double* red = X + lay.red;
    double* V = X + lay.V;
    double* W = X + lay.W;
    double* v = sh.v;
    double* yl = sh.y;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nT = (m + TS - 1) / TS;
    for (int j0 = 0; j0 < m - 1; j0 += NB) {
        const int nb = min(NB, m - 1 - j0);
        for (int jj = 0; jj < nb; ++jj) {
            const int j = j0 + jj;
            // ---- phase A: finish w of the previous column, update column j on own rows
            // (row j of the panel's V and earlier W columns were written before the
            // last cluster barrier; w_j of the previous column comes from lg_finish_w)
            if (tid < jj) {
                if (tid < jj - 1) sh.wj[tid] = W[j + (int64_t)tid * m];
                sh.vj[tid] = V[j + (int64_t)tid * m];
            }
            if (jj > 0) lg_finish_w(g, m, j, jj - 1, A, V, W, rowp, colp, red, sh);
            __syncthreads();
            for (int ch = rk + G * warp; ch * 32 < m; ch += G * (kT / 32)) {
                const int r = ch * 32 + lane;
                if (r >= j && r < m) {
                    double a = A[r + (int64_t)j * m];
                    for (int q = 0; q < jj; ++q)
                        a -= V[r + (int64_t)q * m] * sh.wj[q] + W[r + (int64_t)q * m] * sh.vj[q];
                    A[r + (int64_t)j * m] = a;
                    yl[r] = a;
                }
            }
            __syncthreads();
            {
                double part = 0.0;
                for (int ch = rk + G * warp; ch * 32 < m; ch += G * (kT / 32)) {
                    const int r = ch * 32 + lane;
                    if (r >= j + 2 && r < m) part = fma(yl[r], yl[r], part);
                }
                part = cta_sum(part, sh.red);
                if (tid == 0) red[rk * kRedW + 0] = part;
            }
            for (int q = warp; q < 2 * jj; q += kT / 32) {
                const double* col = (q < jj) ? W + (int64_t)q * m : V + (int64_t)(q - jj) * m;
                double part = 0.0;
                for (int ch = rk; ch * 32 < m; ch += G) {
                    const int r = ch * 32 + lane;
                    if (r >= j + 2 && r < m) part = fma(col[r], yl[r], part);
                }
                part = warp_sum(part);
                if (lane == 0) red[rk * kRedW + ((q < jj) ? 1 + q : 1 + NB + (q - jj))] = part;
            }
            pc.lap(0);
            g.sync();
            pc.lap(1);
            // ---- phase B: reflector, then y = A v over the trailing lower tiles
            // (column j below the subdiagonal is read into v while the scale is
            // formed, and scaled in shared memory after the barrier)
            double wj1 = 0.0, vj1 = 0.0;
            if (tid < jj) {
                double a = 0.0, b = 0.0;
                for (int q = 0; q < G; ++q) {
                    a += red[q * kRedW + 1 + tid];
                    b += red[q * kRedW + 1 + NB + tid];
                }
                sh.pw[tid] = a;
                sh.pv[tid] = b;
                wj1 = W[(j + 1) + (int64_t)tid * m];
                vj1 = V[(j + 1) + (int64_t)tid * m];
            }
            for (int r = j + 2 + tid; r < m; r += kT) v[r] = A[r + (int64_t)j * m];
            if (tid == 32) {
                double xn2 = 0.0;
                for (int q = 0; q < G; ++q) xn2 += red[q * kRedW + 0];
                const double alpha = A[(j + 1) + (int64_t)j * m];
                const double dj = A[j + (int64_t)j * m];
                double t, beta;
                if (xn2 == 0.0) {
                    t = 0.0;
                    beta = alpha;
                } else {
                    beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                    t = (beta - alpha) / beta;
                }
                sh.dsc[0] = t;
                sh.dsc[1] = (t == 0.0) ? 0.0 : 1.0 / (alpha - beta);
                if (rk == 0) {
                    d[j] = dj;
                    e[j] = beta;
                    tau[j] = t;
                }
            }
            __syncthreads();
            const double sc = sh.dsc[1];
            for (int r = tid; r < m; r += kT) {
                double vr;
                if (r <= j) vr = 0.0;
                else if (r == j + 1) vr = 1.0;
                else vr = (sc == 0.0) ? 0.0 : v[r] * sc;
                v[r] = vr;
            }
            if (tid < jj) {
                sh.wtv[tid] = wj1 + sc * sh.pw[tid];
                sh.vtv[tid] = vj1 + sc * sh.pv[tid];
            }
            const int s = j + 1;
            for (int r = s + tid; r < m; r += kT) yl[r] = 0.0;
            __syncthreads();
            for (int ch = rk + G * warp; ch * 32 < m; ch += G * (kT / 32)) {
                const int r = ch * 32 + lane;
                if (r >= s && r < m) V[r + (int64_t)jj * m] = v[r];
            }
            pc.lap(2);
            // A v over the trailing lower triangle, one pass: every warp streams
            // its own units (64 rows x kSegW columns of one tile row) without a
            // barrier, lane holding rows I*64 + lane and + 32: the row sums stay
            // in registers for the unit, each column's sum is a warp reduction;
            // both go to their own slots (rowp[segment][r], colp[tile row][c]),
            // summed in a fixed order when w is formed.  v^T A v comes from the
            // same sums.  Warps are numbered across the CTAs (warp-major), so
            // consecutive units land on different SMs: with fewer units than
            // warps (small orders) every SM's L2 bandwidth still takes part.
            {
                const int I0 = s / TS, cstart = I0 * TS;
                const int gw = warp * G + rk, nw = G * (kT / 32);
                double vav = 0.0;
                int I = I0, ubase = 0;
                for (int u = gw;; u += nw) {
                    while (I < nT && u >= ubase + av_nseg(I, cstart)) {
                        ubase += av_nseg(I, cstart);
                        ++I;
                    }
                    if (I >= nT) break;
                    const int seg = u - ubase;
                    const int c_lo = cstart + seg * kSegW;
                    const int c_hi = min(min(c_lo + kSegW, (I + 1) * TS), m);
                    const int r0 = I * TS + lane, r1 = r0 + 32;
                    const double v0 = (r0 < m) ? v[r0] : 0.0, v1 = (r1 < m) ? v[r1] : 0.0;
                    const double* A0 = A + r0;
                    const double* A1 = A + r1;
                    double rp0 = 0.0, rp1 = 0.0;
                    for (int cb = c_lo; cb < c_hi; cb += 32) {
                        double mycol = 0.0;
#pragma unroll 1
                        for (int g8 = 0; g8 < 32; g8 += kAvGrp) {
                            double a0[kAvGrp], a1[kAvGrp];
#pragma unroll
                            for (int u8 = 0; u8 < kAvGrp; ++u8) {
                                const int c = cb + g8 + u8;
                                const bool cok = c < c_hi && c >= s;
                                a0[u8] = (cok && r0 < m && c <= r0) ? A0[(int64_t)c * m] : 0.0;
                                a1[u8] = (cok && r1 < m && c <= r1) ? A1[(int64_t)c * m] : 0.0;
                            }
#pragma unroll
                            for (int u8 = 0; u8 < kAvGrp; ++u8) {
                                const int c = cb + g8 + u8;
                                const double vc = (c < c_hi) ? v[c] : 0.0;
                                rp0 = fma(a0[u8], vc, rp0);
                                rp1 = fma(a1[u8], vc, rp1);
                                double cp = ((c < r0) ? a0[u8] * v0 : 0.0) + ((c < r1) ? a1[u8] * v1 : 0.0);
                                cp = warp_sum(cp);
                                if (lane == g8 + u8) mycol = cp;
                            }
                        }
                        const int c = cb + lane;
                        if (c < c_hi) {
                            colp[(int64_t)I * m + c] = mycol;
                            vav = fma(v[c], mycol, vav);
                        }
                    }
                    if (r0 < m) rowp[(int64_t)seg * m + r0] = rp0;
                    if (r1 < m) rowp[(int64_t)seg * m + r1] = rp1;
                    vav = fma(v0, rp0, fma(v1, rp1, vav));
                }
                pc.lap(3);
                const double part = cta_sum(vav, sh.red);
                if (tid == 0) red[rk * kRedW + kRedVAv] = part;
            }
            pc.lap(4);
            g.sync();
            pc.lap(5);
        }
        // ---- panel end: w of the last column, then the trailing block
        const int j1 = j0 + nb;
        lg_finish_w(g, m, j1, nb - 1, A, V, W, rowp, colp, red, sh);
        g.sync();
        if (j1 < m) {
            const int nt = (m - j1 + TS - 1) / TS;
            const int64_t ntile = (int64_t)nt * (nt + 1) / 2;
            for (int64_t idx = rk; idx < ntile; idx += G) {
                int rb, cb;
                tri_decode(idx, rb, cb);
                const int r0 = j1 + rb * TS, c0 = j1 + cb * TS;
                const int mr = min(TS, m - r0), nc = min(TS, m - c0);
                tile_update<true, true>(A, m, r0, c0, mr, nc, V, m, W, m, nb, sh.sA, sh.sB);
                tile_update<true, true>(A, m, r0, c0, mr, nc, W, m, V, m, nb, sh.sA, sh.sB);
            }
        }
        g.sync();
        pc.lap(6);
    }
    if (rk == 0 && tid == 0) {
        d[m - 1] = A[(m - 1) + (int64_t)(m - 1) * m];
        tau[m - 1] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// Divide and conquer on a cluster.  A merge is run by one CTA (Split{0, 1,
// false}) or by the whole group (Split{rank, G, true}); its per-element
// arrays sit at offset lo of the problem's arrays, its Q and V blocks at
// column lo of the Q and V arenas, so merges of one level never overlap.
struct Split {
    int part, nparts;
    bool coop;
    const Grp* g;
    __device__ __forceinline__ void sync() const {
        if (coop) g->sync();
        else __syncthreads();
    }
    __device__ __forceinline__ int first() const { return part * kT + (int)threadIdx.x; }
    __device__ __forceinline__ int step() const { return nparts * kT; }
    __device__ __forceinline__ bool lead() const { return part == 0 && threadIdx.x == 0; }
};

__device__ DcSmem dc_shift(const DcSmem& S, int lo) {
    DcSmem q = S;
    q.Ds += lo;
    q.zs += lo;
    q.dk += lo;
    q.zk += lo;
    q.tau += lo;
    q.zh += lo;
    q.val += lo;
    q.perm += lo;
    q.org += lo;
    q.sec += lo;
    q.dl += lo;
    q.rank += lo;
    q.cls += lo;
    q.ktop += lo;
    q.kbot += lo;
    q.rpair += lo;
    q.rcs += lo;
    return q;
}

__device__ void dc_merge(const Split& sp, int m, int lo, int mid, int hi, double beta, const DcSmem& S,
                         double* __restrict__ Z, double* __restrict__ Qp, double* __restrict__ V, int* sc, double* sA,
                         double* sB) {
    const DcSmem Q = dc_shift(S, lo);
    const int n1 = mid - lo, n2 = hi - mid, n = n1 + n2;
    const double rho = 2.0 * fabs(beta);
    const double sgn = beta >= 0.0 ? 1.0 : -1.0;
    const double rs2 = 0.70710678118654752440;
    const double eps = 2.220446049250313e-16;
    const int f0 = sp.first(), st = sp.step();
    // (a) merged order of the two sorted blocks
    for (int j = f0; j < n; j += st) {
        int r;
        if (j < n1) {
            const double x = S.D[lo + j];
            int a = 0, b = n2;
            while (a < b) {
                const int c = (a + b) >> 1;
                if (S.D[mid + c] < x) a = c + 1;
                else b = c;
            }
            r = j + a;
        } else {
            const double x = S.D[mid + j - n1];
            int a = 0, b = n1;
            while (a < b) {
                const int c = (a + b) >> 1;
                if (S.D[lo + c] <= x) a = c + 1;
                else b = c;
            }
            r = (j - n1) + a;
        }
        Q.perm[r] = j;
    }
    sp.sync();
    // (b) sorted d, z and column classes; (c) Q with the block columns in that order
    for (int r = f0; r < n; r += st) {
        const int j = Q.perm[r];
        if (j < n1) {
            Q.Ds[r] = S.D[lo + j];
            Q.zs[r] = Z[(int64_t)(mid - 1) + (int64_t)(lo + j) * m] * rs2;
            Q.cls[r] = 1;
        } else {
            Q.Ds[r] = S.D[mid + j - n1];
            Q.zs[r] = sgn * Z[(int64_t)mid + (int64_t)(mid + j - n1) * m] * rs2;
            Q.cls[r] = 2;
        }
    }
    for (int64_t t = f0; t < (int64_t)n * n; t += st) {
        const int i = (int)(t % n), r = (int)(t / n);
        const int j = Q.perm[r];
        double v = 0.0;
        if (j < n1) {
            if (i < n1) v = Z[(int64_t)(lo + i) + (int64_t)(lo + j) * m];
        } else if (i >= n1) {
            v = Z[(int64_t)(lo + i) + (int64_t)(mid + j - n1) * m];
        }
        Qp[t] = v;
    }
    sp.sync();
    // (d) deflation (one thread, in sorted order)
    if (sp.lead()) {
        double dmax = 0.0;
        for (int r = 0; r < n; ++r) dmax = fmax(dmax, fabs(Q.Ds[r]));
        const double tol = 8.0 * eps * fmax(dmax, rho);
        int k = 0, nd = 0, nrot = 0, pj = -1;
        for (int r = 0; r < n; ++r) {
            if (rho * fabs(Q.zs[r]) <= tol) {
                Q.dl[nd++] = r;
                continue;
            }
            if (pj < 0) {
                pj = r;
                continue;
            }
            double sn = Q.zs[pj], c = Q.zs[r];
            const double t = hypot(c, sn);
            const double dd = Q.Ds[r] - Q.Ds[pj];
            c /= t;
            sn = -sn / t;
            if (fabs(dd * c * sn) <= tol) {
                Q.zs[r] = t;
                Q.zs[pj] = 0.0;
                Q.rpair[nrot] = make_int2(pj, r);
                Q.rcs[nrot] = make_double2(c, sn);
                ++nrot;
                const double t2 = Q.Ds[pj] * c * c + Q.Ds[r] * sn * sn;
                Q.Ds[r] = Q.Ds[pj] * sn * sn + Q.Ds[r] * c * c;
                Q.Ds[pj] = t2;
                Q.cls[r] |= Q.cls[pj];
                Q.dl[nd++] = pj;
                pj = r;
            } else {
                Q.sec[k++] = pj;
                pj = r;
            }
        }
        if (pj >= 0) Q.sec[k++] = pj;
        int nt = 0, nb = 0;
        for (int t = 0; t < k; ++t) {
            const int c = Q.cls[Q.sec[t]];
            if (c & 1) Q.ktop[nt++] = t;
            if (c & 2) Q.kbot[nb++] = t;
        }
        sc[0] = k;
        sc[1] = nd;
        sc[2] = nrot;
        sc[3] = nt;
        sc[4] = nb;
    }
    sp.sync();
    const volatile int* vsc = sc;
    const int k = vsc[0], nd = vsc[1], nrot = vsc[2], ntop = vsc[3], nbot = vsc[4];
    // (e) deflation rotations on the columns of Q (thread per row)
    if (nrot > 0)
        for (int i = f0; i < n; i += st)
            for (int q2 = 0; q2 < nrot; ++q2) {
                const int2 pr = Q.rpair[q2];
                const double2 cs = Q.rcs[q2];
                const double a = Qp[i + (int64_t)pr.x * n], b = Qp[i + (int64_t)pr.y * n];
                Qp[i + (int64_t)pr.x * n] = cs.x * a + cs.y * b;
                Qp[i + (int64_t)pr.y * n] = -cs.y * a + cs.x * b;
            }
    for (int t = f0; t < k; t += st) {
        Q.dk[t] = Q.Ds[Q.sec[t]];
        Q.zk[t] = Q.zs[Q.sec[t]];
    }
    sp.sync();
    // (f) secular roots
    for (int i = f0; i < k; i += st) Q.tau[i] = dc_secular(k, Q.dk, Q.zk, rho, i, &Q.org[i]);
    sp.sync();
    // (g) recomputed z
    for (int j = f0; j < k; j += st) {
        const double dj = Q.dk[j];
        double w = (Q.dk[Q.org[j]] - dj) + Q.tau[j];
        for (int i = 0; i < k; ++i) {
            if (i == j) continue;
            w *= ((Q.dk[Q.org[i]] - dj) + Q.tau[i]) / (Q.dk[i] - dj);
        }
        Q.zh[j] = copysign(sqrt(fmax(w / rho, 0.0)), Q.zk[j]);
    }
    sp.sync();
    // (h) eigenvectors of the rank-one problem (columns of V, k x k) and the new eigenvalues
    for (int i = f0; i < k; i += st) {
        const double dorg = Q.dk[Q.org[i]], ti = Q.tau[i];
        double nrm = 0.0;
        for (int j = 0; j < k; ++j) {
            const double v = Q.zh[j] / ((Q.dk[j] - dorg) - ti);
            nrm = fma(v, v, nrm);
        }
        const double scl = 1.0 / sqrt(nrm);
        for (int j = 0; j < k; ++j) V[j + (int64_t)i * k] = scl * (Q.zh[j] / ((Q.dk[j] - dorg) - ti));
        Q.val[i] = dorg + ti;
    }
    for (int q2 = f0; q2 < nd; q2 += st) Q.val[k + q2] = Q.Ds[Q.dl[q2]];
    sp.sync();
    // (i) positions of the n new eigenvalues in ascending order
    for (int a = f0; a < n; a += st) {
        const double x = Q.val[a];
        int r = 0;
        for (int b2 = 0; b2 < n; ++b2) r += (Q.val[b2] < x || (Q.val[b2] == x && b2 < a)) ? 1 : 0;
        Q.rank[a] = lo + r;
    }
    for (int t = f0; t < ntop; t += st) Q.perm[t] = Q.sec[Q.ktop[t]];
    sp.sync();
    // (j) Z block = Q [V | deflated columns], block-1 rows against the columns touching block 1
    {
        const int ntr = (n1 + TS - 1) / TS, ntc = (k + TS - 1) / TS;
        for (int tt = sp.part; tt < ntr * ntc; tt += sp.nparts) {
            const int r0 = (tt % ntr) * TS, c0 = (tt / ntr) * TS;
            tile_gemm<false>(Z, m, lo, Q.rank, r0, c0, min(TS, n1 - r0), min(TS, k - c0), Qp, n, Q.perm, V, k, Q.ktop,
                             ntop, sA, sB);
        }
    }
    sp.sync();
    for (int t = f0; t < nbot; t += st) Q.perm[t] = Q.sec[Q.kbot[t]];
    sp.sync();
    {
        const int ntr = (n2 + TS - 1) / TS, ntc = (k + TS - 1) / TS;
        for (int tt = sp.part; tt < ntr * ntc; tt += sp.nparts) {
            const int r0 = n1 + (tt % ntr) * TS, c0 = (tt / ntr) * TS;
            tile_gemm<false>(Z, m, lo, Q.rank, r0, c0, min(TS, n - r0), min(TS, k - c0), Qp, n, Q.perm, V, k, Q.kbot,
                             nbot, sA, sB);
        }
    }
    for (int64_t t = f0; t < (int64_t)nd * n; t += st) {
        const int i = (int)(t % n), q2 = (int)(t / n);
        Z[(int64_t)(lo + i) + (int64_t)Q.rank[k + q2] * m] = Qp[i + (int64_t)Q.dl[q2] * n];
    }
    for (int a = f0; a < n; a += st) S.D[Q.rank[a]] = Q.val[a];
    sp.sync();
}

__device__ bool lg_dc(const Grp& g, const EigProb& p, const double* __restrict__ Da, const double* __restrict__ Ea,
                      double* __restrict__ Wa, double* __restrict__ Za, double* __restrict__ Qa,
                      double* __restrict__ Va, double* __restrict__ X, const LgSmem& sh) {
    const int m = p.m;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const LgLayout lay = lg_layout(m, g.size);
    const DcSmem S = dc_smem(reinterpret_cast<unsigned char*>(X + lay.dc), (m + 1) & ~1);
    int* scal = reinterpret_cast<int*>(X + lay.scal);
    double* Z = Za + p.aoff;
    const double* eo = Ea + p.voff;
    int L = 0;
    while (((m + (1 << L) - 1) >> L) > kDcLeaf) ++L;
    const int nleaf = 1 << L;
    for (int i = g.rank * kT + tid; i < m; i += g.size * kT) S.D[i] = Da[p.voff + i];
    if (g.rank == 0 && tid == 0) scal[7] = 0;
    g.sync();
    if (g.rank == 0 && tid == 0)
        for (int q = 1; q < nleaf; ++q) {
            const int pos = (int)(((int64_t)q * m) >> L);
            const double ab = fabs(eo[pos - 1]);
            S.D[pos - 1] -= ab;
            S.D[pos] -= ab;
        }
    g.sync();
    // leaves: a warp each over the whole cluster, numbered warp-major so that
    // few leaves still spread over every SM
    for (int q = warp * g.size + g.rank; q < nleaf; q += g.size * (kT / 32)) {
        const int lo = (int)(((int64_t)q * m) >> L), hi = (int)(((int64_t)(q + 1) * m) >> L), s = hi - lo;
        double dl[kDcLeaf], el[kDcLeaf], zl[kDcLeaf];
        for (int i = 0; i < kDcLeaf; ++i) {
            dl[i] = (i < s) ? S.D[lo + i] : 0.0;
            el[i] = (i < s - 1) ? eo[lo + i] : 0.0;
        }
        const bool ok = dc_leaf(s, dl, el, zl, lane);
        if (!ok && lane == 0) atomicExch(&scal[7], 1);
        int rk = 0;
        if (lane < s) {
            const double x = dl[lane];
            for (int c = 0; c < s; ++c) rk += (dl[c] < x || (dl[c] == x && c < lane)) ? 1 : 0;
        }
        for (int c = 0; c < s; ++c) {
            const int rc = __shfl_sync(0xffffffffu, rk, c);
            if (lane < s) Z[(int64_t)(lo + lane) + (int64_t)(lo + rc) * m] = zl[c];
        }
        __syncwarp();
        if (lane < s) S.D[lo + rk] = dl[lane];
        __syncwarp();
    }
    g.sync();
    if (((volatile int*)scal)[7] != 0) return false;
    for (int lev = L - 1; lev >= 0; --lev) {
        const int nm = 1 << lev;
        if (nm >= g.size) {
            for (int q = g.rank; q < nm; q += g.size) {
                const int lo = (int)(((int64_t)q * m) >> lev), hi = (int)(((int64_t)(q + 1) * m) >> lev);
                const int mid = (int)(((int64_t)(2 * q + 1) * m) >> (lev + 1));
                dc_merge(Split{0, 1, false, &g}, m, lo, mid, hi, eo[mid - 1], S, Z, Qa + p.aoff + (int64_t)lo * m,
                         Va + p.aoff + (int64_t)lo * m, scal + 8 + 8 * q, sh.sA, sh.sB);
            }
        } else {
            for (int q = 0; q < nm; ++q) {
                const int lo = (int)(((int64_t)q * m) >> lev), hi = (int)(((int64_t)(q + 1) * m) >> lev);
                const int mid = (int)(((int64_t)(2 * q + 1) * m) >> (lev + 1));
                dc_merge(Split{g.rank, g.size, true, &g}, m, lo, mid, hi, eo[mid - 1], S, Z,
                         Qa + p.aoff + (int64_t)lo * m, Va + p.aoff + (int64_t)lo * m, scal + 8 + 8 * q, sh.sA, sh.sB);
            }
        }
        g.sync();
    }
    for (int i = g.rank * kT + tid; i < m; i += g.size * kT) Wa[p.voff + i] = S.D[i];
    return true;
}

// Owned rows of S U and U, fe and the eigenpairs on the cluster: CTA rk takes a
// contiguous range of the 2 nown vectors (L rows, then L^-T rows by forward
// substitution), applies Q^T to them, and the product with Z is tiled over
// the cluster.
// Per-CTA scratch of the tile-product reflectors in the Q arena (free after the
// divide and conquer): Y and T Y, NB x nv each.
__host__ __device__ inline int64_t lg_wy_stride(int nv) { return 2 * (int64_t)NB * nv; }

__device__ void lg_rows(const Grp& g, const EigProb& p, const double* __restrict__ Ca,
                        const double* __restrict__ La, const double* __restrict__ Ta, const double* __restrict__ Wa,
                        const double* __restrict__ Za, const int* __restrict__ own_cols, const int* __restrict__ ipos,
                        double* __restrict__ Ba, double* __restrict__ Qa, const double* __restrict__ Ka,
                        double* __restrict__ e_out, double* __restrict__ fe_out, const LgSmem& sh) {
    const int m = p.m, no = p.nown, nb2 = 2 * no;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* Z = Za + p.aoff;
    const double* tau = Ta + p.voff;
    double* R = Ba + p.boff;
    double* G2 = R + (int64_t)nb2 * m;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kT / 32;
    const int per = (nb2 + g.size - 1) / g.size;
    const int u0 = min(nb2, g.rank * per), u1 = min(nb2, u0 + per);
    for (int u = u0; u < u1; ++u) {
        const int t = u < no ? u : u - no;
        const int ct = ipos[own_cols[p.o0 + t]];
        double* x = R + (int64_t)u * m;
        for (int r = tid; r < m; r += kT)
            x[r] = (u < no) ? ((r <= ct) ? L[ct + (int64_t)r * m] : 0.0) : ((r == ct) ? 1.0 : 0.0);
    }
    __syncthreads();
    const int s0 = max(u0, no);
    if (s0 < u1) trsm_cols(true, L, m, R + (int64_t)s0 * m, m, 0, u1 - s0, sh.sD, sh.sA, sh.sB);
    if (u1 > u0) {
        double* scr = Qa + p.aoff + (int64_t)g.rank * lg_wy_stride(per);
        wy_apply_t(C, m, Ka + p.koff, R + (int64_t)u0 * m, u1 - u0, true, scr, scr + (int64_t)NB * per, sh.sA,
                   sh.sB);
    }
    g.sync();
    {
        const int ntr = (m + TS - 1) / TS, ntc = (nb2 + TS - 1) / TS;
        for (int tt = g.rank; tt < ntr * ntc; tt += g.size) {
            const int r0 = (tt % ntr) * TS, c0 = (tt / ntr) * TS;
            tile_gemm<true>(G2, m, 0, nullptr, r0, c0, min(TS, m - r0), min(TS, nb2 - c0), Z, m, nullptr, R, m,
                            nullptr, m, sh.sA, sh.sB);
        }
    }
    g.sync();
    const double* G3 = G2 + (int64_t)no * m;
    for (int j = g.rank * kT + tid; j < m; j += g.size * kT) {
        double f = 0.0;
        for (int t = 0; t < no; ++t) f = fma(G2[(int64_t)t * m + j], G3[(int64_t)t * m + j], f);
        e_out[p.eoff + j] = Wa[p.voff + j];
        fe_out[p.eoff + j] = f;
    }
}

// Every stage of one problem on a group of CTAs.  mode 0: the submatrix
// method's eigenvalues, fe weights and owned rows of U (lg_rows); mode 1: all
// eigenvectors U = L^-T Q Z into Uout (m x m, column-major; L = I for the
// standard problem) and the eigenvalues into wout (ascending).
__device__ void eig_group_solve(const Grp& g, int pi, const EigProb& p, const LgSmem& sh, int mode,
                                const int* __restrict__ maps, const double* __restrict__ H,
                                const double* __restrict__ S, double* __restrict__ Ca, double* __restrict__ La,
                                double* __restrict__ Za, double* __restrict__ Qa, double* __restrict__ Va,
                                double* __restrict__ Da, double* __restrict__ Ea, double* __restrict__ Ta,
                                double* __restrict__ Wa, double* __restrict__ Ba, double* __restrict__ Ka,
                                double* __restrict__ Xa, const int* __restrict__ own_cols, const int* __restrict__ ipos,
                                double* __restrict__ e_out, double* __restrict__ fe_out, double* __restrict__ Uout,
                                double* __restrict__ wout, int* __restrict__ status,
                                unsigned long long* __restrict__ tstage) {
    double* X = Xa + p.xoff;
    const int m = p.m;
    // stage boundaries (global timer, ns) for the print-level-2 stage summary
    auto mark = [&](int q) {
        if (tstage && g.rank == 0 && threadIdx.x == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            tstage[(int64_t)pi * kLgStride + q] = t;
        }
    };
    mark(0);
    lg_gather(g, p, maps, H, S, Ca, La);
    g.sync();
    int st = kStOk;
    if (p.kind == 0) st = lg_potrf(g, m, La + p.aoff, sh);
    g.sync();
    mark(1);
    if (st == kStOk) {
        if (p.kind == 0) lg_reduce(g, p, La, Ca, sh);
        mark(2);
        lg_sytrd(g, p, Ca, Da, Ea, Ta, X, sh, tstage ? tstage + (int64_t)pi * kLgStride + kLgStages : nullptr);
        g.sync();
        mark(3);
        if (!lg_dc(g, p, Da, Ea, Wa, Za, Qa, Va, X, sh)) st = kStNoConv;
        g.sync();
        mark(4);
        if (st == kStOk) {
            build_T(Ca + p.aoff, m, Ta + p.voff, Ka + p.koff, g.rank, g.size, Va + p.aoff + (int64_t)g.rank * NB * NB,
                    sh.sD, sh.sA, sh.sB);
            g.sync();
            if (mode == 0 && p.mode == 2) {
                // density: U_occ = L^-T Q Z_occ in place of Z's occupied (lowest)
                // columns (column ranges per CTA), then the upper tiles of
                // U_occ U_occ^T split over the group
                const int no = p.nocc;
                const int per = (no + g.size - 1) / g.size;
                const int t0 = min(no, g.rank * per), t1 = min(no, t0 + per);
                double* Uz = Za + p.aoff;
                if (t1 > t0) {
                    double* scr = Qa + p.aoff + (int64_t)g.rank * lg_wy_stride(per);
                    wy_apply_t(Ca + p.aoff, m, Ka + p.koff, Uz + (int64_t)t0 * m, t1 - t0, false, scr,
                               scr + (int64_t)NB * per, sh.sA, sh.sB);
                    __syncthreads();
                    if (p.kind == 0)
                        trsm_cols(false, La + p.aoff, m, Uz + (int64_t)t0 * m, m, 0, t1 - t0, sh.sD, sh.sA, sh.sB);
                }
                for (int j = g.rank * kT + threadIdx.x; j < m; j += g.size * kT) e_out[p.eoff + j] = Wa[p.voff + j];
                g.sync();
                const int nt = (m + TS - 1) / TS;
                const int ntile = nt * (nt + 1) / 2;
                double* P = Ba + p.boff;
                for (int idx = g.rank; idx < ntile; idx += g.size) {
                    int cb, rb;
                    tri_decode(idx, cb, rb);   // cb >= rb: upper tiles
                    tile_mma<false, true, MMA_SET, false>(P, m, 0, nullptr, rb * TS, cb * TS, min(TS, m - rb * TS),
                                                          min(TS, m - cb * TS), Uz, m, nullptr, Uz, m, nullptr, p.nocc,
                                                          sh.sA, sh.sB);
                }
            } else if (mode == 0) {
                lg_rows(g, p, Ca, La, Ta, Wa, Za, own_cols, ipos, Ba, Qa, Ka, e_out, fe_out, sh);
            } else {
                const int per = (m + g.size - 1) / g.size;
                const int t0 = min(m, g.rank * per), t1 = min(m, t0 + per);
                for (int64_t q = (int64_t)t0 * m + threadIdx.x; q < (int64_t)t1 * m; q += kT) Uout[q] = Za[p.aoff + q];
                __syncthreads();
                if (t1 > t0) {
                    double* scr = Qa + p.aoff + (int64_t)g.rank * lg_wy_stride(per);
                    wy_apply_t(Ca + p.aoff, m, Ka + p.koff, Uout + (int64_t)t0 * m, t1 - t0, false, scr,
                               scr + (int64_t)NB * per, sh.sA, sh.sB);
                    __syncthreads();
                    if (p.kind == 0)
                        trsm_cols(false, La + p.aoff, m, Uout + (int64_t)t0 * m, m, 0, t1 - t0, sh.sD, sh.sA, sh.sB);
                }
                for (int j = g.rank * kT + threadIdx.x; j < m; j += g.size * kT) wout[j] = Wa[p.voff + j];
            }
        }
    }
    mark(5);
    if (g.rank == 0 && threadIdx.x == 0) status[pi] = st;
}

// One cluster per submatrix above kEigBatchMax (order[] largest first).
__global__ void __launch_bounds__(kT, 1) k_eig_cluster(
    const EigProb* __restrict__ probs, const int* __restrict__ order, int M, const int* __restrict__ maps,
    const double* __restrict__ H, const double* __restrict__ S, double* __restrict__ Ca, double* __restrict__ La,
    double* __restrict__ Za, double* __restrict__ Qa, double* __restrict__ Va, double* __restrict__ Da,
    double* __restrict__ Ea, double* __restrict__ Ta, double* __restrict__ Wa, double* __restrict__ Ba,
    double* __restrict__ Ka, double* __restrict__ Xa, const int* __restrict__ own_cols, const int* __restrict__ ipos,
    double* __restrict__ e_out, double* __restrict__ fe_out, int* __restrict__ status,
    unsigned long long* __restrict__ tstage, int mode, double* __restrict__ Uout, double* __restrict__ wout) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const LgSmem sh = lg_smem(smraw, M);
    cg::cluster_group cl = cg::this_cluster();
    const Grp g{(int)cl.block_rank(), (int)cl.num_blocks(), nullptr, nullptr};
    const int pi = order[blockIdx.x / g.size];
    const EigProb p = probs[pi];
    eig_group_solve(g, pi, p, sh, mode, maps, H, S, Ca, La, Za, Qa, Va, Da, Ea, Ta, Wa, Ba, Ka, Xa, own_cols, ipos,
                    e_out, fe_out, Uout, wout, status, tstage);
}

// One problem on the whole grid of a cooperative launch (software barrier).
__global__ void __launch_bounds__(kT, 1) k_eig_grid(
    const EigProb* __restrict__ probs, int pi, int M, int mode, const int* __restrict__ maps,
    const double* __restrict__ H, const double* __restrict__ S, double* __restrict__ Ca, double* __restrict__ La,
    double* __restrict__ Za, double* __restrict__ Qa, double* __restrict__ Va, double* __restrict__ Da,
    double* __restrict__ Ea, double* __restrict__ Ta, double* __restrict__ Wa, double* __restrict__ Ba,
    double* __restrict__ Ka, double* __restrict__ Xa, const int* __restrict__ own_cols, const int* __restrict__ ipos,
    double* __restrict__ e_out, double* __restrict__ fe_out, double* __restrict__ Uout, double* __restrict__ wout,
    int* __restrict__ status, unsigned* __restrict__ bar, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const LgSmem sh = lg_smem(smraw, M);
    const Grp g{(int)blockIdx.x, (int)gridDim.x, bar, err};
    const EigProb p = probs[pi];
    eig_group_solve(g, pi, p, sh, mode, maps, H, S, Ca, La, Za, Qa, Va, Da, Ea, Ta, Wa, Ba, Ka, Xa, own_cols, ipos,
                    e_out, fe_out, Uout, wout, status, nullptr);
}

// Owned columns of P_k at mu on the cluster (the large-submatrix form of
// k_eig_final): W0 = occ o U[c,:], W = Z W0 tiled over the cluster, then each
// CTA takes a contiguous range of the columns for Q w, L^-T w and the scatter.
__global__ void __launch_bounds__(kT, 1) k_eig_final_cluster(
    const EigProb* __restrict__ probs, const int* __restrict__ order, const double* __restrict__ Ca,
    const double* __restrict__ La, const double* __restrict__ Ta, const double* __restrict__ Wa,
    const double* __restrict__ Za, double* __restrict__ Qa, const double* __restrict__ Ka,
    const int* __restrict__ maps, const int* __restrict__ own_cols, double* __restrict__ Ba, double mu,
    double* __restrict__ Ppk, double* __restrict__ Pdense) {
    extern __shared__ __align__(16) unsigned char smf[];
    double* sA = reinterpret_cast<double*>(smf);
    double* sB = sA + kStageOp;
    double* sD = sB + kStageOp;
    double* sT = sD + TS * (TS + 1);
    cg::cluster_group cl = cg::this_cluster();
    const Grp g{(int)cl.block_rank(), (int)cl.num_blocks(), nullptr, nullptr};
    const EigProb p = probs[order[blockIdx.x / g.size]];
    const int m = p.m, no = p.nown;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* Z = Za + p.aoff;
    const double* tau = Ta + p.voff;
    const double* ev = Wa + p.voff;
    double* W0 = Ba + p.boff;
    const double* U2 = Ba + p.boff + 3 * (int64_t)no * m;
    double* W = Ba + p.boff + (int64_t)no * m;
    const int tid = threadIdx.x;
    for (int64_t q = (int64_t)g.rank * kT + tid; q < (int64_t)no * m; q += (int64_t)g.size * kT) {
        const int j = (int)(q % m);
        const double e = ev[j];
        const double occ = e < mu ? 2.0 : (e == mu ? 1.0 : 0.0);
        W0[q] = occ * U2[q];
    }
    g.sync();
    {
        const int ntr = (m + TS - 1) / TS, ntc = (no + TS - 1) / TS;
        for (int tt = g.rank; tt < ntr * ntc; tt += g.size) {
            const int r0 = (tt % ntr) * TS, c0 = (tt / ntr) * TS;
            tile_gemm<false>(W, m, 0, nullptr, r0, c0, min(TS, m - r0), min(TS, no - c0), Z, m, nullptr, W0, m,
                             nullptr, m, sA, sB);
        }
    }
    g.sync();
    const int per = (no + g.size - 1) / g.size;
    const int t0 = min(no, g.rank * per), t1 = min(no, t0 + per);
    if (t1 > t0) {
        double* scr = Qa + p.aoff + (int64_t)g.rank * lg_wy_stride(per);
        wy_apply_t(C, m, Ka + p.koff, W + (int64_t)t0 * m, t1 - t0, false, scr, scr + (int64_t)NB * per, sA, sB);
        __syncthreads();
        trsm_cols(false, L, m, W + (int64_t)t0 * m, m, 0, t1 - t0, sD, sA, sB);
    }
    if (Pdense) {
        for (int64_t q = (int64_t)t0 * m + tid; q < (int64_t)t1 * m; q += kT) Pdense[p.poff + q] = W[q];
        return;
    }
    const int* mp = maps + p.moff;
    for (int64_t q = (int64_t)t0 * m + tid; q < (int64_t)t1 * m; q += kT) {
        const int t = (int)(q / m), i = (int)(q % m);
        const int64_t cgl = own_cols[p.o0 + t];
        const int64_t gi = mp[i];
        if (gi <= cgl) Ppk[cgl * (cgl + 1) / 2 + gi] = W[q];
    }
}

}  // namespace

struct EigBatch {
    int nprob = 0;
    int maxm = 0;
    int G = 1;                    // CTAs per cluster of the large-submatrix solver
    int nsmall = 0, nlarge = 0;
    std::vector<EigProb> hp;
    DevBuf probs, order, order_l, counter, Ca, La, Za, Qa, Va, Da, Ea, Ta, Wa, Ba, Xa, Ka, status, tstage;
    int prl = 0;
    const char* what = "submatrix";   // the problems' name in error messages
    cudaStream_t side = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~EigBatch() {
        if (side) cudaStreamSynchronize(side);
        for (DevBuf* b : {&probs, &order, &order_l, &counter, &Ca, &La, &Za, &Qa, &Va, &Da, &Ea, &Ta, &Wa, &Ba, &Xa,
                          &Ka, &status, &tstage})
            b->release();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (side) cudaStreamDestroy(side);
    }
};

namespace {

void eig_setup_attrs() {
    static const bool done = [] {
        PTB_CUDA(cudaFuncSetAttribute(k_eig_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)stage_smem_bytes(kEigBatchMax)));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)lg_smem_bytes(kLargeMax)));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_final_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_final_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFinalSmem));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_grid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)lg_smem_bytes(kLargeMax)));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_final, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFinalSmem));
        return true;
    }();
    (void)done;
}

// Clusters of G CTAs of the cluster solver that fit on the device at once.
int eig_active_clusters(int G) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = G;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(G * 64);
    cfg.blockDim = dim3(kT);
    cfg.dynamicSmemBytes = lg_smem_bytes(kLargeMax);
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, (void*)k_eig_cluster, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return ncl;
}

// CTAs per cluster of the large-submatrix solver for one problem or a few
// waves of them: 16 when clusters of 16 keep at least 80 % of the SMs busy (one
// 512-thread CTA each), else 8 on the same rule, else the size among 4 and 2
// that keeps the most SMs busy; a submatrix's stages shorten with the cluster,
// and the longest submatrix sets the step.  PTBGPU_EIG_CLUSTER = 1, 2, 4, 8 or
// 16 overrides it.
int eig_cluster_size(ptbgpu_ctx* c) {
    static int cached[64] = {};
    const int dev = c->device & 63;
    if (cached[dev]) return cached[dev];
    int best = 1, best_ctas = 0;
    if (const char* e = getenv("PTBGPU_EIG_CLUSTER")) {
        const int v = atoi(e);
        if (v == 1 || v == 2 || v == 4 || v == 8 || v == 16) best = v;
    } else {
        const int nsm = c->num_sms > 0 ? c->num_sms : 148;
        for (int G : {16, 8, 4, 2}) {
            const int ncl = eig_active_clusters(G);
            if (ncl == 0) continue;
            if (G >= 8 && ncl * G * 5 >= nsm * 4) {
                best = G;
                break;
            }
            if (ncl * G > best_ctas) {
                best_ctas = ncl * G;
                best = G;
            }
        }
    }
    cached[dev] = best;
    return best;
}

// Cluster size for a batch with nlarge problems above kEigBatchMax.  When they
// need kManyWaves or more waves of the one-problem size, clusters of 2 CTAs
// take them: four times as many run side by side, each with a quarter of the
// cross-CTA steps per flop, and the last wave is shorter.  Measured on 174
// systems of order 1025-3064: 2.7-3.0 s per batch against 3.2-3.6 s with
// clusters of 8; on 50 submatrices up to 2773 clusters of 8 stay faster
// (0.64-0.71 s against 1.38 s with 2).
constexpr int kManyWaves = 6;
int eig_batch_cluster_size(ptbgpu_ctx* c, int nlarge) {
    const int G = eig_cluster_size(c);
    if (getenv("PTBGPU_EIG_CLUSTER") || G <= 2) return G;
    static int active[64] = {}, active2[64] = {};
    const int dev = c->device & 63;
    if (!active[dev]) {
        active2[dev] = eig_active_clusters(2);
        active[dev] = std::max(1, eig_active_clusters(G));
    }
    return nlarge >= kManyWaves * active[dev] && active2[dev] > 0 ? 2 : G;
}

template <class K, class... Args>
void launch_clustered(K kern, int nclusters, int G, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = G;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(nclusters * G);
    cfg.blockDim = dim3(kT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    PTB_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
}

}  // namespace

std::shared_ptr<EigBatch> eig_batch_launch(ptbgpu_ctx* c, int64_t n, const double* H, const double* S,
                                           const std::vector<EigProbHost>& probs, const int* d_maps,
                                            const int* d_own_cols, const int* d_ipos, double* d_e, double* d_fe,
                                            int prl, double* flops, bool join) {
    if (probs.empty()) return nullptr;
    eig_setup_attrs();
    cudaStream_t s = c->stream;
    auto eb = std::make_shared<EigBatch>();
    eb->nprob = (int)probs.size();
    eb->prl = prl;
    int nlarge = 0;
    for (const EigProbHost& q : probs) nlarge += q.m > kEigBatchMax ? 1 : 0;
    eb->G = nlarge > 0 ? eig_batch_cluster_size(c, nlarge) : 1;
    int64_t asz = 0, vsz = 0, bsz = 0, psz = 0, xsz = 0, ksz = 0;
    std::vector<int> ord_s, ord_l;
    for (const EigProbHost& q : probs) {
        PTB_CHECK(q.m >= 1 && q.m <= kLargeMax, PTBGPU_EINVAL, "submatrix %d of order %d outside the eigensolver (1..%d)",
                  q.k + 1, q.m, kLargeMax);
        EigProb p{};
        p.k = q.k;
        p.m = q.m;
        p.nown = q.nown;
        p.moff = q.moff;
        p.eoff = q.eoff;
        p.o0 = q.o0;
        p.gbase = q.gbase;
        p.gld = q.gld < 0 ? n : q.gld;
        p.mode = q.mode;
        p.nocc = q.nocc;
        p.poff = psz;
        psz += (int64_t)q.m * q.nown;
        p.aoff = asz;
        p.voff = vsz;
        p.boff = bsz;
        p.xoff = xsz;
        p.koff = ksz;
        ksz += t_panels(q.m) * NB * NB;
        asz += (int64_t)q.m * q.m;
        vsz += q.m;
        bsz += q.mode == 2 ? (int64_t)q.m * q.m : 4 * (int64_t)q.nown * q.m;
        if (q.m > kEigBatchMax) {
            xsz += lg_layout(q.m, eb->G).total;
            ord_l.push_back((int)eb->hp.size());
        } else {
            ord_s.push_back((int)eb->hp.size());
        }
        eb->maxm = std::max(eb->maxm, q.m);
        eb->hp.push_back(p);
        if (flops) *flops += 7.0 * std::pow((double)q.m, 3);
    }
    const int np = eb->nprob;
    eb->nsmall = (int)ord_s.size();
    eb->nlarge = (int)ord_l.size();
    eb->probs.reserve(sizeof(EigProb) * np);
    for (DevBuf* b : {&eb->Ca, &eb->La, &eb->Za, &eb->Qa, &eb->Va}) b->reserve(sizeof(double) * asz);
    for (DevBuf* b : {&eb->Da, &eb->Ea, &eb->Ta, &eb->Wa}) b->reserve(sizeof(double) * vsz);
    eb->Ba.reserve(sizeof(double) * std::max<int64_t>(bsz, 1));
    eb->Xa.reserve(sizeof(double) * std::max<int64_t>(xsz, 2));
    eb->Ka.reserve(sizeof(double) * std::max<int64_t>(ksz, 2));
    eb->status.reserve(sizeof(int) * np);
    PTB_CUDA(cudaMemcpyAsync(eb->probs.ptr, eb->hp.data(), sizeof(EigProb) * np, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(eb->status.ptr, 0, sizeof(int) * np, s));
    const EigProb* dp = eb->probs.as<EigProb>();
    int* dst = eb->status.as<int>();

    // largest first, so that the small submatrices fill in around the large ones
    auto by_size = [&](int a, int b) { return eb->hp[a].m > eb->hp[b].m; };
    std::stable_sort(ord_s.begin(), ord_s.end(), by_size);
    std::stable_sort(ord_l.begin(), ord_l.end(), by_size);
    eb->order.reserve(sizeof(int) * std::max<size_t>(ord_s.size(), 1));
    eb->order_l.reserve(sizeof(int) * std::max<size_t>(ord_l.size(), 1));
    eb->counter.reserve(sizeof(int));
    if (!ord_s.empty())
        PTB_CUDA(cudaMemcpyAsync(eb->order.ptr, ord_s.data(), sizeof(int) * ord_s.size(), cudaMemcpyHostToDevice, s));
    if (!ord_l.empty())
        PTB_CUDA(cudaMemcpyAsync(eb->order_l.ptr, ord_l.data(), sizeof(int) * ord_l.size(), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(eb->counter.ptr, 0, sizeof(int), s));
    // the large submatrices on their clusters (a side stream, launched first so
    // their clusters find free SMs), the small ones in the persistent launch
    if (eb->nlarge > 0) {
        PTB_CUDA(cudaStreamCreateWithFlags(&eb->side, cudaStreamNonBlocking));
        PTB_CUDA(cudaEventCreateWithFlags(&eb->ev0, cudaEventDisableTiming));
        PTB_CUDA(cudaEventCreateWithFlags(&eb->ev1, cudaEventDisableTiming));
        unsigned long long* dts = nullptr;
        if (prl >= 2) {
            eb->tstage.reserve(sizeof(unsigned long long) * kLgStride * np);
            PTB_CUDA(cudaMemsetAsync(eb->tstage.ptr, 0, sizeof(unsigned long long) * kLgStride * np, s));
            dts = eb->tstage.as<unsigned long long>();
        }
        PTB_CUDA(cudaEventRecord(eb->ev0, s));
        PTB_CUDA(cudaStreamWaitEvent(eb->side, eb->ev0, 0));
        launch_clustered(k_eig_cluster, eb->nlarge, eb->G, lg_smem_bytes(kLargeMax), eb->side, dp,
                         (const int*)eb->order_l.as<int>(), kLargeMax, d_maps, H, S, eb->Ca.as<double>(),
                         eb->La.as<double>(), eb->Za.as<double>(), eb->Qa.as<double>(), eb->Va.as<double>(),
                         eb->Da.as<double>(), eb->Ea.as<double>(), eb->Ta.as<double>(), eb->Wa.as<double>(),
                         eb->Ba.as<double>(), eb->Ka.as<double>(), eb->Xa.as<double>(), d_own_cols, d_ipos, d_e, d_fe,
                         dst, dts, 0, (double*)nullptr, (double*)nullptr);
        count_launch();
        PTB_CUDA(cudaEventRecord(eb->ev1, eb->side));
        log_line(prl, 2, " * submatrix cluster eigensolver: %d problems above order %d, clusters of %d CTAs",
                 eb->nlarge, kEigBatchMax, eb->G);
    }
    if (eb->nsmall > 0) {
        int Msmall = 0;
        for (int q : ord_s) Msmall = std::max(Msmall, eb->hp[q].m);
        const int Ms = (Msmall + 1) & ~1;   // staging sized for the largest small problem
        const int grid = std::min(eb->nsmall, c->num_sms > 0 ? c->num_sms : 148);
        k_eig_fused<<<grid, kT, stage_smem_bytes(Ms), s>>>(
            dp, eb->order.as<int>(), eb->nsmall, eb->counter.as<int>(), Ms, d_maps, H, S, eb->Ca.as<double>(),
            eb->La.as<double>(), eb->Za.as<double>(), eb->Qa.as<double>(), eb->Va.as<double>(), eb->Da.as<double>(),
            eb->Ea.as<double>(), eb->Ta.as<double>(), eb->Wa.as<double>(), eb->Ba.as<double>(), eb->Ka.as<double>(),
            d_own_cols, d_ipos, d_e, d_fe, dst);
        count_launch();
        PTB_CUDA(cudaGetLastError());
    }
    if (eb->nlarge > 0 && join) PTB_CUDA(cudaStreamWaitEvent(s, eb->ev1, 0));
    return eb;
}

void eig_batch_join(ptbgpu_ctx* c, EigBatch& eb) {
    if (eb.nlarge > 0 && eb.ev1) PTB_CUDA(cudaStreamWaitEvent(c->stream, eb.ev1, 0));
}

void eig_batch_check(ptbgpu_ctx* c, EigBatch& eb) {
    cudaStream_t s = c->stream;
    const int np = eb.nprob;
    std::vector<int> hst(np);
    PTB_CUDA(cudaMemcpyAsync(hst.data(), eb.status.ptr, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < np; ++q)
        PTB_CHECK(hst[q] <= 0, PTBGPU_ENOTSPD, "overlap of %s %d not positive definite (leading minor %d)", eb.what,
                  eb.hp[q].k + 1, hst[q]);
    for (int q = 0; q < np; ++q)
        PTB_CHECK(hst[q] == kStOk, PTBGPU_EITER, "tridiagonal eigensolver did not converge on %s %d", eb.what,
                  eb.hp[q].k + 1);
    if (eb.prl >= 2 && eb.nlarge > 0 && eb.tstage.ptr) {
        // per stage: summed over the large submatrices and the longest one, then
        // the span from the first cluster's start to the last one's end
        std::vector<unsigned long long> ts((size_t)kLgStride * np);
        PTB_CUDA(cudaMemcpy(ts.data(), eb.tstage.ptr, sizeof(unsigned long long) * ts.size(), cudaMemcpyDeviceToHost));
        static const char* names[kLgStages - 1] = {"gather + Cholesky", "reduction", "tridiagonalisation",
                                                   "divide and conquer", "owned rows"};
        double sum[kLgStages - 1] = {}, mx[kLgStages - 1] = {};
        unsigned long long t_lo = ~0ull, t_hi = 0;
        for (int q = 0; q < np; ++q) {
            if (eb.hp[q].m <= kEigBatchMax) continue;
            const unsigned long long* t = &ts[(size_t)q * kLgStride];
            t_lo = std::min(t_lo, t[0]);
            t_hi = std::max(t_hi, t[kLgStages - 1]);
            for (int k = 0; k + 1 < kLgStages; ++k) {
                const double d = (t[k + 1] >= t[k] && t[k] != 0) ? (double)(t[k + 1] - t[k]) * 1e-6 : 0.0;
                sum[k] += d;
                mx[k] = std::max(mx[k], d);
            }
        }
        for (int k = 0; k + 1 < kLgStages; ++k)
            log_line(eb.prl, 2, " * cluster eigensolver %-22s sum %10.3f ms, longest %9.3f ms", names[k], sum[k], mx[k]);
        static const char* sub[kLgSub] = {"column update", "barrier 1", "reflector", "A v tiles", "A v partials",
                                          "barrier 2", "panel end"};
        for (int k = 0; k < kLgSub; ++k) {
            double t = 0.0;
            for (int q = 0; q < np; ++q)
                if (eb.hp[q].m > kEigBatchMax) t += (double)ts[(size_t)q * kLgStride + kLgStages + k] * 1e-6;
            log_line(eb.prl, 2, " *   tridiagonalisation %-14s sum %10.3f ms", sub[k], t);
        }
        log_line(eb.prl, 2, " * cluster eigensolver span %10.3f ms (%d submatrices, clusters of %d)",
                 t_hi > t_lo ? (double)(t_hi - t_lo) * 1e-6 : 0.0, eb.nlarge, eb.G);
    }
}

void eig_batch_final(ptbgpu_ctx* c, EigBatch& eb, double mu, int64_t n, const int* d_maps, const int* d_own_cols,
                     double* dP, double* dPdense) {
    (void)n;
    if (eb.nprob == 0) return;
    cudaStream_t s = c->stream;
    if (eb.nsmall > 0) {
        eig_setup_attrs();
        k_eig_final<<<eb.nsmall, kT, kFinalSmem, s>>>(eb.probs.as<EigProb>(), eb.order.as<int>(), eb.Ca.as<double>(),
                                                      eb.La.as<double>(), eb.Ta.as<double>(), eb.Wa.as<double>(),
                                                      eb.Za.as<double>(), eb.Qa.as<double>(), eb.Va.as<double>(),
                                                      eb.Ka.as<double>(), d_maps, d_own_cols, eb.Ba.as<double>(), mu, dP,
                                                      dPdense);
        count_launch();
        PTB_CUDA(cudaGetLastError());
    }
    if (eb.nlarge > 0) {
        launch_clustered(k_eig_final_cluster, eb.nlarge, eb.G, kFinalSmem, s, (const EigProb*)eb.probs.as<EigProb>(),
                         (const int*)eb.order_l.as<int>(), (const double*)eb.Ca.as<double>(),
                         (const double*)eb.La.as<double>(), (const double*)eb.Ta.as<double>(),
                         (const double*)eb.Wa.as<double>(), (const double*)eb.Za.as<double>(), eb.Qa.as<double>(),
                         (const double*)eb.Ka.as<double>(), d_maps, d_own_cols, eb.Ba.as<double>(), mu, dP, dPdense);
        count_launch();
    }
}

// Matrix with both triangles set from the upper one: out[i + j n] = a[min(i,j) + max(i,j) n].
__global__ void k_sym_from_upper(int64_t n, const double* __restrict__ a, double* __restrict__ out) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q % n, j = q / n;
        out[q] = (i <= j) ? a[i + j * n] : a[j + i * n];
    }
}

constexpr int kGridRows = 64;   // rows per CTA of a cooperative-grid solve
constexpr int kGridMax = 64;    // CTAs of a cooperative-grid solve at most
constexpr int kGridMin = 4096;  // orders solved by one cluster instead

void eig_full(ptbgpu_ctx* c, int64_t n, const double* H, const double* S, double* w, double* U) {
    PTB_CHECK(n >= 1 && n <= kLargeMax, PTBGPU_EINVAL, "eigenproblem of order %lld outside the eigensolver (1..%d)",
              (long long)n, kLargeMax);
    eig_setup_attrs();
    cudaStream_t s = c->stream;
    const int m = (int)n;
    int per_sm = 0;
    PTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_eig_grid, kT, lg_smem_bytes(kLargeMax)));
    PTB_CHECK(per_sm >= 1, PTBGPU_ECUDA, "eigensolver kernel does not fit an SM");
    const int nsm = c->num_sms > 0 ? c->num_sms : 148;
    // up to order kGridMin one thread-block cluster (hardware barrier), above it
    // a cooperative grid of one CTA per kGridRows rows, at most kGridMax CTAs
    // (the software barrier's latency grows with the CTA count)
    const bool cluster = m <= kGridMin;
    int G = cluster ? eig_cluster_size(c) : std::min({nsm * per_sm, kGridMax, std::max(1, m / kGridRows)});
    EigBatch eb;
    eb.nprob = 1;
    eb.G = G;
    EigProb p{};
    p.m = m;
    p.kind = S ? 0 : 1;
    p.gld = n;
    eb.hp.push_back(p);
    const int64_t mm = (int64_t)m * m;
    const int per = (m + G - 1) / G;
    const LgLayout lay = lg_layout(m, G);
    for (DevBuf* b : {&eb.Ca, &eb.La, &eb.Za}) b->reserve(sizeof(double) * mm);
    eb.Qa.reserve(sizeof(double) * std::max<int64_t>(mm, (int64_t)G * lg_wy_stride(per) + 2));
    eb.Va.reserve(sizeof(double) * std::max<int64_t>(mm, (int64_t)G * NB * NB + 2));
    for (DevBuf* b : {&eb.Da, &eb.Ea, &eb.Ta, &eb.Wa}) b->reserve(sizeof(double) * n);
    eb.Ka.reserve(sizeof(double) * std::max<int64_t>(t_panels(m) * NB * NB, 2));
    eb.Xa.reserve(sizeof(double) * lay.total);
    eb.Ba.reserve(sizeof(double) * 2);
    eb.probs.reserve(sizeof(EigProb));
    eb.status.reserve(sizeof(int) * 4);
    eb.order.reserve(sizeof(int) * n);   // the identity row map
    std::vector<int> ident(n);
    for (int i = 0; i < m; ++i) ident[i] = i;
    PTB_CUDA(cudaMemcpyAsync(eb.order.ptr, ident.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(eb.probs.ptr, &p, sizeof(EigProb), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(eb.status.ptr, 0, sizeof(int) * 4, s));
    unsigned* bar = reinterpret_cast<unsigned*>(eb.status.as<int>() + 1);   // status, bar[0], bar[1], err
    int* err = eb.status.as<int>() + 3;
    const EigProb* dp = eb.probs.as<EigProb>();
    int pi = 0, M = kLargeMax, mode = 1;
    const int* maps = eb.order.as<int>();
    double *Ca = eb.Ca.as<double>(), *La = eb.La.as<double>(), *Za = eb.Za.as<double>(), *Qa = eb.Qa.as<double>(),
           *Va = eb.Va.as<double>(), *Da = eb.Da.as<double>(), *Ea = eb.Ea.as<double>(), *Ta = eb.Ta.as<double>(),
           *Wa = eb.Wa.as<double>(), *Ba = eb.Ba.as<double>(), *Ka = eb.Ka.as<double>(), *Xa = eb.Xa.as<double>();
    const int* own = nullptr;
    const int* ipos = nullptr;
    double *e_out = nullptr, *fe_out = nullptr;
    int* status = eb.status.as<int>();
    // PTBGPU_EIG_STAGES=1: stage and tridiagonalisation phase times on stderr
    static const bool stages = getenv("PTBGPU_EIG_STAGES") != nullptr;
    if (cluster) {
        const int* order = eb.order.as<int>() + 0;   // identity map: order[0] = 0
        unsigned long long* ts = nullptr;
        if (stages) {
            eb.tstage.reserve(sizeof(unsigned long long) * kLgStride);
            PTB_CUDA(cudaMemsetAsync(eb.tstage.ptr, 0, sizeof(unsigned long long) * kLgStride, s));
            ts = eb.tstage.as<unsigned long long>();
        }
        launch_clustered(k_eig_cluster, 1, G, lg_smem_bytes(kLargeMax), s, dp, order, M, maps, H, S, Ca, La, Za, Qa,
                         Va, Da, Ea, Ta, Wa, Ba, Ka, Xa, own, ipos, e_out, fe_out, status, ts, mode, U, w);
        if (stages) {
            unsigned long long t[kLgStride];
            PTB_CUDA(cudaMemcpyAsync(t, ts, sizeof(t), cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            fprintf(stderr, "eig_full n=%d cluster %d: stages", m, G);
            for (int k = 0; k + 1 < kLgStages; ++k) fprintf(stderr, " %.3f", (double)(t[k + 1] - t[k]) * 1e-6);
            fprintf(stderr, " ms; tridiag phases");
            for (int k = 0; k < kLgSub; ++k) fprintf(stderr, " %.3f", (double)t[kLgStages + k] * 1e-6);
            fprintf(stderr, " ms\n");
        }
    } else {
        void* args[] = {&dp, &pi, &M, &mode, &maps, &H, &S, &Ca, &La, &Za, &Qa, &Va, &Da, &Ea, &Ta, &Wa, &Ba, &Ka, &Xa,
                        &own, &ipos, &e_out, &fe_out, &U, &w, &status, &bar, &err};
        PTB_CUDA(cudaLaunchCooperativeKernel((void*)k_eig_grid, dim3(G), dim3(kT), args, lg_smem_bytes(kLargeMax), s));
    }
    count_launch();
    int hs[4];
    PTB_CUDA(cudaMemcpyAsync(hs, eb.status.ptr, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    PTB_CHECK(hs[3] == 0, PTBGPU_ETIMEOUT, "eigensolver: a grid barrier gave up waiting");
    PTB_CHECK(hs[0] <= 0, PTBGPU_ENOTSPD, "overlap matrix not positive definite (leading minor %d)", hs[0]);
    PTB_CHECK(hs[0] == kStOk, PTBGPU_EITER, "tridiagonal eigensolver did not converge");
}

void eig_full_upper(ptbgpu_ctx* c, int64_t n, double* A, double* B, double* w) {
    cudaStream_t s = c->stream;
    DevBuf h, b, u;
    struct Rel {
        DevBuf *x, *y, *z;
        ~Rel() {
            x->release();
            y->release();
            z->release();
        }
    } rel{&h, &b, &u};
    h.reserve(sizeof(double) * n * n);
    u.reserve(sizeof(double) * n * n);
    const int grid = (int)std::min<int64_t>((n * n + 255) / 256, 148 * 16);
    k_sym_from_upper<<<grid, 256, 0, s>>>(n, A, h.as<double>());
    count_launch();
    if (B) {
        b.reserve(sizeof(double) * n * n);
        k_sym_from_upper<<<grid, 256, 0, s>>>(n, B, b.as<double>());
        count_launch();
    }
    PTB_CUDA(cudaGetLastError());
    eig_full(c, n, h.as<double>(), B ? b.as<double>() : nullptr, w, u.as<double>());
    PTB_CUDA(cudaMemcpyAsync(A, u.ptr, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, s));
    PTB_CUDA(cudaStreamSynchronize(s));
}

// Packed upper triangle of scale * P (P m x m column-major, read above the diagonal).
__global__ void k_pack_scaled(int64_t m, const double* __restrict__ P, double scale, double* __restrict__ pk) {
    const int64_t np = m * (m + 1) / 2;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < np; q += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = (int64_t)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
        while ((j + 1) * (j + 2) / 2 <= q) ++j;
        while (j * (j + 1) / 2 > q) --j;
        const int64_t i = q - j * (j + 1) / 2;
        pk[q] = scale * P[i + j * m];
    }
}

void eig_density_batch(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                       const double* const* Hpk, const double* const* Spk, double* const* Ppk, double filter,
                       int prl, ptbgpu_stats* st) {
    if (ninst <= 0) return;
    cudaStream_t s = c->stream;
    // The systems above kEigBatchMax are copied in and launched on their
    // clusters first; the small ones are copied in while those run, then solved
    // by the persistent launch beside them, and their results copied out while
    // the clusters finish.
    std::vector<int64_t> large, small;
    std::vector<int64_t> pkoff((size_t)ninst + 1, 0);
    int64_t hsz = 0, nsum = 0;
    std::vector<EigProbHost> pr((size_t)ninst);
    for (int64_t k = 0; k < ninst; ++k) {
        const int64_t m = ndim[k];
        PTB_CHECK(m >= 1 && m <= kLargeMax, PTBGPU_EINVAL, "system %lld: ndim %lld outside the eigensolver (1..%d)",
                  (long long)k, (long long)m, kLargeMax);
        PTB_CHECK(nel[k] >= 0 && nel[k] / 2 <= m && Hpk[k] && Spk[k] && Ppk[k], PTBGPU_EINVAL,
                  "system %lld: bad electron count or arrays", (long long)k);
        PTB_CHECK(nel[k] % 2 == 0, PTBGPU_EINVAL,
                  "system %lld: odd electron count %lld (the T = 0 projector here is closed-shell)", (long long)k,
                  (long long)nel[k]);
        EigProbHost& q = pr[k];
        q.k = (int)k;
        q.m = (int)m;
        q.nown = 0;
        q.moff = nsum;
        q.eoff = nsum;
        q.o0 = 0;
        q.gbase = hsz;
        q.gld = m;
        q.mode = 2;
        q.nocc = (int)(nel[k] / 2);
        hsz += m * m;
        nsum += m;
        pkoff[k + 1] = pkoff[k] + m * (m + 1) / 2;
        (m > kEigBatchMax ? large : small).push_back(k);
    }
    struct Bufs {
        DevBuf h, sm, pk, maps, e, dummy;
        ~Bufs() {
            for (DevBuf* b : {&h, &sm, &pk, &maps, &e, &dummy}) b->release();
        }
    } b;
    b.h.reserve(sizeof(double) * hsz);
    b.sm.reserve(sizeof(double) * hsz);
    b.pk.reserve(sizeof(double) * std::max<int64_t>(2 * pkoff[ninst], 1));
    b.maps.reserve(sizeof(int) * nsum);
    b.e.reserve(sizeof(double) * nsum);
    b.dummy.reserve(64);
    std::vector<int> maps((size_t)nsum);
    for (const EigProbHost& q : pr)
        for (int i = 0; i < q.m; ++i) maps[q.moff + i] = i;
    PTB_CUDA(cudaMemcpyAsync(b.maps.ptr, maps.data(), sizeof(int) * nsum, cudaMemcpyHostToDevice, s));
    double* pkH = b.pk.as<double>();
    double* pkS = pkH + pkoff[ninst];
    auto upload = [&](const std::vector<int64_t>& ids) {
        for (int64_t k : ids) {
            const int64_t m = ndim[k], np = m * (m + 1) / 2;
            PTB_CUDA(cudaMemcpyAsync(pkH + pkoff[k], Hpk[k], sizeof(double) * np, cudaMemcpyHostToDevice, s));
            PTB_CUDA(cudaMemcpyAsync(pkS + pkoff[k], Spk[k], sizeof(double) * np, cudaMemcpyHostToDevice, s));
            unpack_sym(s, m, m, pkH + pkoff[k], b.h.as<double>() + pr[k].gbase, filter);
            unpack_sym(s, m, m, pkS + pkoff[k], b.sm.as<double>() + pr[k].gbase, filter);
        }
    };
    auto launch = [&](const std::vector<int64_t>& ids, bool join) {
        std::vector<EigProbHost> probs;
        for (int64_t k : ids) probs.push_back(pr[k]);
        double flops = 0.0;
        auto eb = eig_batch_launch(c, 0, b.h.as<double>(), b.sm.as<double>(), probs, b.maps.as<int>(),
                                   b.dummy.as<int>(), b.dummy.as<int>(), b.e.as<double>(), b.e.as<double>(), prl,
                                   &flops, join);
        eb->what = "system";
        return eb;
    };
    auto download = [&](EigBatch& eb, const std::vector<int64_t>& ids) {
        for (size_t q = 0; q < ids.size(); ++q) {
            const int64_t k = ids[q], m = ndim[k], np = m * (m + 1) / 2;
            const int grid = (int)std::min<int64_t>((np + 255) / 256, 148 * 8);
            k_pack_scaled<<<grid, 256, 0, s>>>(m, eb.Ba.as<double>() + eb.hp[q].boff, 2.0, pkH + pkoff[k]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            PTB_CUDA(cudaMemcpyAsync(Ppk[k], pkH + pkoff[k], sizeof(double) * np, cudaMemcpyDeviceToHost, s));
        }
    };
    std::shared_ptr<EigBatch> ebl, ebs;   // declared after b: released (side stream drained) before its buffers
    upload(large);
    if (!large.empty()) ebl = launch(large, false);
    upload(small);
    if (!small.empty()) {
        ebs = launch(small, true);
        eig_batch_check(c, *ebs);
        download(*ebs, small);
    }
    if (ebl) {
        eig_batch_join(c, *ebl);
        eig_batch_check(c, *ebl);
        download(*ebl, large);
    }
    PTB_CUDA(cudaStreamSynchronize(s));
    if (st)
        for (int64_t k = 0; k < ninst; ++k) st[k].flops += 7.0 * std::pow((double)ndim[k], 3);
}

// Kernel-level entry: dense host problems through the same stages.  Problem k's
// H and S sit at offset sum_{k'<k} m_k'^2 of the concatenated input (ld m_k);
// its owned columns are given by local index.
void sygv_batched_entry(ptbgpu_ctx* c, int64_t np, const int64_t* dims, const double* H, const double* S,
                        const int64_t* nown, const int64_t* owned, double mu, double* e, double* fe, double* Pcols) {
    struct Bufs {
        DevBuf h, s, maps, own, ipos, e, fe, p;
        ~Bufs() {
            for (DevBuf* b : {&h, &s, &maps, &own, &ipos, &e, &fe, &p}) b->release();
        }
    } b;
    cudaStream_t st = c->stream;
    std::vector<EigProbHost> probs;
    std::vector<int> maps, own, ipos;
    int64_t hsz = 0, nsum = 0, osum = 0, psz = 0;
    for (int64_t k = 0; k < np; ++k) {
        const int m = (int)dims[k];
        PTB_CHECK(dims[k] >= 1 && dims[k] <= kLargeMax && nown[k] >= 1 && nown[k] <= dims[k], PTBGPU_EINVAL,
                  "problem %lld: order %lld (1..%d) or owned count %lld out of range", (long long)k,
                  (long long)dims[k], kLargeMax, (long long)nown[k]);
        EigProbHost q{};
        q.k = (int)k;
        q.m = m;
        q.nown = (int)nown[k];
        q.moff = nsum;
        q.eoff = nsum;
        q.o0 = osum;
        q.gbase = hsz;
        q.gld = m;
        probs.push_back(q);
        for (int i = 0; i < m; ++i) {
            maps.push_back(i);
            ipos.push_back(i);
        }
        for (int64_t t = 0; t < nown[k]; ++t) {
            const int64_t li = owned[osum + t];
            PTB_CHECK(li >= 0 && li < m, PTBGPU_EINVAL, "problem %lld: owned index %lld out of range",
                      (long long)k, (long long)li);
            own.push_back((int)(nsum + li));
        }
        hsz += (int64_t)m * m;
        nsum += m;
        osum += nown[k];
        psz += (int64_t)m * nown[k];
    }
    b.h.reserve(sizeof(double) * hsz);
    b.s.reserve(sizeof(double) * hsz);
    b.maps.reserve(sizeof(int) * nsum);
    b.own.reserve(sizeof(int) * osum);
    b.ipos.reserve(sizeof(int) * nsum);
    b.e.reserve(sizeof(double) * nsum);
    b.fe.reserve(sizeof(double) * nsum);
    PTB_CUDA(cudaMemcpyAsync(b.h.ptr, H, sizeof(double) * hsz, cudaMemcpyHostToDevice, st));
    PTB_CUDA(cudaMemcpyAsync(b.s.ptr, S, sizeof(double) * hsz, cudaMemcpyHostToDevice, st));
    PTB_CUDA(cudaMemcpyAsync(b.maps.ptr, maps.data(), sizeof(int) * nsum, cudaMemcpyHostToDevice, st));
    PTB_CUDA(cudaMemcpyAsync(b.own.ptr, own.data(), sizeof(int) * osum, cudaMemcpyHostToDevice, st));
    PTB_CUDA(cudaMemcpyAsync(b.ipos.ptr, ipos.data(), sizeof(int) * nsum, cudaMemcpyHostToDevice, st));
    std::shared_ptr<EigBatch> eb =
        eig_batch_launch(c, 0, b.h.as<double>(), b.s.as<double>(), probs, b.maps.as<int>(), b.own.as<int>(),
                         b.ipos.as<int>(), b.e.as<double>(), b.fe.as<double>(), 0, nullptr);
    eig_batch_check(c, *eb);
    PTB_CUDA(cudaMemcpyAsync(e, b.e.ptr, sizeof(double) * nsum, cudaMemcpyDeviceToHost, st));
    PTB_CUDA(cudaMemcpyAsync(fe, b.fe.ptr, sizeof(double) * nsum, cudaMemcpyDeviceToHost, st));
    if (Pcols) {
        b.p.reserve(sizeof(double) * psz);
        eig_batch_final(c, *eb, mu, 0, b.maps.as<int>(), b.own.as<int>(), nullptr, b.p.as<double>());
        PTB_CUDA(cudaMemcpyAsync(Pcols, b.p.ptr, sizeof(double) * psz, cudaMemcpyDeviceToHost, st));
    }
    PTB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace ptb
