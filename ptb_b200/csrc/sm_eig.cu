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
#include <algorithm>
#include <cmath>
#include <vector>

#include "sm_eig.cuh"

namespace ptb {

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
    int k, m, nown, pad;
    int64_t moff, eoff, o0;
    int64_t gbase, gld;   // the problem's H / S: element (i, j) at gbase + map(i) + map(j) gld
    int64_t poff;         // dense output of the owned columns of P (m x nown, column-major)
    int64_t aoff;     // C, L, Z and merge-workspace arenas (m x m, column-major, ld = m)
    int64_t voff;     // d, e, tau, eigenvalue arenas (m)
    int64_t boff;     // owned-row arena (4 nown x m)
};

// ---------------------------------------------------------------------------
// C[r0+i, c0+j] -= sum_{k < kk} A(i,k) B(k,j) on one TS x TS tile (mr x nc
// valid), 512 threads with 4 x 2 outputs each.
//   A(i,k) = A[(r0+i) + k lda]
//   B(k,j) = BT ? B[(c0+j) + k ldb] : B[k + (c0+j) ldb]
// LOWER: only elements on or below the diagonal of C are written.
template <bool BT, bool LOWER>
__device__ void tile_update(double* __restrict__ C, int ldc, int r0, int c0, int mr, int nc,
                            const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb, int kk,
                            double* sA, double* sB) {
    const int tid = threadIdx.x;
    for (int t = tid; t < TS * NB; t += kT) {
        const int i = t % TS, k = t / TS;
        sA[k * (TS + 1) + i] = (i < mr && k < kk) ? A[(int64_t)(r0 + i) + (int64_t)k * lda] : 0.0;
    }
    if (BT) {
        for (int t = tid; t < TS * NB; t += kT) {
            const int j = t % TS, k = t / TS;
            sB[k * (TS + 1) + j] = (j < nc && k < kk) ? B[(int64_t)(c0 + j) + (int64_t)k * ldb] : 0.0;
        }
    } else {
        for (int t = tid; t < TS * NB; t += kT) {
            const int k = t % NB, j = t / NB;
            sB[k * (TS + 1) + j] = (j < nc && k < kk) ? B[(int64_t)k + (int64_t)(c0 + j) * ldb] : 0.0;
        }
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;   // 16 x 32 threads, 4 x 2 outputs each
    double acc[4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b] = 0.0;
    for (int k = 0; k < kk; ++k) {
        double av[4], bv[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = sA[k * (TS + 1) + tx + 16 * a];
#pragma unroll
        for (int b = 0; b < 2; ++b) bv[b] = sB[k * (TS + 1) + ty + 32 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    // read-modify-write of the C tile: all loads issued before any store (the
    // stores could alias later loads as far as the compiler knows, which would
    // otherwise serialise the round trips to memory)
    double cv[4][2];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        const int j = ty + 32 * b;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = tx + 16 * a;
            const bool ok = j < nc && i < mr && !(LOWER && r0 + i < c0 + j);
            cv[a][b] = ok ? C[(int64_t)(r0 + i) + (int64_t)(c0 + j) * ldc] : 0.0;
        }
    }
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        const int j = ty + 32 * b;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = tx + 16 * a;
            const bool ok = j < nc && i < mr && !(LOWER && r0 + i < c0 + j);
            if (ok) C[(int64_t)(r0 + i) + (int64_t)(c0 + j) * ldc] = cv[a][b] - acc[a][b];
        }
    }
    __syncthreads();
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
// C[ro(i), co(j)] = sum_k A(i, kx(k)) B(k, j) on one TS x TS output tile, the
// K range in NB chunks, 256 threads with 4 x 4 outputs each:
//   A(i, k) = AT ? A[k + (r0+i) lda] : A[(r0+i) + k lda]
//   B(k, j) = BT ? B[(c0+j) + kxb(k) ldb] : B[kxb(k) + (c0+j) ldb]
//   kx, kxb: optional K index maps (shared memory), crow: output row offset,
//   ccol: optional output column map (shared memory) else c0 + j.
template <bool AT, bool BT = false>
__device__ void tile_gemm(double* __restrict__ C, int64_t ldc, int crow, const int* ccol, int r0, int c0, int mr,
                          int nc, const double* __restrict__ A, int64_t lda, const int* kx,
                          const double* __restrict__ B, int64_t ldb, const int* kxb, int K, double* sA, double* sB) {
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;   // 16 x 32 threads, 4 x 2 outputs each
    double acc[4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b] = 0.0;
    // K chunks double-buffered through registers: the next chunk's loads are in
    // flight while the current one is multiplied out of shared memory
    constexpr int kPer = TS * NB / kT;   // staged elements of A (and of B) per thread
    double ra[kPer], rb[kPer];
    auto fetch = [&](int k0) {
        const int kk = min(NB, K - k0);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int t = tid + q * kT;
            int i, k;
            if (AT) {
                k = t % NB;
                i = t / NB;
            } else {
                i = t % TS;
                k = t / TS;
            }
            double v = 0.0;
            if (i < mr && k < kk) {
                const int64_t kg = kx ? kx[k0 + k] : (k0 + k);
                v = AT ? A[kg + (int64_t)(r0 + i) * lda] : A[(int64_t)(r0 + i) + kg * lda];
            }
            ra[q] = v;
            int j, kb;
            if (BT) {
                j = t % TS;
                kb = t / TS;
            } else {
                kb = t % NB;
                j = t / NB;
            }
            double w = 0.0;
            if (j < nc && kb < kk) {
                const int64_t kg = kxb ? kxb[k0 + kb] : (k0 + kb);
                w = BT ? B[(int64_t)(c0 + j) + kg * ldb] : B[kg + (int64_t)(c0 + j) * ldb];
            }
            rb[q] = w;
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int t = tid + q * kT;
            const int i = AT ? t / NB : t % TS, k = AT ? t % NB : t / TS;
            sA[k * (TS + 1) + i] = ra[q];
            const int j = BT ? t % TS : t / NB, kb = BT ? t / TS : t % NB;
            sB[kb * (TS + 1) + j] = rb[q];
        }
    };
    fetch(0);
    stash();
    __syncthreads();
    for (int k0 = 0; k0 < K; k0 += NB) {
        const int kk = min(NB, K - k0);
        const bool more = k0 + NB < K;
        if (more) fetch(k0 + NB);
        for (int k = 0; k < kk; ++k) {
            double av[4], bv[2];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = sA[k * (TS + 1) + tx + 16 * a];
#pragma unroll
            for (int b = 0; b < 2; ++b) bv[b] = sB[k * (TS + 1) + ty + 32 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
        __syncthreads();
        if (more) {
            stash();
            __syncthreads();
        }
    }
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        const int j = ty + 32 * b;
        if (j >= nc) continue;
        const int64_t col = ccol ? ccol[c0 + j] : (c0 + j);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = tx + 16 * a;
            if (i < mr) C[(int64_t)(crow + r0 + i) + col * ldc] = acc[a][b];
        }
    }
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
static_assert(NB * (NB + 1) <= NB * (TS + 1) && NB * kWyChunk <= NB * (TS + 1), "WY scratch fits the tile staging");

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
// Owned rows of S U and U, fe and the eigenpairs.  R holds 2 nown rows of
// length m (row-major, i.e. the column-major m x 2nown matrix R^T): rows
// t < nown are L[c_t,:] -> (S U)[c_t,:], rows nown + t are (L^-T)[c_t,:] ->
// U[c_t,:].  The final product with Z goes into the third block G (R Z).
__device__ void stage_rows(const EigProb& p, const double* __restrict__ Ca, const double* __restrict__ La,
                           const double* __restrict__ Ta, const double* __restrict__ Wa,
                           const double* __restrict__ Za, const int* __restrict__ own_cols,
                           const int* __restrict__ ipos, double* __restrict__ Ba, double* __restrict__ e_out,
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
    // rows of L^-T: x_t = L^-1 e_{c_t}, 32-row blocks
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
    // R <- R Q: each row x becomes Q^T x (the tiles' staging space as scratch)
    wy_apply(C, m, tau, R, nb2, true, WySmem{sA, sB});
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
// One persistent launch for every submatrix of the step: each CTA takes the
// next submatrix (largest first) from a device counter and runs all stages on
// it - gather, Cholesky, reduction, tridiagonalisation, divide and conquer,
// owned rows and fe - so the uneven sizes balance over the SMs without a
// launch per stage or per size bucket.  status[pi]: 0, the order of a
// non-positive pivot of S_k, or kStNoConv.
__host__ __device__ constexpr size_t stage_smem_bytes(int M) {
    return sizeof(double) * (2 * NB * (TS + 1) + NB * (NB + 1)) + dc_smem_bytes(M) + sizeof(int) * 16 +
           sizeof(double) * (2 + kT / 32) + 16;
}

__device__ StageSmem stage_smem(unsigned char* base, int M) {
    StageSmem sh;
    double* d = reinterpret_cast<double*>(base);
    sh.sA = d;
    sh.sB = d + NB * (TS + 1);
    sh.sD = d + 2 * NB * (TS + 1);
    sh.uni = reinterpret_cast<unsigned char*>(d + 2 * NB * (TS + 1) + NB * (NB + 1));
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
    double* __restrict__ Wa, double* __restrict__ Ba, const int* __restrict__ own_cols,
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
            if (st == kStOk) stage_rows(p, Ca, La, Ta, Wa, Za, own_cols, ipos, Ba, e_out, fe_out, sh);
        }
        if (tid == 0) status[pi] = st;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Owned columns of P_k at mu: w_t = occ o U[c_t,:]^T, w <- Z w, w <- Q w
// (reflectors in reverse), w <- L^-T w; scattered into the packed result,
// rows map(i) <= c_t of column c_t (or written dense).
__global__ void __launch_bounds__(kT) k_eig_final(const EigProb* __restrict__ probs, const double* __restrict__ Ca,
                                                  const double* __restrict__ La, const double* __restrict__ Ta,
                                                  const double* __restrict__ Wa, const double* __restrict__ Za,
                                                  const int* __restrict__ maps, const int* __restrict__ own_cols,
                                                  double* __restrict__ Ba, double mu, double* __restrict__ Ppk,
                                                  double* __restrict__ Pdense) {
    __shared__ double sA[NB * (TS + 1)], sB[NB * (TS + 1)];
    const EigProb p = probs[blockIdx.x];
    const int m = p.m, no = p.nown;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* Z = Za + p.aoff;
    const double* tau = Ta + p.voff;
    const double* ev = Wa + p.voff;
    double* W0 = Ba + p.boff;                       // (S U) rows block: free after the prepare step
    const double* U2 = Ba + p.boff + 3 * (int64_t)no * m;   // U[c_t, :] (second half of G)
    double* W = Ba + p.boff + (int64_t)no * m;      // m x nown, column-major
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kT / 32;
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
    // Q W (the tiles' staging space as scratch)
    wy_apply(C, m, tau, W, no, false, WySmem{sA, sB});
    // L^-T w: back substitution, warp per column
    for (int t = warp; t < no; t += nwarp) {
        double* w = W + (int64_t)t * m;
        for (int i = m - 1; i >= 0; --i) {
            const double* li = L + (int64_t)i * m;
            double s = 0.0;
            for (int k = i + 1 + lane; k < m; k += 32) s = fma(li[k], w[k], s);
            s = warp_sum(s);
            if (lane == 0) w[i] = (w[i] - s) / li[i];
            __syncwarp();
        }
    }
    __syncthreads();
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

}  // namespace

struct EigBatch {
    int nprob = 0;
    int maxm = 0;
    std::vector<EigProb> hp;
    DevBuf probs, order, counter, Ca, La, Za, Qa, Va, Da, Ea, Ta, Wa, Ba, status;
    ~EigBatch() {
        for (DevBuf* b : {&probs, &order, &counter, &Ca, &La, &Za, &Qa, &Va, &Da, &Ea, &Ta, &Wa, &Ba, &status})
            b->release();
    }
};

namespace {

void eig_setup_attrs() {
    static const bool done = [] {
        PTB_CUDA(cudaFuncSetAttribute(k_eig_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)stage_smem_bytes(kEigBatchMax)));
        return true;
    }();
    (void)done;
}

}  // namespace

std::shared_ptr<EigBatch> eig_batch_launch(ptbgpu_ctx* c, int64_t n, const double* H, const double* S,
                                           const std::vector<EigProbHost>& probs, const int* d_maps,
                                            const int* d_own_cols, const int* d_ipos, double* d_e, double* d_fe,
                                            int prl, double* flops) {
    (void)prl;
    if (probs.empty()) return nullptr;
    eig_setup_attrs();
    cudaStream_t s = c->stream;
    auto eb = std::make_shared<EigBatch>();
    eb->nprob = (int)probs.size();
    int64_t asz = 0, vsz = 0, bsz = 0, psz = 0;
    for (const EigProbHost& q : probs) {
        PTB_CHECK(q.m >= 1 && q.m <= kEigBatchMax, PTBGPU_EINVAL, "submatrix %d of order %d outside the batched solver",
                  q.k + 1, q.m);
        EigProb p{};
        p.k = q.k;
        p.m = q.m;
        p.nown = q.nown;
        p.moff = q.moff;
        p.eoff = q.eoff;
        p.o0 = q.o0;
        p.gbase = q.gbase;
        p.gld = q.gld < 0 ? n : q.gld;
        p.poff = psz;
        psz += (int64_t)q.m * q.nown;
        p.aoff = asz;
        p.voff = vsz;
        p.boff = bsz;
        asz += (int64_t)q.m * q.m;
        vsz += q.m;
        bsz += 4 * (int64_t)q.nown * q.m;
        eb->maxm = std::max(eb->maxm, q.m);
        eb->hp.push_back(p);
        if (flops) *flops += 7.0 * std::pow((double)q.m, 3);
    }
    const int np = eb->nprob;
    eb->probs.reserve(sizeof(EigProb) * np);
    for (DevBuf* b : {&eb->Ca, &eb->La, &eb->Za, &eb->Qa, &eb->Va}) b->reserve(sizeof(double) * asz);
    for (DevBuf* b : {&eb->Da, &eb->Ea, &eb->Ta, &eb->Wa}) b->reserve(sizeof(double) * vsz);
    eb->Ba.reserve(sizeof(double) * std::max<int64_t>(bsz, 1));
    eb->status.reserve(sizeof(int) * np);
    PTB_CUDA(cudaMemcpyAsync(eb->probs.ptr, eb->hp.data(), sizeof(EigProb) * np, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(eb->status.ptr, 0, sizeof(int) * np, s));
    const EigProb* dp = eb->probs.as<EigProb>();
    int* dst = eb->status.as<int>();

    // largest first, so that the small submatrices fill in around the large ones
    std::vector<int> ord(np);
    for (int q = 0; q < np; ++q) ord[q] = q;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return eb->hp[a].m > eb->hp[b].m; });
    eb->order.reserve(sizeof(int) * np);
    eb->counter.reserve(sizeof(int));
    PTB_CUDA(cudaMemcpyAsync(eb->order.ptr, ord.data(), sizeof(int) * np, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(eb->counter.ptr, 0, sizeof(int), s));
    const int M = (eb->maxm + 1) & ~1;
    const int grid = std::min(np, c->num_sms > 0 ? c->num_sms : 148);
    k_eig_fused<<<grid, kT, stage_smem_bytes(M), s>>>(
        dp, eb->order.as<int>(), np, eb->counter.as<int>(), M, d_maps, H, S, eb->Ca.as<double>(),
        eb->La.as<double>(), eb->Za.as<double>(), eb->Qa.as<double>(), eb->Va.as<double>(), eb->Da.as<double>(),
        eb->Ea.as<double>(), eb->Ta.as<double>(), eb->Wa.as<double>(), eb->Ba.as<double>(), d_own_cols, d_ipos, d_e,
        d_fe, dst);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return eb;
}

void eig_batch_check(ptbgpu_ctx* c, EigBatch& eb) {
    cudaStream_t s = c->stream;
    const int np = eb.nprob;
    std::vector<int> hst(np);
    PTB_CUDA(cudaMemcpyAsync(hst.data(), eb.status.ptr, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < np; ++q)
        PTB_CHECK(hst[q] <= 0, PTBGPU_ENOTSPD, "overlap submatrix %d not positive definite (leading minor %d)",
                  eb.hp[q].k + 1, hst[q]);
    for (int q = 0; q < np; ++q)
        PTB_CHECK(hst[q] == kStOk, PTBGPU_EITER, "tridiagonal eigensolver did not converge on submatrix %d",
                  eb.hp[q].k + 1);
}

void eig_batch_final(ptbgpu_ctx* c, EigBatch& eb, double mu, int64_t n, const int* d_maps, const int* d_own_cols,
                     double* dP, double* dPdense) {
    (void)n;
    if (eb.nprob == 0) return;
    cudaStream_t s = c->stream;
    k_eig_final<<<eb.nprob, kT, 0, s>>>(eb.probs.as<EigProb>(), eb.Ca.as<double>(), eb.La.as<double>(),
                                        eb.Ta.as<double>(), eb.Wa.as<double>(), eb.Za.as<double>(), d_maps,
                                        d_own_cols, eb.Ba.as<double>(), mu, dP, dPdense);
    count_launch();
    PTB_CUDA(cudaGetLastError());
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
        PTB_CHECK(dims[k] >= 1 && dims[k] <= kEigBatchMax && nown[k] >= 1 && nown[k] <= dims[k], PTBGPU_EINVAL,
                  "problem %lld: order %lld (1..%d) or owned count %lld out of range", (long long)k,
                  (long long)dims[k], kEigBatchMax, (long long)nown[k]);
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
