// Batched FP64 generalized eigensolver of the submatrix method: one CTA per
// submatrix for the dense stages, one warp per submatrix for the QL chase.
//
// The reference solves H_k U = S_k U diag(e) with LAPACK dsygvd per submatrix
// (la_sygvd, source/sm.f90:296-299), forms S_k U for the electron-count
// weights fe (source/sm.f90:305-310) and, at the final chemical potential,
// P_k = U occ U^T of which only the owned columns are kept
// (source/sm.f90:343-362).  Only these quantities leave the solver, and all of
// them are reached without forming U:
//
//   S_k = L L^T                      Cholesky, blocked (k_eig_potrf)
//   C   = L^-1 H_k L^-T              two blocked triangular solves (k_eig_reduce)
//   C   = Q T Q^T                    Householder tridiagonalisation, lower,
//                                    Q = H_0 H_1 ... H_{m-3} (k_eig_sytrd)
//   T   = Z diag(e) Z^T              implicit QL with Wilkinson shifts; Z is
//                                    the product of the Givens rotations in the
//                                    order they are made, which are stored
//                                    (k_eig_ql)
//   U   = L^-T Q Z                   never formed:
//     rows c of U    = (L^-T)[c,:] Q Z,  rows c of S U = L[c,:] Q Z  for the
//     owned columns c (k_eig_rows), so fe_j = sum_c (SU)[c,j] U[c,j];
//     P_k[:,c] = U (occ o U[c,:]^T) = L^-T (Q (Z w)) with Z w applying the
//     stored rotations in reverse (k_eig_final).
//
// The QL iteration is the implicit QL algorithm with a Wilkinson shift for
// symmetric tridiagonal matrices (Bowdler, Martin, Reinsch and Wilkinson 1968,
// the tql2 procedure), restated here with its rotations recorded instead of
// accumulated into an m x m matrix.  Each step's quantities are summed in a
// fixed order, so results do not depend on scheduling.
#include <algorithm>
#include <cmath>
#include <vector>

#include "sm_eig.cuh"

namespace ptb {

namespace {

constexpr int kT = 256;           // threads of the per-problem CTAs
constexpr int NB = 32;            // panel width of the blocked stages
constexpr int TS = 64;            // output tile of the blocked updates
constexpr int kQlWarps = 4;       // problems per CTA of the QL kernel
constexpr int kQlMaxIter = 30;    // QL sweeps per eigenvalue before giving up (as LAPACK's dsteqr)

// Status words per problem.
constexpr int kStOk = 0;
constexpr int kStNoConv = -1;     // QL sweeps exhausted
constexpr int kStRotCap = -2;     // rotation / sweep storage exhausted (retried with more)
// > 0: leading minor of that order of S_k is not positive definite

struct EigProb {
    int k, m, nown, pad;
    int64_t moff, eoff, o0;
    int64_t gbase, gld;   // the problem's H / S: element (i, j) at gbase + map(i) + map(j) gld
    int64_t poff;         // dense output of the owned columns of P (m x nown, column-major)
    int64_t aoff;     // C and L arenas (m x m, column-major, ld = m)
    int64_t voff;     // d, e, tau, eigenvalue arenas (m)
    int64_t boff;     // owned-row arena (2 nown x m, row-major)
    int64_t roff, rcap;   // rotations (double2)
    int64_t soff, scap;   // sweeps (int4: l, mm, count, first rotation)
};

// ---------------------------------------------------------------------------
// C[r0+i, c0+j] -= sum_{k < kk} A(i,k) B(k,j) on one TS x TS tile (mr x nc
// valid), 256 threads with 4 x 4 outputs each.
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
    const int tx = tid & 15, ty = tid >> 4;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int k = 0; k < kk; ++k) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = sA[k * (TS + 1) + tx + 16 * a];
#pragma unroll
        for (int b = 0; b < 4; ++b) bv[b] = sB[k * (TS + 1) + ty + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = ty + 16 * b;
        if (j >= nc) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = tx + 16 * a;
            if (i >= mr || (LOWER && r0 + i < c0 + j)) continue;
            double* p = C + (int64_t)(r0 + i) + (int64_t)(c0 + j) * ldc;
            *p -= acc[a][b];
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
// Gather H_k, S_k (source/sm.f90:240-246) into the C and L arenas.
__global__ void __launch_bounds__(kT) k_eig_gather(const EigProb* __restrict__ probs, const int* __restrict__ maps,
                                                   const double* __restrict__ H,
                                                   const double* __restrict__ S, double* __restrict__ Ca,
                                                   double* __restrict__ La) {
    const EigProb p = probs[blockIdx.x];
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
// upper triangle is zeroed.  status = order of the first non-positive pivot.
__global__ void __launch_bounds__(kT) k_eig_potrf(const EigProb* __restrict__ probs, double* __restrict__ La,
                                                  int* __restrict__ status) {
    extern __shared__ double sm[];
    double* sA = sm;                       // NB x (TS+1)
    double* sB = sA + NB * (TS + 1);       // NB x (TS+1)
    double* sD = sB + NB * (TS + 1);       // NB x (NB+1), sD[i + j*(NB+1)]
    __shared__ int fail;
    const EigProb p = probs[blockIdx.x];
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
    if (tid == 0) status[blockIdx.x] = fail;
    if (fail) return;
    for (int j = 1; j < m; ++j)
        for (int i = tid; i < j; i += kT) L[(int64_t)i + (int64_t)j * m] = 0.0;
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
__global__ void __launch_bounds__(kT) k_eig_reduce(const EigProb* __restrict__ probs, const double* __restrict__ La,
                                                   double* __restrict__ Ca, const int* __restrict__ status) {
    extern __shared__ double sm[];
    double* sA = sm;
    double* sB = sA + NB * (TS + 1);
    double* sD = sB + NB * (TS + 1);
    if (status[blockIdx.x] != kStOk) return;
    const EigProb p = probs[blockIdx.x];
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

__global__ void __launch_bounds__(kT) k_eig_sytrd(const EigProb* __restrict__ probs, double* __restrict__ Ca,
                                                  double* __restrict__ Da, double* __restrict__ Ea,
                                                  double* __restrict__ Ta, const int* __restrict__ status) {
    __shared__ double vc[kEigBatchMax], wc[kEigBatchMax], vn[kEigBatchMax];
    __shared__ double red[kT / 32];
    __shared__ double sh_tau, sh_alpha;
    if (status[blockIdx.x] != kStOk) return;
    const EigProb p = probs[blockIdx.x];
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
        for (int k = r0; k < m; ++k) {
            const double vk = vc[k], wk = wc[k], nk = vn[k];
            double* col = A + (int64_t)k * m;
#pragma unroll
            for (int q = 0; q < kSyRows; ++q) {
                const int r = r0 + tid + q * kT;
                if (r < m) {
                    double a = col[r];
                    a -= vr[q] * wk + wr[q] * vk;
                    col[r] = a;
                    acc[q] = fma(a, nk, acc[q]);
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
// Implicit QL with Wilkinson shift on (d, e); lane 0 of a warp per problem
// chases, with d and e in shared memory.  Rotation q of a sweep over [l, mm]
// acts on indices (i, i+1), i = mm-1-q, with (c, s): columns of Z transform as
// z_{i+1} <- s z_i + c z_{i+1}, z_i <- c z_i - s z_{i+1}.
__global__ void k_eig_ql(int nprob, const EigProb* __restrict__ probs, const double* __restrict__ Da,
                         const double* __restrict__ Ea, double* __restrict__ Wa, double2* __restrict__ cs,
                         int4* __restrict__ sw, int* __restrict__ nsw_out, int* __restrict__ status, int maxm,
                         int only_capped) {
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pi = blockIdx.x * kQlWarps + warp;
    if (pi >= nprob) return;
    if (only_capped ? status[pi] != kStRotCap : status[pi] != kStOk) return;
    const EigProb p = probs[pi];
    const int m = p.m;
    double* d = sm + (size_t)warp * 2 * maxm;
    double* e = d + maxm;
    for (int i = lane; i < m; i += 32) {
        d[i] = Da[p.voff + i];
        e[i] = (i < m - 1) ? Ea[p.voff + i] : 0.0;
    }
    __syncwarp();
    if (lane == 0) {
        const double eps = 2.220446049250313e-16;
        double2* rot = cs + p.roff;
        int4* swp = sw + p.soff;
        int64_t nrot = 0;
        int nsw = 0, st = kStOk;
        for (int l = 0; l < m && st == kStOk; ++l) {
            int iter = 0;
            for (;;) {
                int mm = l;
                for (; mm < m - 1; ++mm) {
                    const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
                    if (fabs(e[mm]) <= eps * dd) break;
                }
                if (mm == l) break;
                if (++iter > kQlMaxIter) {
                    st = kStNoConv;
                    break;
                }
                if (nsw >= p.scap || nrot + (mm - l) > p.rcap) {
                    st = kStRotCap;
                    break;
                }
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = hypot(g, 1.0);
                g = d[mm] - d[l] + e[l] / (g + copysign(r, g));
                double s = 1.0, c = 1.0, pp = 0.0;
                const int64_t first = nrot;
                bool underflow = false;
                for (int i = mm - 1; i >= l; --i) {
                    const double f = s * e[i], b = c * e[i];
                    // r = |(f, g)|, (s, c) = (f, g) / r from one reciprocal square
                    // root (the chase is a chain of dependent operations; this
                    // is its longest link)
                    const double q = fma(f, f, g * g);
                    if (q == 0.0) {
                        e[i + 1] = 0.0;
                        d[i + 1] -= pp;
                        e[mm] = 0.0;
                        underflow = true;
                        break;
                    }
                    const double rq = rsqrt(q);
                    e[i + 1] = q * rq;
                    s = f * rq;
                    c = g * rq;
                    g = d[i + 1] - pp;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    pp = s * r;
                    d[i + 1] = g + pp;
                    g = c * r - b;
                    rot[nrot++] = make_double2(c, s);
                }
                swp[nsw++] = make_int4(l, mm, (int)(nrot - first), (int)first);
                if (underflow) continue;
                d[l] -= pp;
                e[l] = g;
                e[mm] = 0.0;
            }
        }
        nsw_out[pi] = nsw;
        status[pi] = st;
    }
    __syncwarp();
    for (int i = lane; i < m; i += 32) Wa[p.voff + i] = d[i];
}

// ---------------------------------------------------------------------------
// Owned rows of S U and U, fe and the eigenpairs.  B holds 2 nown rows of
// length m (row-major): rows t < nown are L[c_t,:] -> (S U)[c_t,:], rows
// nown + t are (L^-T)[c_t,:] -> U[c_t,:].
__global__ void __launch_bounds__(kT) k_eig_rows(const EigProb* __restrict__ probs, const double* __restrict__ Ca,
                                                 const double* __restrict__ La, const double* __restrict__ Ta,
                                                 const double* __restrict__ Wa, const double2* __restrict__ cs,
                                                 const int4* __restrict__ sw, const int* __restrict__ nsw,
                                                 const int* __restrict__ own_cols, const int* __restrict__ ipos,
                                                 double* __restrict__ Ba, double* __restrict__ e_out,
                                                 double* __restrict__ fe_out, const int* __restrict__ status) {
    __shared__ double v[kEigBatchMax];
    if (status[blockIdx.x] != kStOk) return;
    const EigProb p = probs[blockIdx.x];
    const int m = p.m, no = p.nown, nb2 = 2 * no;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* tau = Ta + p.voff;
    double* B = Ba + p.boff;
    double* B2 = B + (int64_t)no * m;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kT / 32;
    // (1) L rows and unit vectors
    for (int t = 0; t < no; ++t) {
        const int ct = ipos[own_cols[p.o0 + t]];
        for (int r = tid; r < m; r += kT) {
            B[(int64_t)t * m + r] = (r <= ct) ? L[ct + (int64_t)r * m] : 0.0;
            B2[(int64_t)t * m + r] = (r == ct) ? 1.0 : 0.0;
        }
    }
    __syncthreads();
    // (2) rows of L^-T: x_t = L^-1 e_{c_t}, 32-row blocks
    for (int i0 = 0; i0 < m; i0 += NB) {
        const int nb = min(NB, m - i0), i1 = i0 + nb;
        for (int t = warp; t < no; t += nwarp) {
            double* x = B2 + (int64_t)t * m;
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
            double* x = B2 + (int64_t)t * m;
            double s = 0.0;
            for (int k = 0; k < nb; ++k) s = fma(L[r + (int64_t)(i0 + k) * m], x[i0 + k], s);
            x[r] -= s;
        }
        __syncthreads();
    }
    // (3) B <- B Q = B H_0 H_1 ... H_{m-3}
    for (int k = 0; k + 2 < m; ++k) {
        const double tk = tau[k];
        if (tk == 0.0) continue;
        for (int r = k + 1 + tid; r < m; r += kT) v[r] = (r == k + 1) ? 1.0 : C[r + (int64_t)k * m];
        __syncthreads();
        for (int b = warp; b < nb2; b += nwarp) {
            double* row = B + (int64_t)b * m;
            double s = 0.0;
            for (int r = k + 1 + lane; r < m; r += 32) s = fma(row[r], v[r], s);
            s = warp_sum(s) * tk;
            for (int r = k + 1 + lane; r < m; r += 32) row[r] -= s * v[r];
        }
        __syncthreads();
    }
    // (4) B <- B Z: the stored rotations in the order they were made
    const double2* rot = cs + p.roff;
    const int4* swp = sw + p.soff;
    const int ns = nsw[blockIdx.x];
    for (int b = tid; b < nb2; b += kT) {
        double* row = B + (int64_t)b * m;
        for (int q = 0; q < ns; ++q) {
            const int4 h = swp[q];
            const int mm = h.y, cnt = h.z;
            const double2* rr = rot + h.w;
            double hi = row[mm];
            for (int u = 0; u < cnt; ++u) {
                const int i = mm - 1 - u;
                const double2 g = rr[u];
                const double lo = row[i];
                row[i + 1] = g.y * lo + g.x * hi;
                hi = g.x * lo - g.y * hi;
            }
            row[mm - cnt] = hi;
        }
    }
    __syncthreads();
    // (5) fe_j = sum_t (SU)[c_t, j] U[c_t, j]; eigenvalues
    for (int j = tid; j < m; j += kT) {
        double f = 0.0;
        for (int t = 0; t < no; ++t) f = fma(B[(int64_t)t * m + j], B2[(int64_t)t * m + j], f);
        e_out[p.eoff + j] = Wa[p.voff + j];
        fe_out[p.eoff + j] = f;
    }
}

// ---------------------------------------------------------------------------
// Owned columns of P_k at mu: w_t = occ o U[c_t,:]^T, w <- Z w (rotations in
// reverse), w <- Q w (reflectors in reverse), w <- L^-T w; scattered into the
// packed result, rows map(i) <= c_t of column c_t.
__global__ void __launch_bounds__(kT) k_eig_final(const EigProb* __restrict__ probs, const double* __restrict__ Ca,
                                                  const double* __restrict__ La, const double* __restrict__ Ta,
                                                  const double* __restrict__ Wa, const double2* __restrict__ cs,
                                                  const int4* __restrict__ sw, const int* __restrict__ nsw,
                                                  const int* __restrict__ maps, const int* __restrict__ own_cols,
                                                  double* __restrict__ Ba, double mu, double* __restrict__ Ppk,
                                                  double* __restrict__ Pdense) {
    __shared__ double v[kEigBatchMax];
    const EigProb p = probs[blockIdx.x];
    const int m = p.m, no = p.nown;
    const double* C = Ca + p.aoff;
    const double* L = La + p.aoff;
    const double* tau = Ta + p.voff;
    const double* ev = Wa + p.voff;
    double* W = Ba + p.boff;                    // reuses the (S U) rows
    const double* U2 = W + (int64_t)no * m;     // U[c_t, :]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kT / 32;
    for (int64_t q = tid; q < (int64_t)no * m; q += kT) {
        const int j = (int)(q % m);
        const double e = ev[j];
        const double occ = e < mu ? 2.0 : (e == mu ? 1.0 : 0.0);
        W[q] = occ * U2[q];
    }
    __syncthreads();
    // Z w: rotations in reverse order
    const double2* rot = cs + p.roff;
    const int4* swp = sw + p.soff;
    const int ns = nsw[blockIdx.x];
    for (int t = tid; t < no; t += kT) {
        double* w = W + (int64_t)t * m;
        for (int q = ns - 1; q >= 0; --q) {
            const int4 h = swp[q];
            const int mm = h.y, cnt = h.z;
            const double2* rr = rot + h.w;
            int i = mm - cnt;
            double lo = w[i];
            for (int u = cnt - 1; u >= 0; --u, ++i) {
                const double2 g = rr[u];
                const double hi = w[i + 1];
                w[i] = g.x * lo + g.y * hi;
                lo = g.x * hi - g.y * lo;
            }
            w[i] = lo;
        }
    }
    __syncthreads();
    // Q w = H_0 (H_1 (... H_{m-3} w))
    for (int k = m - 3; k >= 0; --k) {
        const double tk = tau[k];
        if (tk == 0.0) continue;
        for (int r = k + 1 + tid; r < m; r += kT) v[r] = (r == k + 1) ? 1.0 : C[r + (int64_t)k * m];
        __syncthreads();
        for (int t = warp; t < no; t += nwarp) {
            double* w = W + (int64_t)t * m;
            double s = 0.0;
            for (int r = k + 1 + lane; r < m; r += 32) s = fma(v[r], w[r], s);
            s = warp_sum(s) * tk;
            for (int r = k + 1 + lane; r < m; r += 32) w[r] -= s * v[r];
        }
        __syncthreads();
    }
    // L^-T w: back substitution, warp per column
    for (int t = warp; t < no; t += nwarp) {
        double* w = W + (int64_t)t * m;
        for (int i = m - 1; i >= 0; --i) {
            const double* li = L + (int64_t)i * m;   // column i of L: L[k, i], k > i
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
    DevBuf probs, Ca, La, Da, Ea, Ta, Wa, Ba, cs, sw, nsw, status;
    ~EigBatch() {
        for (DevBuf* b : {&probs, &Ca, &La, &Da, &Ea, &Ta, &Wa, &Ba, &cs, &sw, &nsw, &status}) b->release();
    }
};

namespace {

constexpr size_t kSmemBlocked = sizeof(double) * (2 * NB * (TS + 1) + NB * (NB + 1));

void eig_setup_attrs() {
    static const bool done = [] {
        PTB_CUDA(cudaFuncSetAttribute(k_eig_potrf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBlocked));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBlocked));
        PTB_CUDA(cudaFuncSetAttribute(k_eig_ql, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * 2 * kEigBatchMax * kQlWarps)));
        return true;
    }();
    (void)done;
}

// Rotation and sweep capacities: about m^2 rotations are typical; the first
// pass reserves 1.5 m^2 + 64 m, a problem that needs more is redone with the
// bound kQlMaxIter m^2 (kQlMaxIter sweeps of at most m rotations per eigenvalue).
int64_t rot_cap(int m, bool full) {
    return full ? (int64_t)kQlMaxIter * m * m + 64 : (int64_t)(1.5 * m * m) + 64 * (int64_t)m;
}
int64_t sweep_cap(int m, bool full) { return full ? (int64_t)kQlMaxIter * m + 8 : 4 * (int64_t)m + 8; }

}  // namespace

std::shared_ptr<EigBatch> eig_batch_prepare(ptbgpu_ctx* c, int64_t n, const double* H, const double* S,
                                            const std::vector<EigProbHost>& probs, const int* d_maps,
                                            const int* d_own_cols, const int* d_ipos, double* d_e, double* d_fe,
                                            int prl, double* flops) {
    if (probs.empty()) return nullptr;
    eig_setup_attrs();
    cudaStream_t s = c->stream;
    auto eb = std::make_shared<EigBatch>();
    eb->nprob = (int)probs.size();
    int64_t asz = 0, vsz = 0, bsz = 0, rsz = 0, ssz = 0, psz = 0;
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
        p.roff = rsz;
        p.rcap = rot_cap(q.m, false);
        p.soff = ssz;
        p.scap = sweep_cap(q.m, false);
        asz += (int64_t)q.m * q.m;
        vsz += q.m;
        bsz += 2 * (int64_t)q.nown * q.m;
        rsz += p.rcap;
        ssz += p.scap;
        eb->maxm = std::max(eb->maxm, q.m);
        eb->hp.push_back(p);
        if (flops) *flops += 7.0 * std::pow((double)q.m, 3);
    }
    const int np = eb->nprob;
    eb->probs.reserve(sizeof(EigProb) * np);
    eb->Ca.reserve(sizeof(double) * asz);
    eb->La.reserve(sizeof(double) * asz);
    eb->Da.reserve(sizeof(double) * vsz);
    eb->Ea.reserve(sizeof(double) * vsz);
    eb->Ta.reserve(sizeof(double) * vsz);
    eb->Wa.reserve(sizeof(double) * vsz);
    eb->Ba.reserve(sizeof(double) * std::max<int64_t>(bsz, 1));
    eb->cs.reserve(sizeof(double2) * rsz);
    eb->sw.reserve(sizeof(int4) * ssz);
    eb->nsw.reserve(sizeof(int) * np);
    eb->status.reserve(sizeof(int) * np);
    PTB_CUDA(cudaMemcpyAsync(eb->probs.ptr, eb->hp.data(), sizeof(EigProb) * np, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(eb->status.ptr, 0, sizeof(int) * np, s));
    const EigProb* dp = eb->probs.as<EigProb>();
    int* dst = eb->status.as<int>();

    k_eig_gather<<<np, kT, 0, s>>>(dp, d_maps, H, S, eb->Ca.as<double>(), eb->La.as<double>());
    k_eig_potrf<<<np, kT, kSmemBlocked, s>>>(dp, eb->La.as<double>(), dst);
    k_eig_reduce<<<np, kT, kSmemBlocked, s>>>(dp, eb->La.as<double>(), eb->Ca.as<double>(), dst);
    k_eig_sytrd<<<np, kT, 0, s>>>(dp, eb->Ca.as<double>(), eb->Da.as<double>(), eb->Ea.as<double>(),
                                  eb->Ta.as<double>(), dst);
    const size_t ql_smem = sizeof(double) * 2 * eb->maxm * kQlWarps;
    k_eig_ql<<<(np + kQlWarps - 1) / kQlWarps, 32 * kQlWarps, ql_smem, s>>>(
        np, dp, eb->Da.as<double>(), eb->Ea.as<double>(), eb->Wa.as<double>(), eb->cs.as<double2>(),
        eb->sw.as<int4>(), eb->nsw.as<int>(), dst, eb->maxm, 0);
    count_launch(5);
    PTB_CUDA(cudaGetLastError());
    std::vector<int> hst(np);
    PTB_CUDA(cudaMemcpyAsync(hst.data(), dst, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < np; ++q)
        PTB_CHECK(hst[q] <= 0, PTBGPU_ENOTSPD, "overlap submatrix %d not positive definite (leading minor %d)",
                  eb->hp[q].k + 1, hst[q]);
    // problems whose rotations did not fit: redo them with the full bound
    std::vector<int> redo;
    for (int q = 0; q < np; ++q)
        if (hst[q] == kStRotCap) redo.push_back(q);
    if (!redo.empty()) {
        int64_t extra = 0, extra_s = 0;
        for (int q : redo) {
            extra += rot_cap(eb->hp[q].m, true);
            extra_s += sweep_cap(eb->hp[q].m, true);
        }
        DevBuf cs2, sw2;
        cs2.reserve(sizeof(double2) * (rsz + extra));
        sw2.reserve(sizeof(int4) * (ssz + extra_s));
        PTB_CUDA(cudaMemcpyAsync(cs2.ptr, eb->cs.ptr, sizeof(double2) * rsz, cudaMemcpyDeviceToDevice, s));
        PTB_CUDA(cudaMemcpyAsync(sw2.ptr, eb->sw.ptr, sizeof(int4) * ssz, cudaMemcpyDeviceToDevice, s));
        int64_t ro = rsz, so = ssz;
        for (int q : redo) {
            EigProb& p = eb->hp[q];
            p.roff = ro;
            p.rcap = rot_cap(p.m, true);
            p.soff = so;
            p.scap = sweep_cap(p.m, true);
            ro += p.rcap;
            so += p.scap;
        }
        PTB_CUDA(cudaStreamSynchronize(s));
        std::swap(eb->cs, cs2);
        std::swap(eb->sw, sw2);
        cs2.release();
        sw2.release();
        PTB_CUDA(cudaMemcpyAsync(eb->probs.ptr, eb->hp.data(), sizeof(EigProb) * np, cudaMemcpyHostToDevice, s));
        // the kernel only redoes the problems still marked kStRotCap
        k_eig_ql<<<(np + kQlWarps - 1) / kQlWarps, 32 * kQlWarps, ql_smem, s>>>(
            np, dp, eb->Da.as<double>(), eb->Ea.as<double>(), eb->Wa.as<double>(), eb->cs.as<double2>(),
            eb->sw.as<int4>(), eb->nsw.as<int>(), dst, eb->maxm, 1);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        PTB_CUDA(cudaMemcpyAsync(hst.data(), dst, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaStreamSynchronize(s));
        log_line(prl, 2, " * submatrix QL: %zu problems redone with the full rotation bound", redo.size());
    }
    for (int q = 0; q < np; ++q)
        PTB_CHECK(hst[q] == kStOk, PTBGPU_EITER, "tridiagonal QL iteration did not converge on submatrix %d",
                  eb->hp[q].k + 1);
    k_eig_rows<<<np, kT, 0, s>>>(dp, eb->Ca.as<double>(), eb->La.as<double>(), eb->Ta.as<double>(),
                                 eb->Wa.as<double>(), eb->cs.as<double2>(), eb->sw.as<int4>(), eb->nsw.as<int>(),
                                 d_own_cols, d_ipos, eb->Ba.as<double>(), d_e, d_fe, dst);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return eb;
}

void eig_batch_final(ptbgpu_ctx* c, EigBatch& eb, double mu, int64_t n, const int* d_maps, const int* d_own_cols,
                     double* dP, double* dPdense) {
    (void)n;
    if (eb.nprob == 0) return;
    cudaStream_t s = c->stream;
    k_eig_final<<<eb.nprob, kT, 0, s>>>(eb.probs.as<EigProb>(), eb.Ca.as<double>(), eb.La.as<double>(),
                                        eb.Ta.as<double>(), eb.Wa.as<double>(), eb.cs.as<double2>(),
                                        eb.sw.as<int4>(), eb.nsw.as<int>(), d_maps, d_own_cols, eb.Ba.as<double>(),
                                        mu, dP, dPdense);
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
        eig_batch_prepare(c, 0, b.h.as<double>(), b.s.as<double>(), probs, b.maps.as<int>(), b.own.as<int>(),
                          b.ipos.as<int>(), b.e.as<double>(), b.fe.as<double>(), 0, nullptr);
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
