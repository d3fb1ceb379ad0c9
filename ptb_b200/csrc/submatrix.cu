// Submatrix method, sm_stupid_simple (source/sm.f90:34-409), on the device.
//
//  1. column grouping (host, source/sm.f90:92-162): owned columns per submatrix
//  2. pattern scan: row i joins submatrix k iff H(i,c) > 0 or S(i,c) > 0 or
//     i == c for an owned column c (strictly positive, source/sm.f90:210-228);
//     one coalesced pass over H and S, flags[k][i]
//  3. ordered compaction of the flags into the sorted index maps (CSR) and the
//     position of every owned column inside its map
//  4. submatrices bucketed by padded size M (multiple of 32); H_k, S_k gathered
//     into M x M batches, padded with H = 1e3 I, S = I (eigenvalues far above
//     the mu bracket, eigenvectors outside the real block: they carry no
//     electrons and no density);  S_k = L L^T, C = L^-1 H_k L^-T, C = V w V^T,
//     U = L^-T V  (the generalized problem of la_sygvd, source/sm.f90:296-299)
//  5. fe_j = sum_{c owned} (S_k U)_{ic,j} U_{ic,j}  (source/sm.f90:305-310)
//  6. mu bisection on [-10, 10] with occupations 2 / 1 / 0 for e < / = / > mu,
//     stop on |a-b| < 1e-3 or |nel - nelref| < 1e-5 (REAL(4) literals), then
//     one final pass at the same mu (source/sm.f90:191-383) - one block
//  7. final density: P(map(i), c) = sum_j U_ij occ_j U_{ic,j} for owned c,
//     written directly into the packed result for map(i) <= c (packsym keeps
//     column c, rows <= c; rows outside the map stay zero, source/sm.f90:201-203,
//     343-362, 387).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "sm_eig.cuh"

namespace ptb {

namespace {

constexpr double kPadDiag = 1.0e3;
// generator seed of the mode-4 k-means when the caller supplies no partition
// (the reference seeds its Fortran generator with 42 * (i - 1), source/sm.f90:21-32)
constexpr uint64_t kKmeansSeed = 42;

// (2) flags[k*n + i] |= (H(i,c) > 0 || S(i,c) > 0 || i == c) for column c of submatrix owner[c]
__global__ void k_pattern(int64_t n, const double* __restrict__ H, const double* __restrict__ S,
                          const int* __restrict__ owner, uint8_t* __restrict__ flags) {
    for (int64_t c = blockIdx.x; c < n; c += gridDim.x) {
        const int k = owner[c];
        if (k < 0) continue;
        uint8_t* f = flags + (int64_t)k * n;
        const double* hc = H + c * n;
        const double* sc = S + c * n;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
            if (hc[i] > 0.0 || sc[i] > 0.0 || i == c) f[i] = 1;
    }
}

__global__ void k_count(int64_t n, const uint8_t* __restrict__ flags, int* __restrict__ counts) {
    const int k = blockIdx.x;
    int cnt = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) cnt += flags[(int64_t)k * n + i];
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    __shared__ int sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        counts[k] = t;
    }
}

// (3) ordered compaction; 256 threads per block (one submatrix per block).
__global__ void k_fill(int64_t n, const uint8_t* __restrict__ flags, const int64_t* __restrict__ offs,
                       const int* __restrict__ owner, int* __restrict__ maps, int* __restrict__ ipos) {
    const int k = blockIdx.x;
    const uint8_t* f = flags + (int64_t)k * n;
    int* mp = maps + offs[k];
    __shared__ int warp_tot[8];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t c0 = 0; c0 < n; c0 += blockDim.x) {
        const int64_t i = c0 + threadIdx.x;
        const bool on = i < n && f[i];
        const unsigned m = __ballot_sync(0xffffffffu, on);
        const int before = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) warp_tot[w] = __popc(m);
        __syncthreads();
        int wbase = 0;
        for (int q = 0; q < w; ++q) wbase += warp_tot[q];
        if (on) {
            const int p = base + wbase + before;
            mp[p] = (int)i;
            if (owner[i] == k) ipos[i] = p;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int q = 0; q < 8; ++q) t += warp_tot[q];
            base += t;
        }
        __syncthreads();
    }
}

struct Prob {
    int k;          // submatrix index
    int m;          // real dimension
    int64_t moff;   // offset of its map in maps[]
    int64_t eoff;   // offset of its eigenpairs in e[] / fe[]
};

// (4) gather H_k, S_k into the padded M x M batch (column-major per problem).
__global__ void k_gather(int M, const Prob* __restrict__ probs, const int* __restrict__ maps, int64_t n,
                         const double* __restrict__ H, const double* __restrict__ S, double* __restrict__ Hb,
                         double* __restrict__ Sb) {
    const Prob p = probs[blockIdx.z];
    const int* mp = maps + p.moff;
    double* hb = Hb + (int64_t)blockIdx.z * M * M;
    double* sb = Sb + (int64_t)blockIdx.z * M * M;
    const int i = blockIdx.x * 32 + threadIdx.x;
    for (int j = blockIdx.y * 8 + threadIdx.y; j < M; j += gridDim.y * 8) {
        if (i >= M) continue;
        double h, s;
        if (i < p.m && j < p.m) {
            const int64_t gi = mp[i], gj = mp[j];
            h = H[gi + gj * n];
            s = S[gi + gj * n];
        } else {
            h = (i == j) ? kPadDiag : 0.0;
            s = (i == j) ? 1.0 : 0.0;
        }
        hb[i + (int64_t)j * M] = h;
        sb[i + (int64_t)j * M] = s;
    }
}

// (5) fe_j for problem blockIdx.x: the owned rows of S_k are staged in shared
// memory FE_CH at a time (S_k(ic, l) = S(c, map(l))); warp per eigenvector
// column j, lanes over l (coalesced reads of U's column j).
constexpr int FE_CH = 4;
__global__ void k_fe(int M, const Prob* __restrict__ probs, const int* __restrict__ maps,
                     const int64_t* __restrict__ own_off, const int* __restrict__ own_cols,
                     const int* __restrict__ ipos, int64_t n, const double* __restrict__ S,
                     const double* __restrict__ Ub, const double* __restrict__ w, double* __restrict__ e_out,
                     double* __restrict__ fe_out) {
    extern __shared__ double sm[];
    double* srow = sm;                 // FE_CH x M
    double* fes = sm + FE_CH * M;      // M
    const Prob p = probs[blockIdx.x];
    const int* mp = maps + p.moff;
    const double* U = Ub + (int64_t)blockIdx.x * M * M;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = threadIdx.x; j < p.m; j += blockDim.x) fes[j] = 0.0;
    const int64_t o0 = own_off[p.k], o1 = own_off[p.k + 1];
    for (int64_t ob = o0; ob < o1; ob += FE_CH) {
        const int nc = (int)((o1 - ob) < FE_CH ? (o1 - ob) : FE_CH);
        __syncthreads();
        for (int t = 0; t < nc; ++t) {
            const int64_t c = own_cols[ob + t];
            for (int l = threadIdx.x; l < p.m; l += blockDim.x) srow[t * M + l] = S[c + (int64_t)mp[l] * n];
        }
        __syncthreads();
        for (int j = wp; j < p.m; j += nw) {
            const double* uj = U + (int64_t)j * M;
            double add = 0.0;
            for (int t = 0; t < nc; ++t) {
                double sdot = 0.0;
                for (int l = lane; l < p.m; l += 32) sdot += srow[t * M + l] * uj[l];
                for (int o = 16; o > 0; o >>= 1) sdot += __shfl_xor_sync(0xffffffffu, sdot, o);
                add += sdot * uj[ipos[own_cols[ob + t]]];
            }
            if (lane == 0) fes[j] += add;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < p.m; j += blockDim.x) {
        e_out[p.eoff + j] = w[(int64_t)blockIdx.x * M + j];
        fe_out[p.eoff + j] = fes[j];
    }
}

// fe for one large submatrix from T = S_k U (column-major m x m): thread per j.
__global__ void k_fe_large(int m, const double* __restrict__ T, const double* __restrict__ U,
                           const int* __restrict__ own_cols, int64_t o0, int64_t o1, const int* __restrict__ ipos,
                           const double* __restrict__ w, double* __restrict__ e_out, double* __restrict__ fe_out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        double f = 0.0;
        for (int64_t oc = o0; oc < o1; ++oc) {
            const int64_t ic = ipos[own_cols[oc]];
            f += T[ic + (int64_t)j * m] * U[ic + (int64_t)j * m];
        }
        e_out[j] = w[j];
        fe_out[j] = f;
    }
}

// Z(j, t) = occ_j U(ic_t, j) for the owned columns t of one large submatrix.
__global__ void k_occ_rows(int m, const double* __restrict__ U, const double* __restrict__ w, double mu,
                           const int* __restrict__ own_cols, int64_t o0, int64_t nown, const int* __restrict__ ipos,
                           double* __restrict__ Z) {
    for (int64_t t = blockIdx.y; t < nown; t += gridDim.y) {
        const int64_t ic = ipos[own_cols[o0 + t]];
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
            const double ev = w[j];
            const double occ = ev < mu ? 2.0 : (ev == mu ? 1.0 : 0.0);
            Z[j + t * (int64_t)m] = occ * U[ic + (int64_t)j * m];
        }
    }
}

// Scatter P_k(:, owned) (m x nown, column-major) into the packed result.
__global__ void k_scatter_cols(int m, const double* __restrict__ Pc, const int* __restrict__ mp,
                               const int* __restrict__ own_cols, int64_t o0, int64_t nown, double* __restrict__ Ppk) {
    for (int64_t t = blockIdx.y; t < nown; t += gridDim.y) {
        const int64_t c = own_cols[o0 + t];
        double* col = Ppk + c * (c + 1) / 2;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
            const int64_t gi = mp[i];
            if (gi <= c) col[gi] = Pc[i + t * (int64_t)m];
        }
    }
}

struct MuResult {
    double mu;
    double nel;
    int iters;
    int converged;
    double trace_mu[100];
    double trace_nel[100];
};

__device__ double block_sum_fixed(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// (6) the mu bisection, one block of 1024 threads, fixed summation order.
__global__ void k_mu_bisect(int64_t total, const double* __restrict__ e, const double* __restrict__ fe,
                            double nelref, double tol_mu, double tol_nel, MuResult* out) {
    __shared__ double sh[1024];
    double mua = -10.0, mub = 10.0, mu = 0.0, nel = 0.0;
    bool finaliter = false;
    int it = 0;
    for (int muiter = 1; muiter <= 100; ++muiter) {
        mu = 0.5 * (mua + mub);
        double part = 0.0;
        for (int64_t q = threadIdx.x; q < total; q += blockDim.x) {
            const double ev = e[q];
            const double occ = ev < mu ? 2.0 : (ev == mu ? 1.0 : 0.0);
            part += fe[q] * occ;
        }
        nel = block_sum_fixed(part, sh);
        if (finaliter) break;
        if (threadIdx.x == 0) {
            out->trace_mu[muiter - 1] = mu;
            out->trace_nel[muiter - 1] = nel;
        }
        it = muiter;
        if (fabs(mua - mub) < tol_mu || fabs(nel - nelref) < tol_nel) finaliter = true;
        if (!finaliter) {
            if (nel > nelref) mub = mu;
            else mua = mu;
        }
    }
    if (threadIdx.x == 0) {
        out->mu = mu;
        out->nel = nel;
        out->iters = it;
        out->converged = finaliter ? 1 : 0;
    }
}

// (7) P(map(i), c) for owned column c of problem blockIdx.x; threads over i.
__global__ void k_final(int M, const Prob* __restrict__ probs, const int* __restrict__ maps,
                        const int64_t* __restrict__ own_off, const int* __restrict__ own_cols,
                        const int* __restrict__ ipos, const double* __restrict__ Ub, const double* __restrict__ w,
                        double mu, double* __restrict__ Ppk) {
    extern __shared__ double wv[];   // occ_j U(ic, j)
    const Prob p = probs[blockIdx.x];
    const int* mp = maps + p.moff;
    const double* U = Ub + (int64_t)blockIdx.x * M * M;
    const double* ev = w + (int64_t)blockIdx.x * M;
    for (int64_t oc = own_off[p.k] + blockIdx.y; oc < own_off[p.k + 1]; oc += gridDim.y) {
        const int64_t c = own_cols[oc];
        const int ic = ipos[c];
        __syncthreads();
        for (int j = threadIdx.x; j < p.m; j += blockDim.x) {
            const double occ = ev[j] < mu ? 2.0 : (ev[j] == mu ? 1.0 : 0.0);
            wv[j] = occ * U[ic + (int64_t)j * M];
        }
        __syncthreads();
        double* col = Ppk + c * (c + 1) / 2;
        for (int i = threadIdx.x; i < p.m; i += blockDim.x) {
            const int64_t gi = mp[i];
            if (gi > c) continue;
            double s = 0.0;
            for (int j = 0; j < p.m; ++j) s += U[i + (int64_t)j * M] * wv[j];
            col[gi] = s;
        }
    }
}

// Column grouping, source/sm.f90:92-162 (mode 4 from the supplied partition,
// column order as source/sm.f90:483-496).
std::vector<std::vector<int>> group_columns(int64_t ndim, const int64_t* aoat, int64_t nat, int64_t mode,
                                            const int64_t* partition) {
    std::vector<std::vector<int>> comb;
    if (mode == PTBGPU_COLUMNS_SINGLE) {
        comb.resize(ndim);
        for (int64_t i = 0; i < ndim; ++i) comb[i] = {(int)i};
    } else if (mode == PTBGPU_COLUMNS_ATOMS) {
        comb.push_back({0});
        for (int64_t i = 1; i < ndim; ++i) {
            if (aoat[i] == aoat[i - 1]) comb.back().push_back((int)i);
            else comb.push_back({(int)i});
        }
    } else if (mode == PTBGPU_COLUMNS_FULL_MATRIX) {
        comb.resize(1);
        comb[0].resize(ndim);
        std::iota(comb[0].begin(), comb[0].end(), 0);
    } else if (mode == PTBGPU_COLUMNS_KMEANS) {
        PTB_CHECK(partition != nullptr && nat > 0, PTBGPU_EINVAL,
                  "columns mode 4 needs an atom -> cluster partition");
        int64_t nsm = 0;
        for (int64_t a = 0; a < nat; ++a) {
            PTB_CHECK(partition[a] >= 1, PTBGPU_EINVAL, "partition ids are 1-based");
            nsm = std::max(nsm, partition[a]);
        }
        std::vector<std::vector<int>> by_atom(nat + 1);
        for (int64_t j = 0; j < ndim; ++j) {
            PTB_CHECK(aoat[j] >= 1 && aoat[j] <= nat, PTBGPU_EINVAL, "aoat out of range");
            by_atom[aoat[j]].push_back((int)j);
        }
        comb.resize(nsm);
        for (int64_t k = 1; k <= nsm; ++k)
            for (int64_t a = 1; a <= nat; ++a)
                if (partition[a - 1] == k) comb[k - 1].insert(comb[k - 1].end(), by_atom[a].begin(), by_atom[a].end());
        comb.erase(std::remove_if(comb.begin(), comb.end(), [](const std::vector<int>& v) { return v.empty(); }),
                   comb.end());
    } else {
        fail(PTBGPU_ENOTIMPL, "not implemented");
    }
    return comb;
}

// ---- deterministic k-means partition (columns mode 4) ---------------------
// source/sm.f90:127-154,459-514 with source/kmpp.f.  The reference draws from
// the Fortran global generator inside an OpenMP loop, so its partition is not
// reproducible; here every cluster count k gets its own splitmix64 stream
// (seed ^ k * const), so the result depends on the seed only.

// splitmix64 (Vigna): add the golden gamma, two xor-shift-multiply rounds.
struct SplitMix64 {
    uint64_t s;
    double uniform() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1.0p-53;
    }
};

// k-means++ seeding and Lloyd iterations on the atom positions (xyz(3, n)),
// as source/kmpp.f:24-178: first centre at int(u n), the others with
// probability proportional to the squared distance to the nearest chosen
// centre, nearest centre with ties to the lower index, centres = sum * (1/count).
// Returns 0-based labels, or an empty vector when a cluster empties.
std::vector<int> kmeans_pp(const double* xyz, int64_t n, int k, uint64_t seed) {
    SplitMix64 rng{seed ^ ((uint64_t)k * 0xD1B54A32D192ED03ull)};
    const double big = 1e33;
    auto d2 = [&](int64_t i, const double* c) {
        const double a = xyz[3 * i] - c[0], b = xyz[3 * i + 1] - c[1], e = xyz[3 * i + 2] - c[2];
        return a * a + b * b + e * e;
    };
    std::vector<double> work(n, big), C(3 * (size_t)k);
    int64_t i1 = std::min<int64_t>((int64_t)(rng.uniform() * (double)n), n - 1);
    for (int j = 0; j < 3; ++j) C[j] = xyz[3 * i1 + j];
    for (int l = 1; l < k; ++l) {
        double tot = 0.0;
        const double* c = &C[3 * (l - 1)];
        for (int64_t i = 0; i < n; ++i) {
            const double d = d2(i, c);
            if (d < work[i]) work[i] = d;
            tot += work[i];
        }
        const double w = rng.uniform() * tot;
        double acc = 0.0;
        i1 = n - 1;
        for (int64_t i = 0; i < n; ++i) {
            acc += work[i];
            if (acc > w) {
                i1 = i;
                break;
            }
        }
        for (int j = 0; j < 3; ++j) C[3 * l + j] = xyz[3 * i1 + j];
    }
    std::vector<int> z(n, -1);
    for (int it = 0; it < 1000; ++it) {
        bool change = false;
        for (int64_t i = 0; i < n; ++i) {
            double best = big;
            int l1 = 0;
            for (int l = 0; l < k; ++l) {
                const double d = d2(i, &C[3 * l]);
                if (d < best) {
                    best = d;
                    l1 = l;
                }
            }
            if (z[i] != l1) {
                z[i] = l1;
                change = true;
            }
        }
        if (!change) break;
        std::vector<int64_t> cnt(k, 0);
        std::vector<double> sum(3 * (size_t)k, 0.0);
        for (int64_t i = 0; i < n; ++i) {
            ++cnt[z[i]];
            for (int j = 0; j < 3; ++j) sum[3 * z[i] + j] += xyz[3 * i + j];
        }
        for (int l = 0; l < k; ++l) {
            if (cnt[l] == 0) return {};
            const double w = 1.0 / (double)cnt[l];
            for (int j = 0; j < 3; ++j) C[3 * l + j] = sum[3 * l + j] * w;
        }
    }
    return z;
}

// sum_k m_k^2.5 with m_k the rows coupled to a column of cluster k
// (source/sm.f90:498-512); rows[i] lists the atoms coupled to row i; k <= 64.
double kmeans_effort(const std::vector<std::vector<int>>& rows, const std::vector<int>& z, int k) {
    std::vector<int64_t> m(k, 0);
    for (const auto& r : rows) {
        uint64_t mask = 0;
        for (int a : r) mask |= 1ull << z[a];
        for (int l = 0; l < k; ++l)
            if (mask >> l & 1ull) ++m[l];
    }
    double e = 0.0;
    for (int l = 0; l < k; ++l) {
        const double v = (double)m[l];
        e += v * v * std::sqrt(v);
    }
    return e;
}

}  // namespace

// Mode-4 partition: k-means for 1..min(64, nat) clusters, the least
// sum m_k^2.5 wins (ties: fewer clusters).  dH, dS: full column-major FP64.
// The per-atom coupling pattern comes from the device pattern scan; the
// candidates run on host threads, each with its own generator stream.
std::vector<int64_t> kmeans_partition(ptbgpu_ctx* c, int64_t n, const double* dH, const double* dS, int64_t nat,
                                      const double* xyz, const int64_t* aoat, uint64_t seed, int* nsm_out,
                                      double* effort_out) {
    PTB_CHECK(nat > 0 && xyz && aoat, PTBGPU_EINVAL, "k-means partition needs nat, xyz and aoat");
    cudaStream_t s = c->stream;
    std::vector<int> owner(n);
    for (int64_t j = 0; j < n; ++j) {
        PTB_CHECK(aoat[j] >= 1 && aoat[j] <= nat, PTBGPU_EINVAL, "aoat out of range");
        owner[j] = (int)(aoat[j] - 1);
    }
    DevBuf& bo = c->buf(B_SM0);
    bo.reserve(sizeof(int) * n);
    PTB_CUDA(cudaMemcpyAsync(bo.ptr, owner.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    DevBuf& bf = c->buf(B_SM3);
    bf.reserve((size_t)nat * n);
    PTB_CUDA(cudaMemsetAsync(bf.ptr, 0, (size_t)nat * n, s));
    k_pattern<<<(int)std::min<int64_t>(n, 148 * 8), 256, 0, s>>>(n, dH, dS, bo.as<int>(), bf.as<uint8_t>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    std::vector<uint8_t> flags((size_t)nat * n);
    PTB_CUDA(cudaMemcpyAsync(flags.data(), bf.ptr, flags.size(), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    std::vector<std::vector<int>> rows(n);
    for (int64_t a = 0; a < nat; ++a)
        for (int64_t i = 0; i < n; ++i)
            if (flags[a * n + i]) rows[i].push_back((int)a);
    const int kmax = (int)std::min<int64_t>(64, nat);
    std::vector<std::vector<int>> labels(kmax + 1);
    std::vector<double> effort(kmax + 1, HUGE_VAL);
    std::atomic<int> next{1};
    auto work = [&] {
        for (int k = next++; k <= kmax; k = next++) {
            labels[k] = kmeans_pp(xyz, nat, k, seed);
            if (!labels[k].empty()) effort[k] = kmeans_effort(rows, labels[k], k);
        }
    };
    const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    int best = 0;
    for (int k = 1; k <= kmax; ++k)
        if (effort[k] < (best ? effort[best] : HUGE_VAL)) best = k;
    PTB_CHECK(best > 0, PTBGPU_EITER, "k-means failed for every cluster count");
    if (nsm_out) *nsm_out = best;
    if (effort_out) *effort_out = effort[best];
    std::vector<int64_t> part(nat);
    for (int64_t a = 0; a < nat; ++a) part[a] = labels[best][a] + 1;
    return part;
}

namespace {

template <class T>
T* upload(ptbgpu_ctx* c, int id, const std::vector<T>& v) {
    DevBuf& b = c->buf(id);
    b.reserve(sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty())
        PTB_CUDA(cudaMemcpyAsync(b.ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c->stream));
    return b.as<T>();
}

}  // namespace

namespace {

// One size bucket of prepared submatrices (or one large submatrix).
struct Bucket {
    int M = 0, count = 0;
    bool is_large = false;
    Prob single{};
    DevBuf probs, U, w;
};

// Side streams for the large submatrices of the cuSOLVER comparison path
// (PTBGPU_SM_EIG=library; one generalized eigensolve each): cuSOLVER's dsygvd
// at these sizes is latency-bound (tridiagonalisation), so
// several run at once, each on its own stream and handles, driven by its own
// host thread.  Kept on the context between calls.
struct SidePool {
    static constexpr int kStreams = 8;
    int device = 0;
    cudaStream_t st[kStreams] = {};
    cusolverDnHandle_t sol[kStreams] = {};
    cublasHandle_t blas[kStreams] = {};
    cudaEvent_t done[kStreams] = {};
    DevBuf ws[kStreams], sk[kStreams], tb[kStreams];
    ~SidePool() {
        for (int i = 0; i < kStreams; ++i) {
            if (st[i]) cudaStreamSynchronize(st[i]);
            ws[i].release();
            sk[i].release();
            tb[i].release();
            if (sol[i]) cusolverDnDestroy(sol[i]);
            if (blas[i]) cublasDestroy(blas[i]);
            if (done[i]) cudaEventDestroy(done[i]);
            if (st[i]) cudaStreamDestroy(st[i]);
        }
    }
};

SidePool& side_pool(ptbgpu_ctx* c) {
    if (!c->sm_side) {
        auto sp = std::make_shared<SidePool>();
        sp->device = c->device;
        for (int i = 0; i < SidePool::kStreams; ++i) {
            PTB_CUDA(cudaStreamCreateWithFlags(&sp->st[i], cudaStreamNonBlocking));
            PTB_CUSOLVER(cusolverDnCreate(&sp->sol[i]));
            PTB_CUSOLVER(cusolverDnSetStream(sp->sol[i], sp->st[i]));
            PTB_CUBLAS(cublasCreate(&sp->blas[i]));
            PTB_CUBLAS(cublasSetStream(sp->blas[i], sp->st[i]));
            PTB_CUDA(cudaEventCreateWithFlags(&sp->done[i], cudaEventDisableTiming));
        }
        c->sm_side = sp;
    }
    return *static_cast<SidePool*>(c->sm_side.get());
}

// __global__ helper: nel(mu) = sum fe_q occ(e_q, mu) over the prepared
// eigenpairs, one block of 1024 threads with the same partition and reduction
// order as k_mu_bisect (so a one-rank host bisection reproduces it exactly).
__global__ void k_nel_at(int64_t total, const double* __restrict__ e, const double* __restrict__ fe, double mu,
                         double* __restrict__ out) {
    __shared__ double sh[1024];
    double part = 0.0;
    for (int64_t q = threadIdx.x; q < total; q += blockDim.x) {
        const double ev = e[q];
        const double occ = ev < mu ? 2.0 : (ev == mu ? 1.0 : 0.0);
        part += fe[q] * occ;
    }
    const double nel = block_sum_fixed(part, sh);
    if (threadIdx.x == 0) *out = nel;
}

}  // namespace

// The submatrix method between its phases.  Device data lives in context
// buffers (filtered H and S in B_H / B_S, owners, owned columns, map offsets,
// maps and row positions in B_SM0..B_SM7, eigenvalues and fe weights of the
// prepared submatrices in B_MISC0 / B_MISC1) and in the buckets below.
struct SmPlan {
    int64_t n = 0;
    int nsm = 0;
    int prl = 0;
    std::vector<int64_t> own_off;
    std::vector<int> counts;
    std::vector<int64_t> moff;
    std::vector<Bucket> bks;
    int64_t total = 0;     // prepared eigenpairs
    double flops = 0.0;
    bool prepared = false;
    std::shared_ptr<EigBatch> eig;   // submatrices of the batched eigensolver
    ~SmPlan() {
        for (Bucket& bk : bks) {
            bk.probs.release();
            bk.U.release();
            bk.w.release();
        }
    }
};

namespace {

// ---- size-bucket schedule of the cuSOLVER comparison path ------------------
// The batched cuSOLVER eigensolver (PTBGPU_SM_EIG=library) costs about L(M) + p(M) B for B problems
// padded to M (a launch/latency term that does not shrink with B, and a
// per-problem term): fine buckets of a few problems each pay L many times.
// The cost model is measured once per device and padded size (random symmetric
// test matrices, B = 1 and B = 16), and the problems, sorted by size, are cut
// into contiguous buckets by dynamic programming on the modelled cost.
struct EigCost {
    double L = 0.0, p = 0.0;   // ms
};

__global__ void k_fill_test(int M, int B, double* __restrict__ A) {
    const int64_t total = (int64_t)B * M * M;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / ((int64_t)M * M), r = t % ((int64_t)M * M);
        const int64_t i = r % M, j = r / M;
        const uint64_t lo = (uint64_t)(i < j ? i : j), hi = (uint64_t)(i < j ? j : i);
        uint64_t h = (lo * 0x9E3779B97F4A7C15ull) ^ (hi * 0xC2B2AE3D27D4EB4Full) ^ ((uint64_t)b * 0x165667B19E3779F9ull);
        h ^= h >> 31;
        h *= 0xD6E8FEB86659FD93ull;
        h ^= h >> 32;
        A[t] = (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5 + (i == j ? 2.0 : 0.0);
    }
}

std::mutex g_eig_mu;
std::map<std::pair<int, int>, EigCost> g_eig_cost;

// Measured cost of the batched eigensolver at padded size M (cached per device).
// Returns false when the batched routine is unavailable at this size.
bool eig_cost(ptbgpu_ctx* c, cusolverDnParams_t params, int M, EigCost* out) {
    std::lock_guard<std::mutex> lock(g_eig_mu);
    const auto key = std::make_pair(c->device, M);
    auto it = g_eig_cost.find(key);
    if (it != g_eig_cost.end()) {
        *out = it->second;
        return true;
    }
    constexpr int Bt = 16;
    cudaStream_t s = c->stream;
    DevBuf a, w, ws, info;
    a.reserve(sizeof(double) * (size_t)Bt * M * M);
    w.reserve(sizeof(double) * (size_t)Bt * M);
    info.reserve(sizeof(int) * Bt);
    size_t wsd = 0, wsh = 0;
    if (cusolverDnXsyevBatched_bufferSize(c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, M,
                                          CUDA_R_64F, a.ptr, M, CUDA_R_64F, w.ptr, CUDA_R_64F, &wsd, &wsh, Bt) !=
        CUSOLVER_STATUS_SUCCESS)
        return false;
    ws.reserve(std::max<size_t>(wsd, 16));
    std::vector<char> hws(std::max<size_t>(wsh, 16));
    cudaEvent_t e0 = c->take_event(), e1 = c->take_event();
    auto run = [&](int B) -> float {
        k_fill_test<<<592, 256, 0, s>>>(M, B, a.as<double>());
        PTB_CUDA(cudaGetLastError());
        PTB_CUDA(cudaEventRecord(e0, s));
        PTB_CUSOLVER(cusolverDnXsyevBatched(c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, M,
                                            CUDA_R_64F, a.ptr, M, CUDA_R_64F, w.ptr, CUDA_R_64F, ws.ptr, wsd,
                                            hws.data(), wsh, info.as<int>(), B));
        PTB_CUDA(cudaEventRecord(e1, s));
        PTB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PTB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms;
    };
    run(1);   // first call of this size: one-time setup inside the library
    const float t1 = std::min(run(1), run(1));
    const float tb = run(Bt);
    EigCost ec;
    ec.p = std::max(0.0, (double)(tb - t1) / (Bt - 1));
    ec.L = std::max(0.0, (double)t1 - ec.p);
    g_eig_cost[key] = ec;
    *out = ec;
    return true;
}

// Contiguous buckets of the problems sorted by size, padded to multiples of 32,
// with the least modelled cost.  Returns (padded size, problems) per bucket.
std::vector<std::pair<int, std::vector<Prob>>> tuned_buckets(ptbgpu_ctx* c, cusolverDnParams_t params,
                                                             std::vector<Prob> probs, int prl) {
    std::vector<std::pair<int, std::vector<Prob>>> out;
    if (probs.empty()) return out;
    std::stable_sort(probs.begin(), probs.end(), [](const Prob& a, const Prob& b) { return a.m < b.m; });
    const int P = (int)probs.size();
    std::map<int, EigCost> cost;
    for (const Prob& p : probs) {
        const int M = (int)round_up(p.m, 32);
        if (cost.count(M)) continue;
        EigCost ec;
        if (!eig_cost(c, params, M, &ec)) {   // no batched routine: fine buckets
            std::map<int, std::vector<Prob>> fine;
            for (const Prob& q : probs) fine[(int)round_up(q.m, 32)].push_back(q);
            for (auto& kv : fine) out.push_back({kv.first, kv.second});
            return out;
        }
        cost[M] = ec;
    }
    std::vector<double> best(P + 1, 0.0);
    std::vector<int> from(P + 1, 0);
    for (int j = 1; j <= P; ++j) {
        const int M = (int)round_up(probs[j - 1].m, 32);
        const EigCost& ec = cost[M];
        best[j] = INFINITY;
        for (int i = 1; i <= j; ++i) {
            const double v = best[i - 1] + ec.L + ec.p * (double)(j - i + 1);
            if (v < best[j]) {
                best[j] = v;
                from[j] = i;
            }
        }
    }
    for (int j = P; j > 0; j = from[j] - 1) {
        const int i = from[j];
        out.push_back({(int)round_up(probs[j - 1].m, 32), std::vector<Prob>(probs.begin() + (i - 1), probs.begin() + j)});
    }
    std::reverse(out.begin(), out.end());
    if (prl >= 2) {
        std::string line;
        char buf[64];
        for (const auto& b : out) {
            snprintf(buf, sizeof(buf), " %dx%zu", b.first, b.second.size());
            line += buf;
        }
        log_line(prl, 2, " * submatrix bucket schedule (M x problems):%s  modelled %.1f ms", line.c_str(), best[P]);
    }
    return out;
}

SmPlan& plan_of(ptbgpu_ctx* c) {
    PTB_CHECK(c->sm_plan != nullptr, PTBGPU_EINVAL, "no submatrix plan on this context (call the plan phase first)");
    return *static_cast<SmPlan*>(c->sm_plan.get());
}

}  // namespace

// (1)-(3): filtered H and S, grouping (mode 4 without a partition runs the
// seeded k-means), pattern scan, ordered maps.  Replaces any earlier plan.
SmPlan& sm_plan(ptbgpu_ctx* c, int64_t n, const double* dH, const double* dS, int64_t nat, const double* xyz,
                const int64_t* aoat, int64_t columns, int64_t mode, const int64_t* partition, const ptbgpu_opts* o) {
    const int prl = o ? (int)o->print_level : 0;
    const double filter = o ? o->filter : 0.0;
    if (mode == PTBGPU_SUBMATRIX_SIGN) fail(PTBGPU_ENOTIMPL, "submatrix_mode.eq.1 not implemented");
    PTB_CHECK(mode == PTBGPU_SUBMATRIX_SYGV, PTBGPU_ENOTIMPL, "not implemented submatrix_mode %lld", (long long)mode);
    PTB_CHECK(n > 0 && n < (int64_t)1 << 31, PTBGPU_EINVAL, "bad ndim");
    cudaStream_t s = c->stream;
    c->sm_plan.reset();
    auto owner_plan = std::make_shared<SmPlan>();
    SmPlan& pl = *owner_plan;
    pl.n = n;
    pl.prl = prl;
    log_line(prl, 1, " Stupid simple implementation of the submatrix method: %lld %lld", (long long)columns,
             (long long)mode);

    DevBuf& bh = c->buf(B_H);
    DevBuf& bs = c->buf(B_S);
    bh.reserve(sizeof(double) * n * n);
    bs.reserve(sizeof(double) * n * n);
    double* H = bh.as<double>();
    double* S = bs.as<double>();
    unpack_sym(s, n, n, dH, H, filter);
    unpack_sym(s, n, n, dS, S, filter);

    std::vector<int64_t> own_part;
    if (columns == PTBGPU_COLUMNS_KMEANS && partition == nullptr) {
        int k = 0;
        double eff = 0.0;
        own_part = kmeans_partition(c, n, H, S, nat, xyz, aoat, kKmeansSeed, &k, &eff);
        partition = own_part.data();
        log_line(prl, 1, " k-means partition: %d clusters, effort %.6e", k, eff);
    }
    std::vector<std::vector<int>> comb = group_columns(n, aoat, nat, columns, partition);
    const int nsm = (int)comb.size();
    pl.nsm = nsm;
    std::vector<int> owner(n, -1), own_cols;
    pl.own_off.assign(nsm + 1, 0);
    for (int k = 0; k < nsm; ++k) {
        pl.own_off[k + 1] = pl.own_off[k] + (int64_t)comb[k].size();
        for (int col : comb[k]) {
            owner[col] = k;
            own_cols.push_back(col);
        }
    }
    int* d_owner = upload(c, B_SM0, owner);
    upload(c, B_SM1, own_cols);
    upload(c, B_SM2, pl.own_off);

    DevBuf& bf = c->buf(B_SM3);
    bf.reserve((size_t)nsm * n);
    PTB_CUDA(cudaMemsetAsync(bf.ptr, 0, (size_t)nsm * n, s));
    k_pattern<<<(int)std::min<int64_t>(n, 148 * 8), 256, 0, s>>>(n, H, S, d_owner, bf.as<uint8_t>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    DevBuf& bc = c->buf(B_SM4);
    bc.reserve(sizeof(int) * nsm);
    k_count<<<nsm, 256, 0, s>>>(n, bf.as<uint8_t>(), bc.as<int>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    pl.counts.resize(nsm);
    PTB_CUDA(cudaMemcpyAsync(pl.counts.data(), bc.ptr, sizeof(int) * nsm, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    pl.moff.assign(nsm + 1, 0);
    for (int k = 0; k < nsm; ++k) pl.moff[k + 1] = pl.moff[k] + pl.counts[k];
    int64_t* d_moff = upload(c, B_SM5, pl.moff);
    DevBuf& bm = c->buf(B_SM6);
    bm.reserve(sizeof(int) * std::max<int64_t>(pl.moff[nsm], 1));
    DevBuf& bip = c->buf(B_SM7);
    bip.reserve(sizeof(int) * n);
    k_fill<<<nsm, 256, 0, s>>>(n, bf.as<uint8_t>(), d_moff, d_owner, bm.as<int>(), bip.as<int>());
    count_launch();
    PTB_CUDA(cudaGetLastError());

    const int64_t sumdims = pl.moff[nsm];
    double effort_full = std::pow((double)n, 2.5), effort_sms = 0.0;
    for (int k = 0; k < nsm; ++k) effort_sms += std::pow((double)pl.counts[k], 2.5);
    log_line(prl, 1, " number of submatrices= %d", nsm);
    log_line(prl, 1, " average sm dim= %lld", (long long)(sumdims / nsm));
    log_line(prl, 1, " effort for full matrix ops= %g", effort_full);
    log_line(prl, 1, " sums of efforts for submatrices= %g", effort_sms);
    log_line(prl, 1, " ratio %g", effort_sms / effort_full);
    c->sm_plan = owner_plan;
    return pl;
}

// (4)-(5): gather, reduction, eigensolve and fe weights of the listed
// submatrices (0-based, each at most once), by the library's eigensolver
// (sm_eig.cu) or, with PTBGPU_SM_EIG=library, in buckets of padded size <= 1024
// through the batched cuSOLVER / cuBLAS calls and one dsygvd per larger one.
// Their eigenpairs replace any earlier prepared set.
void sm_prepare(ptbgpu_ctx* c, SmPlan& pl, const std::vector<int>& ids) {
    cudaStream_t s = c->stream;
    const int prl = pl.prl;
    const int64_t n = pl.n;
    for (Bucket& bk : pl.bks) {
        bk.probs.release();
        bk.U.release();
        bk.w.release();
    }
    pl.bks.clear();
    pl.eig.reset();
    pl.prepared = false;
    pl.flops = 0.0;
    std::vector<char> seen(pl.nsm, 0);
    for (int k : ids) {
        PTB_CHECK(k >= 0 && k < pl.nsm && !seen[k], PTBGPU_EINVAL, "bad or repeated submatrix index %d", k);
        seen[k] = 1;
    }
    const double* H = c->buf(B_H).as<double>();
    const double* S = c->buf(B_S).as<double>();
    const int* d_own_cols = c->buf(B_SM1).as<int>();
    const int64_t* d_own_off = c->buf(B_SM2).as<int64_t>();
    const int* d_maps = c->buf(B_SM6).as<int>();
    const int* d_ipos = c->buf(B_SM7).as<int>();
    auto t_last = std::chrono::steady_clock::now();
    auto mark = [&](const char* what) {
        if (prl < 2) return;
        PTB_CUDA(cudaStreamSynchronize(s));
        auto now = std::chrono::steady_clock::now();
        log_line(prl, 2, " * submatrix %-28s %10.3f ms", what,
                 std::chrono::duration<double, std::milli>(now - t_last).count());
        t_last = now;
    };

    constexpr int kBatchMax = kEigBatchMax;
    std::vector<Prob> small, large;
    int64_t eoff = 0;
    for (int k : ids) {
        Prob p{k, pl.counts[k], pl.moff[k], eoff};
        eoff += pl.counts[k];
        if (pl.counts[k] > kBatchMax) large.push_back(p);
        else small.push_back(p);
    }
    pl.total = eoff;
    DevBuf& be = c->buf(B_MISC0);
    DevBuf& bfe = c->buf(B_MISC1);
    be.reserve(sizeof(double) * std::max<int64_t>(eoff, 1));
    bfe.reserve(sizeof(double) * std::max<int64_t>(eoff, 1));
    // every submatrix through the library's eigensolver: up to kEigBatchMax one
    // CTA each in a persistent launch, above it one thread-block cluster each;
    // PTBGPU_SM_EIG=library sends them through cuSOLVER instead (batched routines
    // in tuned size buckets, dsygvd above kEigBatchMax; kept for comparison)
    static const bool use_library = [] {
        const char* v = getenv("PTBGPU_SM_EIG");
        return v != nullptr && std::string(v) == "library";
    }();
    // launched on the context's stream after the side streams' start event, so
    // that it runs while the large submatrices are solved on the side streams
    std::vector<EigProbHost> own_probs;
    if (!use_library) {
        own_probs.reserve(small.size() + large.size());
        for (const Prob& p : small)
            own_probs.push_back(
                {p.k, p.m, (int)(pl.own_off[p.k + 1] - pl.own_off[p.k]), p.moff, p.eoff, pl.own_off[p.k]});
        small.clear();
        // above kEigBatchMax: one thread-block cluster per submatrix, up to kEigLargeMax
        std::vector<Prob> rest;
        for (const Prob& p : large) {
            if (p.m <= kEigLargeMax)
                own_probs.push_back(
                    {p.k, p.m, (int)(pl.own_off[p.k + 1] - pl.own_off[p.k]), p.moff, p.eoff, pl.own_off[p.k]});
            else
                rest.push_back(p);
        }
        large.swap(rest);
    }
    auto launch_own = [&] {
        if (own_probs.empty() || pl.eig) return;
        pl.eig = eig_batch_launch(c, n, H, S, own_probs, d_maps, d_own_cols, d_ipos, be.as<double>(),
                                  bfe.as<double>(), prl, &pl.flops);
        log_line(prl, 2, " * submatrix batched eigensolver: %zu problems launched", own_probs.size());
    };
    DevBuf sb, ptrs, infos, ws, tbuf;
    cusolverDnParams_t params;
    PTB_CUSOLVER(cusolverDnCreateParams(&params));
    std::vector<std::pair<int, std::vector<Prob>>> buckets;
    try {
        buckets = tuned_buckets(c, params, small, prl);
    } catch (...) {
        cusolverDnDestroyParams(params);
        throw;
    }
    pl.bks.resize(buckets.size() + large.size());
    auto cleanup = [&] {
        cusolverDnDestroyParams(params);
        sb.release();
        ptrs.release();
        infos.release();
        ws.release();
        tbuf.release();
    };
    static const bool fe_attr = [] {   // thread-safe one-time setup
        PTB_CUDA(cudaFuncSetAttribute(k_fe, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        PTB_CUDA(cudaFuncSetAttribute(k_final, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        return true;
    }();
    (void)fe_attr;
    const double one = 1.0, zero = 0.0;
    try {
        size_t bi = 0;
        for (auto& kv : buckets) {
            const int M = kv.first;
            std::vector<Prob>& pv = kv.second;
            const int B = (int)pv.size();
            Bucket& bk = pl.bks[bi++];
            bk.M = M;
            bk.count = B;
            bk.probs.reserve(sizeof(Prob) * B);
            PTB_CUDA(cudaMemcpyAsync(bk.probs.ptr, pv.data(), sizeof(Prob) * B, cudaMemcpyHostToDevice, s));
            bk.U.reserve(sizeof(double) * (size_t)B * M * M);
            bk.w.reserve(sizeof(double) * (size_t)B * M);
            sb.reserve(sizeof(double) * (size_t)B * M * M);
            double* Hb = bk.U.as<double>();
            double* Sb = sb.as<double>();
            dim3 gg((M + 31) / 32, (unsigned)std::max(1, std::min(M / 8, 64)), B);
            k_gather<<<gg, dim3(32, 8), 0, s>>>(M, bk.probs.as<Prob>(), d_maps, n, H, S, Hb, Sb);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            std::vector<double*> hp(2 * (size_t)B);
            for (int q = 0; q < B; ++q) {
                hp[q] = Sb + (size_t)q * M * M;
                hp[B + q] = Hb + (size_t)q * M * M;
            }
            ptrs.reserve(sizeof(double*) * hp.size());
            PTB_CUDA(cudaMemcpyAsync(ptrs.ptr, hp.data(), sizeof(double*) * hp.size(), cudaMemcpyHostToDevice, s));
            infos.reserve(sizeof(int) * B);
            double** dS_arr = ptrs.as<double*>();
            double** dH_arr = dS_arr + B;
            PTB_CUSOLVER(cusolverDnDpotrfBatched(c->solver, CUBLAS_FILL_MODE_LOWER, M, dS_arr, M, infos.as<int>(), B));
            std::vector<int> hinfo(B);
            PTB_CUDA(cudaMemcpyAsync(hinfo.data(), infos.ptr, sizeof(int) * B, cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            for (int q = 0; q < B; ++q)
                PTB_CHECK(hinfo[q] == 0, PTBGPU_ENOTSPD, "overlap submatrix %d not positive definite (info=%d)",
                          pv[q].k + 1, hinfo[q]);
            PTB_CUBLAS(cublasDtrsmBatched(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                                          CUBLAS_DIAG_NON_UNIT, M, M, &one, dS_arr, M, dH_arr, M, B));
            PTB_CUBLAS(cublasDtrsmBatched(c->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                                          CUBLAS_DIAG_NON_UNIT, M, M, &one, dS_arr, M, dH_arr, M, B));
            size_t wsd = 0, wsh = 0;
            cusolverStatus_t bst = cusolverDnXsyevBatched_bufferSize(
                c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, M, CUDA_R_64F, Hb, M,
                CUDA_R_64F, bk.w.ptr, CUDA_R_64F, &wsd, &wsh, B);
            if (bst == CUSOLVER_STATUS_SUCCESS) {
                ws.reserve(std::max<size_t>(wsd, 16));
                std::vector<char> hws(std::max<size_t>(wsh, 16));
                mark("reduction (potrf, 2 trsm)");
                bst = cusolverDnXsyevBatched(c->solver, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, M,
                                             CUDA_R_64F, Hb, M, CUDA_R_64F, bk.w.ptr, CUDA_R_64F, ws.ptr, wsd,
                                             hws.data(), wsh, infos.as<int>(), B);
                PTB_CUDA(cudaStreamSynchronize(s));
                mark("batched eigensolve");
            }
            if (bst != CUSOLVER_STATUS_SUCCESS) {
                // per-matrix eigensolves of the reduced problems (same layout)
                for (int q = 0; q < B; ++q) {
                    dsyevd(c, M, M, Hb + (size_t)q * M * M, bk.w.as<double>() + (size_t)q * M);
                }
                PTB_CUDA(cudaMemsetAsync(infos.ptr, 0, sizeof(int) * B, s));
            }
            PTB_CUDA(cudaMemcpyAsync(hinfo.data(), infos.ptr, sizeof(int) * B, cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            for (int q = 0; q < B; ++q)
                PTB_CHECK(hinfo[q] == 0, PTBGPU_EITER, "eigensolver failed on submatrix %d (info=%d)", pv[q].k + 1,
                          hinfo[q]);
            PTB_CUBLAS(cublasDtrsmBatched(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                                          CUBLAS_DIAG_NON_UNIT, M, M, &one, dS_arr, M, dH_arr, M, B));
            k_fe<<<B, 256, sizeof(double) * (FE_CH + 1) * M, s>>>(M, bk.probs.as<Prob>(), d_maps, d_own_off,
                                                                  d_own_cols, d_ipos, n, S, Hb, bk.w.as<double>(),
                                                                  be.as<double>(), bfe.as<double>());
            count_launch();
            PTB_CUDA(cudaGetLastError());
            mark("back-transform and fe");
            for (const Prob& p : pv) pl.flops += 9.0 * std::pow((double)p.m, 3);
            log_line(prl, 2, " * submatrix bucket M=%d: %d problems", M, B);
        }
        // large submatrices: one generalized eigensolve each (dsygvd), fe from T = S_k U,
        // spread over the side streams (largest first), each driven by its own host thread
        if (!large.empty()) {
            SidePool& sp = side_pool(c);
            std::vector<size_t> order(large.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return large[a].m > large[b].m; });
            std::vector<Bucket*> lb(large.size());
            for (size_t q = 0; q < large.size(); ++q) {
                const Prob& p = large[q];
                Bucket& bk = pl.bks[bi++];
                bk.is_large = true;
                bk.single = p;
                bk.M = p.m;
                bk.count = 1;
                bk.probs.reserve(sizeof(Prob));
                PTB_CUDA(cudaMemcpyAsync(bk.probs.ptr, &p, sizeof(Prob), cudaMemcpyHostToDevice, s));
                bk.U.reserve(sizeof(double) * (size_t)p.m * p.m);
                bk.w.reserve(sizeof(double) * (size_t)p.m);
                lb[q] = &bk;
                pl.flops += 9.0 * std::pow((double)p.m, 3);
            }
            infos.reserve(sizeof(int) * large.size());
            PTB_CUDA(cudaMemsetAsync(infos.ptr, 0, sizeof(int) * large.size(), s));
            cudaEvent_t ready = c->take_event();
            PTB_CUDA(cudaEventRecord(ready, s));
            launch_own();
            const int nw = (int)std::min<size_t>(SidePool::kStreams, large.size());
            std::atomic<size_t> next{0};
            std::vector<std::string> errs(nw);
            std::vector<int64_t> launches(nw, 0);
            auto work = [&](int w) {
                try {
                    PTB_CUDA(cudaSetDevice(c->device));
                    cudaStream_t st = sp.st[w];
                    PTB_CUDA(cudaStreamWaitEvent(st, ready, 0));
                    for (size_t t = next++; t < order.size(); t = next++) {
                        const size_t q = order[t];
                        const Prob& p = large[q];
                        Bucket& bk = *lb[q];
                        const int m = p.m;
                        sp.sk[w].reserve(sizeof(double) * (size_t)m * m);
                        sp.tb[w].reserve(sizeof(double) * (size_t)m * m);
                        double* U = bk.U.as<double>();
                        double* Sk = sp.sk[w].as<double>();
                        double* T = sp.tb[w].as<double>();
                        dim3 gg((m + 31) / 32, 64, 1);
                        k_gather<<<gg, dim3(32, 8), 0, st>>>(m, bk.probs.as<Prob>(), d_maps, n, H, S, U, Sk);
                        PTB_CUDA(cudaGetLastError());
                        int lwork = 0;
                        PTB_CUSOLVER(cusolverDnDsygvd_bufferSize(sp.sol[w], CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                                 CUBLAS_FILL_MODE_UPPER, m, U, m, Sk, m,
                                                                 bk.w.as<double>(), &lwork));
                        sp.ws[w].reserve(sizeof(double) * (size_t)std::max(lwork, 1));
                        PTB_CUSOLVER(cusolverDnDsygvd(sp.sol[w], CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                      CUBLAS_FILL_MODE_UPPER, m, U, m, Sk, m, bk.w.as<double>(),
                                                      sp.ws[w].as<double>(), lwork, infos.as<int>() + q));
                        k_gather<<<gg, dim3(32, 8), 0, st>>>(m, bk.probs.as<Prob>(), d_maps, n, H, S, T, Sk);
                        PTB_CUDA(cudaGetLastError());
                        PTB_CUBLAS(cublasDgemm(sp.blas[w], CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, &one, Sk, m, U, m,
                                               &zero, T, m));
                        k_fe_large<<<(m + 255) / 256, 256, 0, st>>>(m, T, U, d_own_cols, pl.own_off[p.k],
                                                                   pl.own_off[p.k + 1], d_ipos, bk.w.as<double>(),
                                                                   be.as<double>() + p.eoff,
                                                                   bfe.as<double>() + p.eoff);
                        PTB_CUDA(cudaGetLastError());
                        launches[w] += 3;
                    }
                    PTB_CUDA(cudaEventRecord(sp.done[w], st));
                } catch (const Error& e) {
                    errs[w] = e.msg;
                } catch (const std::exception& e) {
                    errs[w] = e.what();
                }
            };
            std::vector<std::thread> pool;
            for (int w = 0; w < nw; ++w) pool.emplace_back(work, w);
            for (auto& t : pool) t.join();
            for (int w = 0; w < nw; ++w)
                if (!errs[w].empty()) {
                    // let every side stream drain before the shared buffers can be released
                    for (int v = 0; v < nw; ++v) cudaStreamSynchronize(sp.st[v]);
                    fail(PTBGPU_ECUDA, "large submatrix eigensolve: %s", errs[w].c_str());
                }
            for (int w = 0; w < nw; ++w) {
                PTB_CUDA(cudaStreamWaitEvent(s, sp.done[w], 0));
                count_launch((int)launches[w]);
            }
            std::vector<int> hinfo(large.size());
            PTB_CUDA(cudaMemcpyAsync(hinfo.data(), infos.ptr, sizeof(int) * hinfo.size(), cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            for (size_t q = 0; q < large.size(); ++q)
                PTB_CHECK(hinfo[q] == 0, PTBGPU_ENOTSPD, "dsygvd failed on submatrix %d (info=%d)", large[q].k + 1,
                          hinfo[q]);
            mark("large eigensolves (side streams)");
        }
        launch_own();   // no large submatrices
        if (pl.eig) {
            eig_batch_check(c, *pl.eig);
            mark("batched eigensolver");
        }
        PTB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
    pl.prepared = true;
}

// Electron count of the prepared submatrices at mu (the rank-local term of the
// bisection in source/sm.f90:322-340).
double sm_nel(ptbgpu_ctx* c, SmPlan& pl, double mu) {
    PTB_CHECK(pl.prepared, PTBGPU_EINVAL, "submatrices not prepared");
    cudaStream_t s = c->stream;
    DevBuf& bo = c->buf(B_MISC2);
    bo.reserve(sizeof(double) * 64);
    k_nel_at<<<1, 1024, 0, s>>>(pl.total, c->buf(B_MISC0).as<double>(), c->buf(B_MISC1).as<double>(), mu,
                                bo.as<double>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    double v = 0.0;
    PTB_CUDA(cudaMemcpyAsync(&v, bo.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    return v;
}

// (7): dP := 0, then the owned columns of every prepared submatrix at mu.
void sm_finish(ptbgpu_ctx* c, SmPlan& pl, double mu, double* dP) {
    PTB_CHECK(pl.prepared, PTBGPU_EINVAL, "submatrices not prepared");
    cudaStream_t s = c->stream;
    const int64_t n = pl.n;
    const int* d_own_cols = c->buf(B_SM1).as<int>();
    const int64_t* d_own_off = c->buf(B_SM2).as<int64_t>();
    const int* d_maps = c->buf(B_SM6).as<int>();
    const int* d_ipos = c->buf(B_SM7).as<int>();
    const double one = 1.0, zero = 0.0;
    PTB_CUDA(cudaMemsetAsync(dP, 0, sizeof(double) * (size_t)npacked(n), s));
    if (pl.eig) eig_batch_final(c, *pl.eig, mu, n, d_maps, d_own_cols, dP);
    DevBuf tbuf;
    try {
        for (Bucket& bk : pl.bks) {
            if (!bk.is_large) {
                dim3 g(bk.count, 4);
                k_final<<<g, 256, sizeof(double) * bk.M, s>>>(bk.M, bk.probs.as<Prob>(), d_maps, d_own_off,
                                                             d_own_cols, d_ipos, bk.U.as<double>(), bk.w.as<double>(),
                                                             mu, dP);
                count_launch();
                PTB_CUDA(cudaGetLastError());
                continue;
            }
            const Prob& p = bk.single;
            const int m = p.m;
            const int64_t o0 = pl.own_off[p.k], nown = pl.own_off[p.k + 1] - o0;
            tbuf.reserve(sizeof(double) * (size_t)m * nown * 2);
            double* Z = tbuf.as<double>();
            double* Pc = Z + (size_t)m * nown;
            dim3 g((m + 255) / 256, (unsigned)std::min<int64_t>(nown, 65535));
            k_occ_rows<<<g, 256, 0, s>>>(m, bk.U.as<double>(), bk.w.as<double>(), mu, d_own_cols, o0, nown, d_ipos,
                                        Z);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            PTB_CUBLAS(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, m, (int)nown, m, &one, bk.U.as<double>(), m, Z,
                                   m, &zero, Pc, m));
            k_scatter_cols<<<g, 256, 0, s>>>(m, Pc, d_maps + p.moff, d_own_cols, o0, nown, dP);
            count_launch();
            PTB_CUDA(cudaGetLastError());
        }
        PTB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        tbuf.release();
        throw;
    }
    tbuf.release();
}

// The whole step on one device: plan, every submatrix, the device bisection
// (source/sm.f90:191-383), the final density.
void sm_density_device(ptbgpu_ctx* c, int64_t n, int64_t nelref, const double* dH, const double* dS, double* dP,
                       int64_t nat, const double* xyz, const int64_t* aoat, int64_t columns, int64_t mode,
                       const int64_t* partition, const ptbgpu_opts* o, ptbgpu_stats* st) {
    using clk = std::chrono::steady_clock;
    auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    const auto t0 = clk::now();
    SmPlan& pl = sm_plan(c, n, dH, dS, nat, xyz, aoat, columns, mode, partition, o);
    const auto t1 = clk::now();
    const int prl = pl.prl;
    std::vector<int> all(pl.nsm);
    std::iota(all.begin(), all.end(), 0);
    sm_prepare(c, pl, all);
    const auto t2 = clk::now();
    cudaStream_t s = c->stream;
    DevBuf bmu;
    bmu.reserve(sizeof(MuResult));
    const double tol_mu = (double)1e-3f, tol_nel = (double)1e-5f;
    k_mu_bisect<<<1, 1024, 0, s>>>(pl.total, c->buf(B_MISC0).as<double>(), c->buf(B_MISC1).as<double>(),
                                   (double)nelref, tol_mu, tol_nel, bmu.as<MuResult>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    MuResult mr;
    PTB_CUDA(cudaMemcpyAsync(&mr, bmu.ptr, sizeof(MuResult), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    bmu.release();
    for (int it = 0; it < mr.iters; ++it)
        log_line(prl, 1, " muiter %d mu %.15g %.15g of %lld", it + 1, mr.trace_mu[it], mr.trace_nel[it],
                 (long long)nelref);
    PTB_CHECK(mr.converged, PTBGPU_EITER, "chemical potential bisection did not converge");
    log_line(prl, 1, " iteration of chemical potential converged");
    const auto t3 = clk::now();
    sm_finish(c, pl, mr.mu, dP);
    PTB_CUDA(cudaStreamSynchronize(s));
    const auto t4 = clk::now();
    // the reference's closing timer block (source/sm.f90:408), its tags in its slot order
    log_timer_block(prl, "Submatrix", secs(t0, t4),
                    {{"submatrix combination", secs(t0, t1)}, {"mu iter", secs(t2, t3)},
                     {"submatrix eigendecomp", secs(t1, t2)}, {"submatrix final iter", secs(t3, t4)}});
    if (st) {
        st->mu = mr.mu;
        st->nel = mr.nel;
        st->mu_iterations = mr.iters;
        st->nsm = pl.nsm;
        st->sum_dims = pl.moff[pl.nsm];
        st->max_dim = *std::max_element(pl.counts.begin(), pl.counts.end());
        st->flops += pl.flops;
    }
}

// ---- phase entry points for the C-ABI (one rank's share of the step) -------
void sm_plan_entry(ptbgpu_ctx* c, int64_t n, const double* dH, const double* dS, int64_t nat, const double* xyz,
                   const int64_t* aoat, int64_t columns, int64_t mode, const int64_t* partition, const ptbgpu_opts* o,
                   int64_t* nsm, int64_t* dims) {
    SmPlan& pl = sm_plan(c, n, dH, dS, nat, xyz, aoat, columns, mode, partition, o);
    if (nsm) *nsm = pl.nsm;
    if (dims)
        for (int k = 0; k < pl.nsm; ++k) dims[k] = pl.counts[k];
}

void sm_prepare_entry(ptbgpu_ctx* c, int64_t nlocal, const int64_t* ids, ptbgpu_stats* st) {
    SmPlan& pl = plan_of(c);
    std::vector<int> v((size_t)nlocal);
    for (int64_t q = 0; q < nlocal; ++q) {
        PTB_CHECK(ids[q] >= 0 && ids[q] < pl.nsm, PTBGPU_EINVAL, "submatrix index %lld out of range",
                  (long long)ids[q]);
        v[q] = (int)ids[q];
    }
    sm_prepare(c, pl, v);
    if (st) {
        st->nsm = nlocal;
        int64_t sd = 0, md = 0;
        for (int k : v) {
            sd += pl.counts[k];
            md = std::max<int64_t>(md, pl.counts[k]);
        }
        st->sum_dims = sd;
        st->max_dim = md;
        st->flops += pl.flops;
    }
}

double sm_nel_entry(ptbgpu_ctx* c, double mu) { return sm_nel(c, plan_of(c), mu); }

void sm_finish_entry(ptbgpu_ctx* c, double mu, double* dP) { sm_finish(c, plan_of(c), mu, dP); }

}  // namespace ptb
