// Batched FP64 generalized eigensolver of the submatrix method (sm_eig.cu).
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"

namespace ptb {

// Largest submatrix the batched solver takes (its per-problem shared-memory
// vectors are sized for it); larger ones go to the side-stream path.
constexpr int kEigBatchMax = 1024;
// Largest submatrix the library's eigensolver takes at all: orders above
// kEigBatchMax run on a thread-block cluster each, whose tridiagonalisation
// keeps two vectors of this length in shared memory.
constexpr int kEigLargeMax = 12032;

// One submatrix as the host plan describes it.
struct EigProbHost {
    int k;          // submatrix index
    int m;          // dimension
    int nown;       // owned columns
    int64_t moff;   // offset of its row map in the maps array
    int64_t eoff;   // offset of its eigenpairs in the flat e / fe arrays
    int64_t o0;     // offset of its owned columns in the owned-column list
    int64_t gbase = 0;   // its H / S element (i, j) at gbase + map(i) + map(j) gld
    int64_t gld = -1;    // -1: the system's ndim
    int mode = 0;        // 0: eigenvalues, fe and owned rows (submatrix method); 2: density P = 2 U_occ U_occ^T
    int nocc = 0;        // mode 2: occupied (lowest) eigenvectors
};

struct EigBatch;

// Launches (on the context's stream, no host synchronisation) the gather,
// Cholesky, reduction, tridiagonalisation, divide and conquer, and the owned
// rows of U and S U with the (e, fe) pairs into d_e / d_fe at each problem's
// eoff.  Returns null for an empty list.  eig_batch_check waits for the stream
// and raises ENOTSPD (an overlap block not positive definite) or EITER (a
// leaf's QL iteration did not converge).
std::shared_ptr<EigBatch> eig_batch_launch(ptbgpu_ctx* c, int64_t n, const double* H, const double* S,
                                           const std::vector<EigProbHost>& probs, const int* d_maps,
                                           const int* d_own_cols, const int* d_ipos, double* d_e, double* d_fe,
                                           int prl, double* flops, bool join = true);
// With join = false the launch's side stream (the clusters of the problems
// above kEigBatchMax) is not waited for on the context's stream; this does it.
void eig_batch_join(ptbgpu_ctx* c, EigBatch& eb);
void eig_batch_check(ptbgpu_ctx* c, EigBatch& eb);

// The owned columns of P_k = U occ U^T at mu for every prepared problem,
// written into the packed result (rows map(i) <= c of column c), or with
// dPdense non-null as m x nown column-major blocks, one after another.
void eig_batch_final(ptbgpu_ctx* c, EigBatch& eb, double mu, int64_t n, const int* d_maps,
                     const int* d_own_cols, double* dP, double* dPdense = nullptr);

// All eigenpairs of a dense problem on the device with the same solver on the
// whole GPU (one cooperative launch): H U = S U diag(w) (S null: the standard
// problem), H and S full symmetric (n x n, ld n; only the lower triangles are
// read), w ascending, U column-major with U^T S U = I.  Orders up to
// kEigLargeMax.
void eig_full(ptbgpu_ctx* c, int64_t n, const double* H, const double* S, double* w, double* U);
// The same with LAPACK's dsyevd / dsygvd argument convention ('V', upper
// triangles read): A (and B) n x n, ld n; A is overwritten by the eigenvectors.
void eig_full_upper(ptbgpu_ctx* c, int64_t n, double* A, double* B, double* w);

// The density step of many independent systems in one launch of the
// eigensolver (ptbgpu_eig_density_batch): Hpk / Spk / Ppk host packed arrays
// per system, P_k = 2 sum_{i < nel_k/2} u_i u_i^T of H_k U = S_k U e after the
// filter; stats per system (may be null).
void eig_density_batch(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                       const double* const* Hpk, const double* const* Spk, double* const* Ppk, double filter,
                       int prl, ptbgpu_stats* st);

// Kernel-level entry of ptbgpu_sygv_batched (dense host problems).
void sygv_batched_entry(ptbgpu_ctx* c, int64_t np, const int64_t* dims, const double* H, const double* S,
                        const int64_t* nown, const int64_t* owned, double mu, double* e, double* fe, double* Pcols);

}  // namespace ptb
