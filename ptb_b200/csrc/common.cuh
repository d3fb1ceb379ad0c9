// Internal definitions shared by the CUDA translation units of libptbgpu.
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "ptbgpu.h"

namespace ptb {

// Error carried out of the internal layers to the C-ABI boundary.
struct Error {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const char* fmt, ...);

#define PTB_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            ::ptb::fail(PTBGPU_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                        cudaGetErrorString(e_));                                           \
    } while (0)

#define PTB_CUBLAS(call)                                                                   \
    do {                                                                                   \
        cublasStatus_t s_ = (call);                                                        \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                   \
            ::ptb::fail(PTBGPU_ECUDA, "%s:%d %s: cublas status %d", __FILE__, __LINE__,     \
                        #call, (int)s_);                                                   \
    } while (0)

#define PTB_CUSOLVER(call)                                                                 \
    do {                                                                                   \
        cusolverStatus_t s_ = (call);                                                      \
        if (s_ != CUSOLVER_STATUS_SUCCESS)                                                 \
            ::ptb::fail(PTBGPU_ECUDA, "%s:%d %s: cusolver status %d", __FILE__, __LINE__,   \
                        #call, (int)s_);                                                   \
    } while (0)

#define PTB_CHECK(cond, code, ...)                                                         \
    do {                                                                                   \
        if (!(cond)) ::ptb::fail(code, __VA_ARGS__);                                       \
    } while (0)

// Device buffer that grows on demand and is reused across calls.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    void reserve(size_t nbytes);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Device-side error word written by kernels whose bounded waits give up.
struct DeviceFlags {
    int timeout;      // nonzero: a bounded wait expired (value = site id)
    int nan;          // nonzero: a NaN was met
};

}  // namespace ptb

struct ptbgpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t solver = nullptr;
    cudaEvent_t ev[4] = {};
    std::string last_error;
    int num_sms = 0;
    // named scratch buffers (grown on demand, kept for the context's lifetime);
    // a fixed array so that references handed out by buf() never move
    static constexpr int kMaxBufs = 64;
    ptb::DevBuf bufs[kMaxBufs];
    ptb::DevBuf& buf(int id);
    ptb::DeviceFlags* flags = nullptr;   // device
    int* info_dev = nullptr;             // device int for LAPACK-style info
    void* pinned = nullptr;              // small pinned staging area (4 KB)
    // trace-correcting purification state (device)
    void* sp2_state = nullptr;
    // submatrix method between its phases (plan, prepare, nel, finish): kept
    // until the next plan or the context's end; its destructor frees its buffers
    std::shared_ptr<void> sm_plan;
    // side streams and handles of the submatrix method's large eigensolves
    std::shared_ptr<void> sm_side;
    // device tile lists of the int8-sliced FP64 products of the module code
    std::shared_ptr<void> oz_tile_cache;
    // worker contexts of the multi-instance batch (same device, own streams and buffers)
    std::vector<ptbgpu_ctx*> workers;
    // launches of this library's kernels since the last call started
    int64_t launches = 0;
    // timed tensor-core launches: event pairs recorded on `stream`
    std::vector<cudaEvent_t> evpool;
    size_t evused = 0;
    struct Timed {
        int kind;            // 0 SP2 product, 1 general product, 2 int8-sliced FP64 product
        cudaEvent_t a, b;
    };
    std::vector<Timed> timed;
    double oz_ops = 0.0;   // executed int8 ops of the int8-sliced products since the call started
    cudaEvent_t take_event();
};

namespace ptb {

// Scratch-buffer slots of a context (kept distinct so one call can hold several).
enum BufId {
    B_H = 0, B_S, B_A, B_L, B_W0, B_W1, B_W2, B_W3,   // FP64 n x n work
    B_PK0, B_PK1, B_PK2,                              // packed FP64
    B_XF0, B_XF1, B_X1F0, B_X1F1,                     // FP32 iterates
    B_HI0, B_LO0, B_HI1, B_LO1,                       // bf16 planes of the current iterate
    B_TRAJ,                                           // bf16 planes of the whole SP2 trajectory
    B_X1HI, B_X1LO,                                   // bf16 planes of the DMPT response
    B_STATS, B_TILES, B_SOLVER_WS, B_MISC0, B_MISC1, B_MISC2, B_MISC3,
    B_SM0, B_SM1, B_SM2, B_SM3, B_SM4, B_SM5, B_SM6, B_SM7,
    B_OZ0, B_OZ1, B_OZE0, B_OZE1, B_OZR, B_OZT, B_OZS,  // int8 slices, row exponents, scratch of the
                                                        // emulated FP64 products
    B_G0, B_G1, B_G2, B_G3, B_G4, B_G5, B_G6, B_G7, B_G8, B_G9, B_G10,   // grouped purification (released after)
    B_COUNT
};

inline int64_t npacked(int64_t n) { return n * (n + 1) / 2; }
inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Shared helpers implemented in dense_ops.cu.
void unpack_sym(cudaStream_t s, int64_t n, int64_t ld, const double* pk, double* full, double filter);
void pack_cols(cudaStream_t s, int64_t n, int64_t ld, const double* full, double* pk);
void filter_packed(cudaStream_t s, int64_t n, double* pk, double filter);
void set_identity(cudaStream_t s, int64_t n, int64_t ld, double* a, double diag);
void gershgorin_bounds(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a, double* emin, double* emax);
double trace_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a);
double dot_dev(ptbgpu_ctx* c, int64_t count, const double* a, const double* b);      // sum a_i b_i
double trace_prod_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a, const double* b);  // tr(AB) = sum a_ij b_ji
double sum_dev(ptbgpu_ctx* c, int64_t count, const double* a);
double frob_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a);
double colabs_max_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a);        // gershgorin norm
double rowabs_max_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a);        // infinity norm
bool   has_nan_dev(ptbgpu_ctx* c, int64_t count, const double* a);
// y = alpha*x + beta*y (+ gamma on the diagonal) over an n x n block with leading dim ld
void axpby_diag(cudaStream_t s, int64_t n, int64_t ld, double alpha, const double* x, double beta,
                double* y, double gamma);
void symmetrize_upper(cudaStream_t s, int64_t n, int64_t ld, double* a);   // a_ji := a_ij for i<j (row-major upper)
void copy_mat(cudaStream_t s, int64_t n, int64_t ld_src, const double* src, int64_t ld_dst, double* dst);
void d2f_split(cudaStream_t s, int64_t n, int64_t ldp, const double* x, float* xf, void* hi, void* lo);
void d2f_split3(cudaStream_t s, int64_t ldp, const float* xf, const void* hi, void* mid, void* lo);

// cuBLAS / cuSOLVER wrappers on row-major symmetric work (see dense_ops.cu)
void dgemm_nn(ptbgpu_ctx* c, int64_t n, int64_t ld, double alpha, const double* A, const double* B,
              double beta, double* C);
void dsyrk_sq(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* X, double* C);   // C = X X (X symmetric), full C
int  dpotrf_lower(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A);              // returns info
void dtrtri_lower(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A);
// Device-result forms of frob_dev / has_nan_dev (no host synchronisation): the
// Frobenius norm into a device double; a NaN sets *flag = 1.
void frob_to_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a, double* out);
void nan_flag_dev(ptbgpu_ctx* c, int64_t count, const double* a, int* flag);
void dsyevd(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A, double* w);
int  dsygvd(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A, double* B, double* w);

// FP64-class product on the int8 tensor cores (sp2.cu): C = alpha op(A) op(B),
// column-major n x n device matrices, S slices; oz_check raises ETIMEOUT if a
// product's bounded waits gave up (it synchronises the stream).
void oz_dgemm(ptbgpu_ctx* c, int64_t n, double alpha, const double* A, bool ta, const double* B, bool tb,
              double* C, int S = 8);
void oz_check(ptbgpu_ctx* c, const char* what);

// timing helpers
struct EventTimer {
    cudaEvent_t a, b;
    cudaStream_t s;
    explicit EventTimer(cudaStream_t st);
    ~EventTimer();
    void start();
    float stop_ms();
};

void log_line(int level, int want, const char* fmt, ...);
// The reference's timer block (source/timer.f90:194-215 layout: the total under
// `total_tag`, then "* tag" lines, seconds with 9 decimals), printed from print level 1.
void log_timer_block(int level, const char* total_tag, double total_s,
                     const std::vector<std::pair<const char*, double>>& items);

// Launches of this library's kernels by the calling host thread (a context is
// driven by one thread at a time); the C-ABI layer resets it per call.
int64_t& launch_counter();
inline void count_launch(int n = 1) { launch_counter() += n; }

}  // namespace ptb
