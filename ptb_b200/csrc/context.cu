// Context lifecycle, error plumbing and scratch buffers of libptbgpu.
#include <cstring>

#include "common.cuh"

namespace ptb {

[[noreturn]] void fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw Error{code, std::string(buf)};
}

void DevBuf::reserve(size_t nbytes) {
    if (nbytes <= bytes) return;
    release();
    nbytes = (nbytes + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&ptr, nbytes);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        (void)cudaGetLastError();
        fail(PTBGPU_ENOMEM, "cudaMalloc(%zu) failed: %s", nbytes, cudaGetErrorString(e));
    }
    bytes = nbytes;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

int64_t& launch_counter() {
    static thread_local int64_t n = 0;
    return n;
}

void log_line(int level, int want, const char* fmt, ...) {
    if (level < want) return;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stdout, fmt, ap);
    va_end(ap);
    fputc('\n', stdout);
    fflush(stdout);
}

void log_timer_block(int level, const char* total_tag, double total_s,
                     const std::vector<std::pair<const char*, double>>& items) {
    if (level < 1) return;
    fprintf(stdout, "\n%-40s   %15.9f sec\n", total_tag, total_s);
    for (const auto& it : items) fprintf(stdout, "* %-40s %15.9f sec\n", it.first, it.second);
    fputc('\n', stdout);
    fflush(stdout);
}

}  // namespace ptb

cudaEvent_t ptbgpu_ctx::take_event() {
    if (evused == evpool.size()) {
        cudaEvent_t e;
        PTB_CUDA(cudaEventCreate(&e));
        evpool.push_back(e);
    }
    return evpool[evused++];
}

static_assert(ptb::B_COUNT <= ptbgpu_ctx::kMaxBufs, "more scratch-buffer ids than slots");

ptb::DevBuf& ptbgpu_ctx::buf(int id) {
    PTB_CHECK(id >= 0 && id < kMaxBufs, PTBGPU_EINVAL, "scratch buffer id %d out of range", id);
    return bufs[id];
}

extern "C" {

int ptbgpu_init(int device, ptbgpu_ctx** out) {
    if (!out) return PTBGPU_EINVAL;
    *out = nullptr;
    ptbgpu_ctx* c = new ptbgpu_ctx();
    try {
        c->device = device;
        PTB_CUDA(cudaSetDevice(device));
        int major = 0, minor = 0;
        PTB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
        PTB_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
        PTB_CHECK(major == 10 && minor == 0, PTBGPU_ECUDA,
                  "libptbgpu is built for sm_100a (B200); device %d is sm_%d%d", device, major, minor);
        PTB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
        PTB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        PTB_CUBLAS(cublasCreate(&c->blas));
        PTB_CUBLAS(cublasSetStream(c->blas, c->stream));
        PTB_CUBLAS(cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH));
        PTB_CUSOLVER(cusolverDnCreate(&c->solver));
        PTB_CUSOLVER(cusolverDnSetStream(c->solver, c->stream));
        for (auto& e : c->ev) PTB_CUDA(cudaEventCreate(&e));
        PTB_CUDA(cudaMalloc(&c->flags, sizeof(ptb::DeviceFlags)));
        PTB_CUDA(cudaMemset(c->flags, 0, sizeof(ptb::DeviceFlags)));
        PTB_CUDA(cudaMalloc(&c->info_dev, sizeof(int)));
        PTB_CUDA(cudaMallocHost(&c->pinned, 4096));
    } catch (const ptb::Error& e) {
        fprintf(stderr, "ptbgpu_init: %s\n", e.msg.c_str());
        int code = e.code;
        ptbgpu_finalize(c);
        return code;
    }
    *out = c;
    return PTBGPU_OK;
}

int ptbgpu_finalize(ptbgpu_ctx* c) {
    if (!c) return PTBGPU_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->sm_plan.reset();
    c->sm_side.reset();
    for (ptbgpu_ctx* w : c->workers) ptbgpu_finalize(w);
    c->workers.clear();
    for (auto& b : c->bufs) b.release();
    if (c->flags) cudaFree(c->flags);
    if (c->info_dev) cudaFree(c->info_dev);
    if (c->sp2_state) cudaFree(c->sp2_state);
    if (c->pinned) cudaFreeHost(c->pinned);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->evpool) cudaEventDestroy(e);
    if (c->solver) cusolverDnDestroy(c->solver);
    if (c->blas) cublasDestroy(c->blas);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PTBGPU_OK;
}

int ptbgpu_last_error(const ptbgpu_ctx* c, char* buf, size_t len) {
    if (!c || !buf || len == 0) return PTBGPU_EINVAL;
    strncpy(buf, c->last_error.c_str(), len - 1);
    buf[len - 1] = '\0';
    return PTBGPU_OK;
}

int ptbgpu_runtime_info(const ptbgpu_ctx* c, char* buf, size_t len) {
    if (!c || !buf || len == 0) return PTBGPU_EINVAL;
    int rt = 0, drv = 0, cub = 0, maj = 0, min = 0, pat = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    cublasGetVersion(c->blas, &cub);
    cusolverGetProperty(MAJOR_VERSION, &maj);
    cusolverGetProperty(MINOR_VERSION, &min);
    cusolverGetProperty(PATCH_LEVEL, &pat);
    cudaDeviceProp p{};
    cudaGetDeviceProperties(&p, c->device);
    snprintf(buf, len, "device %s (sm_%d%d, %d SMs) cudart %d driver %d cublas %d cusolver %d.%d.%d", p.name,
             p.major, p.minor, p.multiProcessorCount, rt, drv, cub, maj, min, pat);
    return PTBGPU_OK;
}

void ptbgpu_default_settings(ptbgpu_pur_settings* s) {
    if (!s) return;
    s->mode = PTBGPU_MODE_FULL;
    s->type = PTBGPU_TYPE_DIAG;
    s->cycles = 40;
    s->prlvl = 1;
    s->nel = 0;
    s->submatrix_mode = PTBGPU_SUBMATRIX_SYGV;
    s->submatrix_columns = PTBGPU_COLUMNS_ATOMS;
    s->metric_type = PTBGPU_METRIC_INV_SQRT;
    s->metric_cycles = 50;
    s->metric_iterative = 0;
    s->chempot_cycles = 60;
    s->chempot_guess = -1.5;
    s->chempot_increment = 0.1;
}

void ptbgpu_default_opts(ptbgpu_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->precision = PTBGPU_PREC_MIXED;
    o->print_level = 0;
    o->max_iter = 100;
    o->electronic_temp = 300.0;
    o->split3_iters = -1;
    o->fp64_slices = 8;
    o->refine_rounds = 4;
    o->refine_tol = 1e-7;
}

}  // extern "C"
