// Self-test of the bounded device waits' error path.  Every wait of the
// library's kernels (mbarrier phases of the tensor-core pipelines) gives up
// after a time limit, records a site id in the context's device error word and
// lets the kernel finish, and the host turns a nonzero word into
// PTBGPU_ETIMEOUT.  This entry runs one such wait on a flag that nothing sets,
// with a short limit, so the whole path can be tested without a fault.
#include "common.cuh"

namespace ptb {

namespace {

constexpr int kSelftestSite = 90;

__global__ void k_wait_unset_flag(const volatile int* flag, uint64_t limit_ns, int* err) {
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (*flag == 0) {
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns) {
            atomicCAS(err, 0, kSelftestSite);
            return;
        }
        __nanosleep(1000);
    }
}

}  // namespace

}  // namespace ptb

extern "C" int ptbgpu_selftest_bounded_wait(ptbgpu_ctx* c, int64_t limit_us) {
    if (!c) return PTBGPU_EINVAL;
    if (limit_us < 1 || limit_us > 2000000) {
        c->last_error = "limit_us must be 1..2000000";
        return PTBGPU_EINVAL;
    }
    try {
        PTB_CUDA(cudaSetDevice(c->device));
        cudaStream_t s = c->stream;
        PTB_CUDA(cudaMemsetAsync(c->info_dev, 0, sizeof(int), s));                  // the flag: never set
        PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));
        ptb::k_wait_unset_flag<<<1, 1, 0, s>>>(c->info_dev, (uint64_t)limit_us * 1000ull, &c->flags->timeout);
        PTB_CUDA(cudaGetLastError());
        int site = 0;
        PTB_CUDA(cudaMemcpyAsync(&site, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaStreamSynchronize(s));
        PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));   // the context stays usable
        PTB_CUDA(cudaStreamSynchronize(s));
        if (site != 0) {
            char buf[128];
            snprintf(buf, sizeof(buf), "bounded wait gave up after %lld us (site %d)", (long long)limit_us, site);
            c->last_error = buf;
            return PTBGPU_ETIMEOUT;
        }
        c->last_error = "the wait ended without its flag being set";
        return PTBGPU_ECUDA;
    } catch (const ptb::Error& e) {
        c->last_error = e.msg;
        return e.code;
    }
}
