// C ABI of libdonofb200 (declarations and reference mapping in donof_b200.h).
#include <stdarg.h>
#include <string.h>

#include <atomic>
#include <new>

#include "kernels.cuh"

namespace donof {

static thread_local std::string g_tls_error;
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void g_launch_adjust(long long delta) {
    g_launches.fetch_add((unsigned long long)delta, std::memory_order_relaxed);
}

void set_error(donof_ctx* ctx, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->last_error = buf;
    g_tls_error = buf;
}

// Device memory comes from the stream-ordered allocator on the context's
// stream: an allocation or free waits only for that stream's earlier work, never
// for the whole device (cudaFree would), so jobs served side by side do not
// stall each other when one of them starts, grows a buffer or ends.
int dev_alloc(donof_ctx* ctx, void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 256, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(ctx, "device allocation of %zu bytes: %s", bytes, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? DONOF_ERR_OOM : DONOF_ERR_CUDA;
    }
    return DONOF_OK;
}

void dev_free(donof_ctx* ctx, const void* p) {
    if (p) cudaFreeAsync(const_cast<void*>(p), ctx->stream);
}

int take_failures(donof_ctx* ctx) {
    if (!ctx->fail_host) return 0;
    int mask = 0;
    for (int k = 0; k < FAIL_WORDS; ++k)
        if (ctx->fail_host[k]) {
            mask |= 1 << k;
            ctx->fail_host[k] = 0;
        }
    return mask;
}

int sync_and_check(donof_ctx* ctx) {
    DONOF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return failure_status(ctx);
}

int failure_status(donof_ctx* ctx) {
    const int f = take_failures(ctx) & ((1 << FAIL_MBAR) | (1 << FAIL_BARRIER));
    if (f) {
        set_error(ctx, "a kernel gave up on a bounded %s wait; the call's outputs are not valid",
                  (f & (1 << FAIL_MBAR)) ? "mbarrier" : "grid-barrier");
        return DONOF_ERR_TIMEOUT;
    }
    return DONOF_OK;
}

namespace {
// Sets the context's FAIL_NONFINITE word if any of the count values is a NaN or
// an infinity (the word may be host memory: plain stores of 1).
__global__ void scan_nonfinite_kernel(const double* __restrict__ v, long long count, int* __restrict__ word) {
    bool bad = false;
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if ((reinterpret_cast<uintptr_t>(v) & 15) == 0) {
        const long long n2 = count / 2;
        const double2* v2 = reinterpret_cast<const double2*>(v);
        for (long long k = i; k < n2; k += stride) {
            const double2 x = __ldg(v2 + k);
            bad |= !isfinite(x.x) || !isfinite(x.y);
        }
        for (long long k = 2 * n2 + i; k < count; k += stride) bad |= !isfinite(__ldg(v + k));
    } else {
        for (long long k = i; k < count; k += stride) bad |= !isfinite(__ldg(v + k));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) *reinterpret_cast<volatile int*>(word) = 1;
}
}  // namespace

// DONOF_ERR_ARG if the device array holds a NaN or an infinity (one pass,
// synchronises the context stream).
int check_finite(donof_ctx* ctx, const double* v, long long count, const char* what) {
    if (!ctx->fail_dev) return DONOF_OK;
    long long blocks = (count / 2 + 255) / 256;
    if (blocks > 8LL * ctx->sm_count) blocks = 8LL * ctx->sm_count;
    if (blocks < 1) blocks = 1;
    scan_nonfinite_kernel<<<(int)blocks, 256, 0, ctx->stream>>>(v, count, ctx->fail_dev + FAIL_NONFINITE);
    count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->fail_host[FAIL_NONFINITE]) {
        ctx->fail_host[FAIL_NONFINITE] = 0;
        set_error(ctx, "%s holds a NaN or an infinity", what);
        return DONOF_ERR_ARG;
    }
    return DONOF_OK;
}

int DevBuf::ensure(donof_ctx* ctx, size_t want) {
    if (want <= bytes && ptr != nullptr) return DONOF_OK;
    if (ptr) {
        dev_free(ctx, ptr);
        ptr = nullptr;
        bytes = 0;
    }
    ++gen;
    if (want == 0) want = 256;
    DONOF_CHECK(dev_alloc(ctx, &ptr, want));
    bytes = want;
    return DONOF_OK;
}

void DevBuf::release(donof_ctx* ctx) {
    dev_free(ctx, ptr);
    ptr = nullptr;
    bytes = 0;
}

int orbopt_run(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
               const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
               double threshgorb, double* C, double* E_out, int* nit_out, int* success_out,
               int precision);
int convert_b_f32(donof_job* job);
int mixed_t1_debug(donof_job* job, cudaStream_t st, const double* C, int nbf5, float* tmp_out);

}  // namespace donof

using namespace donof;

namespace {

int use_device(donof_ctx* ctx) {
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    return DONOF_OK;
}

int check_sizes(donof_ctx* ctx, int nbf, int nbf5, int nalpha, int nbeta) {
    if (nbf <= 0 || nbf5 <= 0 || nbf5 > nbf) {
        set_error(ctx, "invalid sizes nbf=%d nbf5=%d", nbf, nbf5);
        return DONOF_ERR_ARG;
    }
    if (nbeta < 0 || nalpha < nbeta || nalpha > nbf5) {
        set_error(ctx, "invalid occupations nalpha=%d nbeta=%d nbf5=%d", nalpha, nbeta, nbf5);
        return DONOF_ERR_ARG;
    }
    return DONOF_OK;
}

#define REQUIRE(ctx, cond, msg)                 \
    do {                                        \
        if (!(cond)) {                          \
            set_error((ctx), "%s", (msg));      \
            return DONOF_ERR_ARG;               \
        }                                       \
    } while (0)

// Moves caller host arrays to and from device staging slots.  Host data goes
// through the context's page-locked buffer: an input is copied into it on the
// host and then sent by an asynchronous DMA; an output is DMA'd into it and
// copied to the caller's array once finish() has synchronised the stream.
// Page-locked transfers run at full PCIe speed whatever memory the caller
// passes.  A caller array that is itself page-locked (cudaMallocHost,
// cudaHostRegister, a pinned torch tensor) is DMA'd directly, with no host
// copy.  Without pin(), or when no page-locked memory can be allocated, the
// copies use the caller's memory directly.
struct Stager {
    donof_ctx* ctx;
    cudaStream_t st;
    char* base;
    size_t off = 0;
    char* pinned = nullptr;
    size_t pinned_bytes = 0, hoff = 0;
    struct Out {
        void* dst;
        const char* src;
        size_t bytes;
    };
    Out outs[8];
    int nout = 0;

    static size_t bytes(size_t count) { return ((count * sizeof(double) + 255) / 256) * 256; }

    // the caller's array is page-locked host memory the DMA engines can reach
    static bool page_locked(const void* h) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    }

    // page-locked room for `total` bytes of inputs and outputs
    int pin(size_t total) {
        if (ctx->hstage_busy) {  // an earlier call that failed may still be copying through it
            DONOF_CUDA(ctx, cudaStreamSynchronize(st));
            ctx->hstage_busy = false;
        }
        if (ctx->hstage_bytes < total) {
            if (ctx->hstage) cudaFreeHost(ctx->hstage);
            ctx->hstage = nullptr;
            ctx->hstage_bytes = 0;
            if (cudaMallocHost(&ctx->hstage, total) != cudaSuccess) {
                // no page-locked memory to be had: copy from the caller's arrays directly
                cudaGetLastError();
                ctx->hstage = nullptr;
                return DONOF_OK;
            }
            ctx->hstage_bytes = total;
        }
        pinned = static_cast<char*>(ctx->hstage);
        pinned_bytes = ctx->hstage_bytes;
        return DONOF_OK;
    }
    // device slot for `count` doubles, filled from h (if not null)
    double* put(const double* h, size_t count) {
        double* d = reinterpret_cast<double*>(base + off);
        const size_t b = bytes(count);
        off += b;
        if (h == nullptr) return d;
        if (pinned && !page_locked(h) && hoff + b <= pinned_bytes) {
            memcpy(pinned + hoff, h, count * sizeof(double));
            cudaMemcpyAsync(d, pinned + hoff, count * sizeof(double), cudaMemcpyHostToDevice, st);
            hoff += b;
            ctx->hstage_busy = true;
        } else {
            cudaMemcpyAsync(d, h, count * sizeof(double), cudaMemcpyHostToDevice, st);
        }
        return d;
    }
    // device -> caller array h, complete after finish()
    int get(double* h, const double* d, size_t count) {
        const size_t b = bytes(count);
        if (pinned && !page_locked(h) && hoff + b <= pinned_bytes && nout < 8) {
            DONOF_CUDA(ctx, cudaMemcpyAsync(pinned + hoff, d, count * sizeof(double), cudaMemcpyDeviceToHost, st));
            outs[nout++] = Out{h, pinned + hoff, count * sizeof(double)};
            hoff += b;
            ctx->hstage_busy = true;
        } else {
            DONOF_CUDA(ctx, cudaMemcpyAsync(h, d, count * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        return DONOF_OK;
    }
    int finish() {
        const int s = sync_and_check(ctx);
        if (s == DONOF_ERR_CUDA) return s;
        for (int i = 0; i < nout; ++i) memcpy(outs[i].dst, outs[i].src, outs[i].bytes);
        ctx->hstage_busy = false;
        return s;
    }
};

int effective_precision(donof_job* job, int precision) {
    if (precision != DONOF_PREC_FP64 && precision != DONOF_PREC_MIXED) {
        set_error(job->ctx, "unknown precision %d", precision);
        return -1;
    }
    if (precision == DONOF_PREC_MIXED && job->b16hi == nullptr) {
        set_error(job->ctx, "mixed precision requested but the job holds no bf16 split of b");
        return -1;
    }
    return precision;
}

}  // namespace

extern "C" {

int donof_version(void) { return 1; }

unsigned long long donof_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int donof_profile_enable(donof_ctx* ctx, int enable) {
    if (!ctx) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    if (enable && !ctx->prof_ev[0]) {
        DONOF_CUDA(ctx, cudaEventCreate(&ctx->prof_ev[0]));
        DONOF_CUDA(ctx, cudaEventCreate(&ctx->prof_ev[1]));
    }
    ctx->profile = enable != 0;
    ctx->prof_recorded = false;
    return DONOF_OK;
}

int donof_profile_last_ms(donof_ctx* ctx, float* ms) {
    if (!ctx || !ms) return DONOF_ERR_ARG;
    if (!ctx->profile || !ctx->prof_recorded) {
        set_error(ctx, "no profiled kernel recorded");
        return DONOF_ERR_STATE;
    }
    DONOF_CHECK(use_device(ctx));
    DONOF_CUDA(ctx, cudaEventSynchronize(ctx->prof_ev[1]));
    DONOF_CUDA(ctx, cudaEventElapsedTime(ms, ctx->prof_ev[0], ctx->prof_ev[1]));
    return DONOF_OK;
}

int donof_error_flags(donof_ctx* ctx, int* flags) {
    if (!ctx || !flags) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    DONOF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *flags = take_failures(ctx);
    return DONOF_OK;
}

int donof_job_error_flag(donof_job* job, int* flag) {
    if (!job || !flag) return DONOF_ERR_ARG;
    int f = 0;
    DONOF_CHECK(donof_error_flags(job->ctx, &f));
    *flag = f ? 1 : 0;
    return DONOF_OK;
}

int donof_set_wait_limit(donof_ctx* ctx, long long cycles) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, cycles >= 0, "the wait budget must be >= 0");
    ctx->wait_limit = cycles;
    return DONOF_OK;
}

int donof_mixed_tmp_dev(donof_job* job, const double* C, int nbf5, float* tmp) {
    if (!job || !C || !tmp) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(job->ctx));
    return mixed_t1_debug(job, job->ctx->stream, C, nbf5, tmp);
}

int donof_job_set_fp64_tc(donof_job* job, int enable) {
    if (!job) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(job->ctx));
    if (enable) return ozaki_build(job);
    ozaki_free(job);
    return DONOF_OK;
}

int donof_job_fp64_tc(const donof_job* job) { return job && job->oz_b ? 1 : 0; }

int donof_t1_dev(donof_job* job, const double* C, int nbf5, double* tmp) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    REQUIRE(ctx, C != nullptr && tmp != nullptr, "null pointer");
    REQUIRE(ctx, nbf5 > 0 && nbf5 <= job->nbf, "invalid nbf5");
    DONOF_CHECK(use_device(ctx));
    if (job->oz_b) return t1_ozaki(job, ctx->stream, C, nbf5, tmp);
    DONOF_CHECK(transforms_f64(job, ctx->stream, C, nbf5));
    DONOF_CUDA(ctx, cudaMemcpyAsync(tmp, job->tmp.ptr, sizeof(double) * (size_t)job->nbf * nbf5 * job->naux,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
    return DONOF_OK;
}

int donof_transform_dev(donof_job* job, int precision, const double* C, int nbf5, double* b_pq) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    REQUIRE(ctx, C != nullptr, "null C");
    REQUIRE(ctx, nbf5 > 0 && nbf5 <= job->nbf, "invalid nbf5");
    const int prec = effective_precision(job, precision);
    if (prec < 0) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    if (prec == DONOF_PREC_MIXED) {
        DONOF_CHECK(transforms_mixed(job, ctx->stream, C, nbf5));
    } else {
        DONOF_CHECK(transforms_f64(job, ctx->stream, C, nbf5));
    }
    if (b_pq != nullptr)
        DONOF_CUDA(ctx, cudaMemcpyAsync(b_pq, job->bpq.ptr, sizeof(double) * (size_t)nbf5 * nbf5 * job->naux,
                                        cudaMemcpyDeviceToDevice, ctx->stream));
    return DONOF_OK;
}

const char* donof_status_string(int s) {
    switch (s) {
        case DONOF_OK: return "ok";
        case DONOF_ERR_ARG: return "invalid argument";
        case DONOF_ERR_CUDA: return "CUDA error";
        case DONOF_ERR_OOM: return "out of device memory";
        case DONOF_ERR_STATE: return "invalid state";
        case DONOF_ERR_NOT_CONVERGED: return "not converged";
        case DONOF_ERR_TIMEOUT: return "a bounded wait ran out";
        default: return "unknown status";
    }
}

const char* donof_last_error(const donof_ctx* ctx) {
    if (ctx) return ctx->last_error.c_str();
    return g_tls_error.c_str();
}

int donof_create(int device, donof_ctx** out) {
    if (out == nullptr) {
        set_error(nullptr, "donof_create: null output pointer");
        return DONOF_ERR_ARG;
    }
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        set_error(nullptr, "donof_create: device %d not available (%d devices, %s)", device, count,
                  cudaGetErrorString(e));
        return e != cudaSuccess ? DONOF_ERR_CUDA : DONOF_ERR_ARG;
    }
    donof_ctx* ctx = new (std::nothrow) donof_ctx();
    if (!ctx) return DONOF_ERR_OOM;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error(nullptr, "donof_create: cannot create a stream on device %d", device);
        delete ctx;
        return DONOF_ERR_CUDA;
    }
    ctx->own_stream = true;
    {
        // failure words: page-locked host memory the kernels write through its device alias
        void* h = nullptr;
        void* d = nullptr;
        if (cudaHostAlloc(&h, 256, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
            cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
            set_error(nullptr, "donof_create: cannot map the failure words on device %d", device);
            if (h) cudaFreeHost(h);
            cudaStreamDestroy(ctx->stream);
            delete ctx;
            return DONOF_ERR_CUDA;
        }
        memset(h, 0, 256);
        ctx->fail_host = static_cast<volatile int*>(h);
        ctx->fail_dev = static_cast<int*>(d);
    }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    {
        // keep freed blocks in the device's default pool (process-local) instead of
        // returning them to the driver at every synchronisation
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    *out = ctx;
    return DONOF_OK;
}

int donof_destroy(donof_ctx* ctx) {
    if (!ctx) return DONOF_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->stage_in.release(ctx);
    ctx->stage_out.release(ctx);
    ctx->rot.release(ctx);
    if (ctx->hstage) cudaFreeHost(ctx->hstage);
    if (ctx->fail_host) cudaFreeHost(const_cast<int*>(ctx->fail_host));
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->aux_stream) cudaStreamDestroy(ctx->aux_stream);
    if (ctx->prof_ev[0]) cudaEventDestroy(ctx->prof_ev[0]);
    if (ctx->prof_ev[1]) cudaEventDestroy(ctx->prof_ev[1]);
    delete ctx;
    return DONOF_OK;
}

int donof_set_stream(donof_ctx* ctx, void* stream) {
    if (!ctx) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    if (ctx->own_stream && ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    ctx->stream = static_cast<cudaStream_t>(stream);
    ctx->own_stream = false;
    return DONOF_OK;
}

void* donof_get_stream(donof_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int donof_set_cta_limit(donof_ctx* ctx, int max_ctas) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, max_ctas >= 0, "max_ctas must be >= 0");
    ctx->cta_limit = max_ctas;
    return DONOF_OK;
}

int donof_synchronize(donof_ctx* ctx) {
    if (!ctx) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    DONOF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return DONOF_OK;
}

static int make_job(donof_ctx* ctx, int nbf, int naux, int precision, donof_job** job) {
    REQUIRE(ctx, job != nullptr, "null job pointer");
    REQUIRE(ctx, nbf > 0 && naux > 0, "nbf and naux must be positive");
    REQUIRE(ctx, precision == DONOF_PREC_FP64 || precision == DONOF_PREC_MIXED, "unknown precision");
    donof_job* j = new (std::nothrow) donof_job();
    if (!j) return DONOF_ERR_OOM;
    j->ctx = ctx;
    j->nbf = nbf;
    j->naux = naux;
    j->precision = precision;
    *job = j;
    return DONOF_OK;
}

int donof_b_upload(donof_ctx* ctx, const double* b_host, int nbf, int naux, int precision,
                   donof_job** job) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, b_host != nullptr, "null b");
    DONOF_CHECK(use_device(ctx));
    donof_job* j = nullptr;
    DONOF_CHECK(make_job(ctx, nbf, naux, precision, &j));
    const size_t bytes = sizeof(double) * (size_t)nbf * nbf * naux;
    void* d = nullptr;
    int s0 = dev_alloc(ctx, &d, bytes);
    if (s0 != DONOF_OK) {
        delete j;
        return s0;
    }
    cudaError_t e = cudaMemcpyAsync(d, b_host, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        dev_free(ctx, d);
        delete j;
        set_error(ctx, "upload of b: %s", cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    j->b = static_cast<const double*>(d);
    j->own_b = true;
    {
        const int sf = check_finite(ctx, j->b, (long long)nbf * nbf * naux, "b");
        if (sf != DONOF_OK) {
            donof_job_free(j);
            return sf;
        }
    }
    if (precision == DONOF_PREC_MIXED) {
        int s = convert_b_f32(j);
        if (s != DONOF_OK) {
            donof_job_free(j);
            return s;
        }
    }
    *job = j;
    return DONOF_OK;
}

int donof_iaux(donof_ctx* ctx, const double* G, const double* I3c, int nbf, int naux, int precision,
               donof_job** job) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, G != nullptr && I3c != nullptr, "null G or I");
    DONOF_CHECK(use_device(ctx));
    donof_job* j = nullptr;
    DONOF_CHECK(make_job(ctx, nbf, naux, precision, &j));
    const size_t bytes = sizeof(double) * (size_t)nbf * nbf * naux;
    void* d = nullptr;
    int s = dev_alloc(ctx, &d, bytes);
    if (s != DONOF_OK) {
        delete j;
        return s;
    }
    s = iaux_f64(ctx, ctx->stream, G, I3c, nbf, naux, static_cast<double*>(d), &j->part);
    if (s != DONOF_OK) {
        cudaStreamSynchronize(ctx->stream);
        dev_free(ctx, d);
        j->part.release(ctx);
        delete j;
        return s;
    }
    j->b = static_cast<const double*>(d);
    j->own_b = true;
    s = check_finite(ctx, j->b, (long long)nbf * nbf * naux, "b = I G^-1/2");
    if (s != DONOF_OK) {
        donof_job_free(j);
        return s;
    }
    if (precision == DONOF_PREC_MIXED) {
        s = convert_b_f32(j);
        if (s != DONOF_OK) {
            donof_job_free(j);
            return s;
        }
    }
    *job = j;
    return DONOF_OK;
}

int donof_b_attach(donof_ctx* ctx, const double* b_dev, int nbf, int naux, int precision,
                   donof_job** job) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, b_dev != nullptr, "null b");
    DONOF_CHECK(use_device(ctx));
    donof_job* j = nullptr;
    DONOF_CHECK(make_job(ctx, nbf, naux, precision, &j));
    j->b = b_dev;
    j->own_b = false;
    {
        const int sf = check_finite(ctx, j->b, (long long)nbf * nbf * naux, "b");
        if (sf != DONOF_OK) {
            donof_job_free(j);
            return sf;
        }
    }
    if (precision == DONOF_PREC_MIXED) {
        int s = convert_b_f32(j);
        if (s != DONOF_OK) {
            donof_job_free(j);
            return s;
        }
    }
    *job = j;
    return DONOF_OK;
}

int donof_job_free(donof_job* job) {
    if (!job) return DONOF_OK;
    donof_ctx* ctx = job->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);  // no work of the job is in flight (graphs are destroyed below)
    if (job->own_b) dev_free(ctx, job->b);
    dev_free(ctx, job->b16hi);
    dev_free(ctx, job->b16lo);
    ozaki_free(job);
    job->tmp.release(ctx);
    job->bpq.release(ctx);
    job->W.release(ctx);
    job->part.release(ctx);
    job->small.release(ctx);
    job->orb.release(ctx);
    if (job->orb_exec) cudaGraphExecDestroy(job->orb_exec);
    if (job->orb_graph) cudaGraphDestroy(job->orb_graph);
    job->io.release(ctx);
    job->drv.release(ctx);
    delete job;
    return DONOF_OK;
}

int donof_job_set_precision(donof_job* job, int precision) {
    if (!job) return DONOF_ERR_ARG;
    const int prec = effective_precision(job, precision);
    if (prec < 0) return DONOF_ERR_ARG;
    job->precision = prec;
    return DONOF_OK;
}

size_t donof_job_device_bytes(const donof_job* job) {
    if (!job) return 0;
    size_t s = job->tmp.bytes + job->bpq.bytes + job->W.bytes + job->part.bytes + job->small.bytes +
               job->orb.bytes + job->io.bytes;
    if (job->own_b) s += sizeof(double) * (size_t)job->nbf * job->nbf * job->naux;
    if (job->b16hi) s += 4 * (size_t)64 * ((job->nbf + 63) / 64) * job->nbf * job->naux;
    if (job->oz_b) s += ozaki_bytes(job->nbf, job->naux) + job->oz_c.bytes;
    return s;
}

int donof_lagrange2_prec_dev(donof_job* job, int precision, const double* C, const double* n,
                             const double* H, const double* cj12, const double* ck12, int nbf5,
                             int nalpha, int nbeta, double* elag, double* H_mat, double* E_elec) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    DONOF_CHECK(check_sizes(ctx, job->nbf, nbf5, nalpha, nbeta));
    REQUIRE(ctx, C && n && H && cj12 && ck12 && elag && H_mat, "null array argument");
    const int prec = effective_precision(job, precision);
    if (prec < 0) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    if (prec == DONOF_PREC_MIXED)
        return lagrange2_mixed(job, ctx->stream, C, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, H_mat,
                               E_elec);
    return lagrange2_f64(job, ctx->stream, C, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, H_mat,
                         E_elec);
}

int donof_lagrange2_dev(donof_job* job, const double* C, const double* n, const double* H,
                        const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta,
                        double* elag, double* H_mat, double* E_elec) {
    if (!job) return DONOF_ERR_ARG;
    return donof_lagrange2_prec_dev(job, job->precision, C, n, H, cj12, ck12, nbf5, nalpha, nbeta,
                                    elag, H_mat, E_elec);
}

int donof_lagrange2(donof_job* job, const double* C, const double* n, const double* H,
                    const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta,
                    double* elag, double* H_mat, double* E_elec) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    DONOF_CHECK(check_sizes(ctx, job->nbf, nbf5, nalpha, nbeta));
    REQUIRE(ctx, C && n && H && cj12 && ck12 && elag && H_mat, "null array argument");
    DONOF_CHECK(use_device(ctx));
    const size_t nbf = job->nbf, nn = nbf * nbf, n55 = (size_t)nbf5 * nbf5;
    const size_t need = Stager::bytes(nn) * 3 + Stager::bytes(nbf5) + Stager::bytes(n55) * 2 +
                        Stager::bytes(nbf * nbf5) + Stager::bytes(1);
    DONOF_CHECK(job->io.ensure(ctx, need));
    Stager sg{ctx, ctx->stream, job->io.as<char>()};
    DONOF_CHECK(sg.pin(job->io.bytes));
    const double* dC = sg.put(C, nn);
    const double* dH = sg.put(H, nn);
    const double* dn = sg.put(n, nbf5);
    const double* dcj = sg.put(cj12, n55);
    const double* dck = sg.put(ck12, n55);
    double* del = sg.put(nullptr, nn);
    double* dHm = sg.put(nullptr, nbf * nbf5);
    double* dE = sg.put(nullptr, 1);
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(donof_lagrange2_dev(job, dC, dn, dH, dcj, dck, nbf5, nalpha, nbeta, del, dHm, dE));
    DONOF_CHECK(sg.get(elag, del, nn));
    DONOF_CHECK(sg.get(H_mat, dHm, nbf * nbf5));
    if (E_elec)
        DONOF_CHECK(sg.get(E_elec, dE, 1));
    DONOF_CHECK(sg.finish());
    return DONOF_OK;
}

int donof_lagrange2_partial_dev(donof_job* job, const double* C, const double* n, const double* cj12,
                                const double* ck12, int nbf5, int nalpha, int nbeta, double* Y) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    DONOF_CHECK(check_sizes(ctx, job->nbf, nbf5, nalpha, nbeta));
    REQUIRE(ctx, C && n && cj12 && ck12 && Y, "null array argument");
    DONOF_CHECK(use_device(ctx));
    return lagrange2_partial_f64(job, ctx->stream, C, n, cj12, ck12, nbf5, nalpha, nbeta, Y);
}

int donof_lagrange2_finish_dev(donof_job* job, const double* C, const double* n, const double* H, int nbf5,
                               const double* Y, double* elag, double* H_mat, double* E_elec) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    REQUIRE(ctx, nbf5 > 0 && nbf5 <= job->nbf, "invalid nbf5");
    REQUIRE(ctx, C && n && H && Y && elag && H_mat, "null array argument");
    DONOF_CHECK(use_device(ctx));
    return lagrange2_finish_f64(job, ctx->stream, C, n, H, nbf5, Y, elag, H_mat, E_elec);
}

int donof_jkh_mo_prec_dev(donof_job* job, int precision, const double* C, const double* H, int nbf5,
                          double* J_MO, double* K_MO, double* H_core) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    REQUIRE(ctx, nbf5 > 0 && nbf5 <= job->nbf, "invalid nbf5");
    REQUIRE(ctx, C && H && J_MO && K_MO && H_core, "null array argument");
    const int prec = effective_precision(job, precision);
    if (prec < 0) return DONOF_ERR_ARG;
    DONOF_CHECK(use_device(ctx));
    if (prec == DONOF_PREC_MIXED) return jkh_mo_mixed(job, ctx->stream, C, H, nbf5, J_MO, K_MO, H_core);
    return jkh_mo_f64(job, ctx->stream, C, H, nbf5, J_MO, K_MO, H_core);
}

int donof_jkh_mo_dev(donof_job* job, const double* C, const double* H, int nbf5, double* J_MO,
                     double* K_MO, double* H_core) {
    if (!job) return DONOF_ERR_ARG;
    return donof_jkh_mo_prec_dev(job, job->precision, C, H, nbf5, J_MO, K_MO, H_core);
}

int donof_jkh_mo(donof_job* job, const double* C, const double* H, int nbf5, double* J_MO,
                 double* K_MO, double* H_core) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    REQUIRE(ctx, nbf5 > 0 && nbf5 <= job->nbf, "invalid nbf5");
    REQUIRE(ctx, C && H && J_MO && K_MO && H_core, "null array argument");
    DONOF_CHECK(use_device(ctx));
    const size_t nbf = job->nbf, nn = nbf * nbf, n55 = (size_t)nbf5 * nbf5;
    DONOF_CHECK(job->io.ensure(ctx, Stager::bytes(nn) * 2 + Stager::bytes(n55) * 2 + Stager::bytes(nbf5)));
    Stager sg{ctx, ctx->stream, job->io.as<char>()};
    DONOF_CHECK(sg.pin(job->io.bytes));
    const double* dC = sg.put(C, nn);
    const double* dH = sg.put(H, nn);
    double* dJ = sg.put(nullptr, n55);
    double* dK = sg.put(nullptr, n55);
    double* dh = sg.put(nullptr, nbf5);
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(donof_jkh_mo_dev(job, dC, dH, nbf5, dJ, dK, dh));
    DONOF_CHECK(sg.get(J_MO, dJ, n55));
    DONOF_CHECK(sg.get(K_MO, dK, n55));
    DONOF_CHECK(sg.get(H_core, dh, nbf5));
    DONOF_CHECK(sg.finish());
    return DONOF_OK;
}

int donof_rotate_dev(donof_ctx* ctx, const double* y, int nbf, int nbf5, const double* C,
                     double* C_new) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, nbf > 0 && nbf5 > 0 && nbf5 <= nbf, "invalid sizes");
    REQUIRE(ctx, y && C && C_new, "null array argument");
    REQUIRE(ctx, C != C_new, "C_new must not alias C");
    DONOF_CHECK(use_device(ctx));
    return rotate_f64(ctx, ctx->stream, y, nbf, nbf5, C, C_new);
}

int donof_rotate(donof_ctx* ctx, const double* y, int nbf, int nbf5, const double* C, double* C_new) {
    if (!ctx) return DONOF_ERR_ARG;
    REQUIRE(ctx, nbf > 0 && nbf5 > 0 && nbf5 <= nbf, "invalid sizes");
    REQUIRE(ctx, y && C && C_new, "null array argument");
    DONOF_CHECK(use_device(ctx));
    const size_t nn = (size_t)nbf * nbf, nvar = (size_t)nvar_of(nbf, nbf5);
    DONOF_CHECK(ctx->stage_in.ensure(ctx, Stager::bytes(nvar) + Stager::bytes(nn) * 2));
    Stager sg{ctx, ctx->stream, ctx->stage_in.as<char>()};
    DONOF_CHECK(sg.pin(ctx->stage_in.bytes));
    const double* dy = sg.put(y, nvar);
    const double* dC = sg.put(C, nn);
    double* dCn = sg.put(nullptr, nn);
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(rotate_f64(ctx, ctx->stream, dy, nbf, nbf5, dC, dCn));
    DONOF_CHECK(sg.get(C_new, dCn, nn));
    DONOF_CHECK(sg.finish());
    return DONOF_OK;
}

int donof_orbgrad(donof_job* job, const double* y, const double* C, const double* n, const double* H,
                  const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta,
                  double* grad) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    DONOF_CHECK(check_sizes(ctx, job->nbf, nbf5, nalpha, nbeta));
    REQUIRE(ctx, C && n && H && cj12 && ck12 && grad, "null array argument");
    DONOF_CHECK(use_device(ctx));
    const size_t nbf = job->nbf, nn = nbf * nbf, n55 = (size_t)nbf5 * nbf5;
    const size_t nvar = (size_t)nvar_of((int)nbf, nbf5);
    const size_t need = Stager::bytes(nvar) * 2 + Stager::bytes(nn) * 4 + Stager::bytes(nbf5) +
                        Stager::bytes(n55) * 2 + Stager::bytes(nbf * nbf5);
    DONOF_CHECK(job->io.ensure(ctx, need));
    Stager sg{ctx, ctx->stream, job->io.as<char>()};
    DONOF_CHECK(sg.pin(job->io.bytes));
    const double* dy = sg.put(y, nvar);
    const double* dC = sg.put(C, nn);
    const double* dH = sg.put(H, nn);
    const double* dn = sg.put(n, nbf5);
    const double* dcj = sg.put(cj12, n55);
    const double* dck = sg.put(ck12, n55);
    double* dCr = sg.put(nullptr, nn);
    double* del = sg.put(nullptr, nn);
    double* dHm = sg.put(nullptr, nbf * nbf5);
    double* dg = sg.put(nullptr, nvar);
    DONOF_CUDA(ctx, cudaGetLastError());
    const double* Cuse = dC;
    if (y != nullptr) {
        DONOF_CHECK(rotate_f64(ctx, ctx->stream, dy, (int)nbf, nbf5, dC, dCr));
        Cuse = dCr;
    }
    DONOF_CHECK(donof_lagrange2_dev(job, Cuse, dn, dH, dcj, dck, nbf5, nalpha, nbeta, del, dHm, nullptr));
    DONOF_CHECK(pack_grad(ctx, ctx->stream, del, (int)nbf, nbf5, dg, nullptr));
    DONOF_CHECK(sg.get(grad, dg, nvar));
    DONOF_CHECK(sg.finish());
    return DONOF_OK;
}

int donof_orbopt(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
                 const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
                 double threshgorb, double* C_inout, double* E, int* nit, int* success) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    DONOF_CHECK(check_sizes(ctx, job->nbf, nbf5, nalpha, nbeta));
    REQUIRE(ctx, n && cj12 && ck12 && H && C_inout && alpha && maxloop && E && nit && success,
            "null argument");
    REQUIRE(ctx, method >= DONOF_ORB_ADAM && method <= DONOF_ORB_DEMON, "unknown optimiser");
    REQUIRE(ctx, *maxloop >= 1, "maxloop must be >= 1");
    DONOF_CHECK(use_device(ctx));
    const size_t nbf = job->nbf, nn = nbf * nbf, n55 = (size_t)nbf5 * nbf5;
    DONOF_CHECK(job->io.ensure(ctx, Stager::bytes(nn) * 2 + Stager::bytes(nbf5) + Stager::bytes(n55) * 2));
    Stager sg{ctx, ctx->stream, job->io.as<char>()};
    DONOF_CHECK(sg.pin(job->io.bytes));
    double* dC = sg.put(C_inout, nn);
    const double* dH = sg.put(H, nn);
    const double* dn = sg.put(n, nbf5);
    const double* dcj = sg.put(cj12, n55);
    const double* dck = sg.put(ck12, n55);
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(orbopt_run(job, method, dn, dcj, dck, dH, nbf5, nalpha, nbeta, alpha, maxloop, threshgorb,
                           dC, E, nit, success, job->precision));
    DONOF_CHECK(sg.get(C_inout, dC, nn));
    DONOF_CHECK(sg.finish());
    return DONOF_OK;
}

int donof_orbopt_dev(donof_job* job, int method, const double* n, const double* cj12, const double* ck12,
                     const double* H, int nbf5, int nalpha, int nbeta, double* alpha, int* maxloop,
                     double threshgorb, double* C_inout, double* E, int* nit, int* success) {
    if (!job) return DONOF_ERR_ARG;
    donof_ctx* ctx = job->ctx;
    DONOF_CHECK(check_sizes(ctx, job->nbf, nbf5, nalpha, nbeta));
    REQUIRE(ctx, n && cj12 && ck12 && H && C_inout && alpha && maxloop && E && nit && success,
            "null argument");
    REQUIRE(ctx, method >= DONOF_ORB_ADAM && method <= DONOF_ORB_DEMON, "unknown optimiser");
    REQUIRE(ctx, *maxloop >= 1, "maxloop must be >= 1");
    DONOF_CHECK(use_device(ctx));
    return orbopt_run(job, method, n, cj12, ck12, H, nbf5, nalpha, nbeta, alpha, maxloop, threshgorb, C_inout,
                      E, nit, success, job->precision);
}

}  // extern "C"
