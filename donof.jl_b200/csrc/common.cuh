// Shared definitions for libdonofb200: status codes, context and job objects.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

#include "../../include/donof_b200.h"

namespace donof {

// Count of kernel launches made by the library (diagnostics; see
// donof_launch_count).  Every launch site calls count_launch(); graph
// replays add their kernel count through g_launch_adjust.
void count_launch();
void g_launch_adjust(long long delta);

// Last error text is kept per context (and in a thread-local fallback for
// calls that fail before a context exists).
void set_error(donof_ctx* ctx, const char* fmt, ...);

#define DONOF_CUDA(ctx, call)                                                    \
    do {                                                                         \
        cudaError_t _e = (call);                                                 \
        if (_e != cudaSuccess) {                                                 \
            ::donof::set_error((ctx), "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                               cudaGetErrorString(_e));                          \
            return (_e == cudaErrorMemoryAllocation) ? DONOF_ERR_OOM             \
                                                     : DONOF_ERR_CUDA;           \
        }                                                                        \
    } while (0)

#define DONOF_CHECK(x)                 \
    do {                               \
        int _s = (x);                  \
        if (_s != DONOF_OK) return _s; \
    } while (0)

// A device buffer that grows on demand (never shrinks until freed).
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    unsigned gen = 0;  // bumped on every reallocation (captured graphs check it)
    int ensure(donof_ctx* ctx, size_t want);
    void release(donof_ctx* ctx);  // after the context's stream has no work using it
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

}  // namespace donof

struct donof_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    int sm_count = 148;
    // host-pointer staging (device side) shared by the host-buffer entry points
    donof::DevBuf stage_in, stage_out;
    // page-locked host buffer the host-buffer entry points copy through
    // (grown on demand; hstage_busy while a call's copies may be in flight)
    void* hstage = nullptr;
    size_t hstage_bytes = 0;
    bool hstage_busy = false;
    // scratch for the rotation (exp of the generator)
    donof::DevBuf rot;
    // optional timing of the dominant kernel of each call (donof_profile_*):
    // events recorded on the launching stream around that kernel
    bool profile = false;
    cudaEvent_t prof_ev[2] = {nullptr, nullptr};
    bool prof_recorded = false;
    // private stream for graph capture when the context uses the legacy default stream
    cudaStream_t aux_stream = nullptr;
    // most CTAs a persistent or cooperative kernel of this context may use (0: one
    // per SM); a server running several jobs at once gives each a share of the SMs
    int cta_limit = 0;
    // Failure words written by the context's kernels, in page-locked host memory
    // mapped into the device (kernels store 1 into a word; the host reads it after
    // synchronising the stream, no copy needed).  Sticky until read and cleared.
    //   [FAIL_MBAR]     a mixed-form kernel gave up on a bounded mbarrier wait
    //   [FAIL_BARRIER]  a cooperative kernel gave up on its bounded grid barrier
    //   [FAIL_NONFINITE] a finiteness scan found a NaN or an infinity
    volatile int* fail_host = nullptr;
    int* fail_dev = nullptr;
    // cycle budget of every bounded wait in this context's kernels (0: the
    // built-in ~1-2 s); a small value makes waits run out, for testing the
    // failure path without a fault or a hang
    long long wait_limit = 0;
};

namespace donof {
enum { FAIL_MBAR = 0, FAIL_BARRIER = 1, FAIL_NONFINITE = 2, FAIL_WORDS = 4 };
// Reads and clears the context's failure words (the stream must have been
// synchronised): returns a bit mask, bit k set when word k was set.
int take_failures(donof_ctx* ctx);
// After the caller has synchronised the stream the kernels ran on: turns a
// recorded wait failure into DONOF_ERR_TIMEOUT (with the error text), else
// DONOF_OK.  sync_and_check synchronises the context stream first.
int failure_status(donof_ctx* ctx);
int sync_and_check(donof_ctx* ctx);
// DONOF_ERR_ARG (with the error text) if the device array holds a NaN or an
// infinity; one pass, synchronises the context stream, allocates nothing.
int check_finite(donof_ctx* ctx, const double* v, long long count, const char* what);
// Stream-ordered device allocation on the context's stream (capi.cu).
int dev_alloc(donof_ctx* ctx, void** p, size_t bytes);
void dev_free(donof_ctx* ctx, const void* p);
// CTAs for the persistent and cooperative kernels of a context.
inline int ctx_ctas(const donof_ctx* c) {
    return (c->cta_limit > 0 && c->cta_limit < c->sm_count) ? c->cta_limit : c->sm_count;
}
// Bracket the dominant kernel of a call with the context's profiling events.
inline void prof_begin(donof_ctx* ctx, cudaStream_t st) {
    if (ctx->profile && ctx->prof_ev[0]) cudaEventRecord(ctx->prof_ev[0], st);
}
inline void prof_end(donof_ctx* ctx, cudaStream_t st) {
    if (ctx->profile && ctx->prof_ev[1]) {
        cudaEventRecord(ctx->prof_ev[1], st);
        ctx->prof_recorded = true;
    }
}
}  // namespace donof

struct donof_job {
    donof_ctx* ctx = nullptr;
    int nbf = 0, naux = 0, precision = DONOF_PREC_FP64;
    const double* b = nullptr;  // device [m + nbf*n + nbf*nbf*l]
    bool own_b = false;
    // bf16 split of b for the mixed-precision form: b = hi + lo, quarter-major
    // layout [mi + 64*n + 64*nbf*qb + 64*nbf*nb*l] with m = 64*qb + mi, nb = ceil(nbf/64)
    void* b16hi = nullptr;
    void* b16lo = nullptr;
    // int8 digit slices of b for the FP64 form's T1 on the tensor cores
    // (ozaki.cu): oz_b[n + ldn*(m + nbf*(i + S*l))] with row scales oz_sa[m + nbf*l];
    // oz_c holds the per-call slices of C5; oz_gen counts enable/disable switches
    void* oz_b = nullptr;
    double* oz_sa = nullptr;
    donof::DevBuf oz_c;
    unsigned oz_gen = 0;
    // per-call scratch, sized for the largest nbf5 seen
    donof::DevBuf tmp, bpq, W, part, small;
    // device-resident orbital-optimiser state
    donof::DevBuf orb;
    // host-API staging
    donof::DevBuf io;
    // device arrays of the native energy loop (energy.cu)
    donof::DevBuf drv;
    // captured optimiser loop (graph with a conditional WHILE node) and the
    // inputs it was captured for
    cudaGraph_t orb_graph = nullptr;
    cudaGraphExec_t orb_exec = nullptr;
    unsigned long long orb_key[10] = {};
    int orb_per_iter = 0;
};
