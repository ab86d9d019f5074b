// Host-side dispatch of the FP64 DMMA GEMM (tile shape, operand layout,
// 16-byte vs 8-byte staging) and the split-K reduction.
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "gemm_f64.cuh"
#include "kernels.cuh"

namespace donof {

namespace {

template <int BM, int BN, int WM, int WN, bool AK, bool BKM, bool VEC>
cudaError_t launch_persistent(const GemmF64Args& p, cudaStream_t st) {
    constexpr int BK = 16, STAGES = 3;
    using Cfg = GemmF64Cfg<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    auto kern = gemm_f64_persistent_kernel<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    static std::atomic<unsigned long long> attr_mask{0};
    static std::atomic<int> per_sm_cached{0};
    static std::atomic<int> sm_cached{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::THREADS, Cfg::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        per_sm_cached.store(per_sm < 1 ? 1 : per_sm, std::memory_order_release);
        sm_cached.store(sms, std::memory_order_release);
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    const long long total = (long long)((p.M + BM - 1) / BM) * ((p.N + BN - 1) / BN) * p.batch * p.splits;
    long long grid = (long long)per_sm_cached.load(std::memory_order_acquire) * sm_cached.load(std::memory_order_acquire);
    if (grid > total) grid = total;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(p); count_launch();
    return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, bool AK, bool BKM, bool VEC>
cudaError_t launch_cfg(const GemmF64Args& p, cudaStream_t st, bool persistent) {
    if (persistent) return launch_persistent<BM, BN, WM, WN, AK, BKM, VEC>(p, st);
    constexpr int BK = 16, STAGES = 3;
    using Cfg = GemmF64Cfg<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    auto kern = gemm_f64_kernel<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    // the shared-memory opt-in is per function and device; remember it per device
    static std::atomic<unsigned long long> attr_mask{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cfg::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    dim3 grid((p.M + BM - 1) / BM, (p.N + BN - 1) / BN, p.batch * p.splits);
    kern<<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(p); count_launch();
    return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, bool AK, bool BKM>
cudaError_t launch_vec(const GemmF64Args& p, bool vec, cudaStream_t st, bool persistent) {
    return vec ? launch_cfg<BM, BN, WM, WN, AK, BKM, true>(p, st, persistent)
               : launch_cfg<BM, BN, WM, WN, AK, BKM, false>(p, st, persistent);
}

template <int BM, int BN, int WM, int WN>
cudaError_t launch_layout(const GemmF64Args& p, bool ak, bool bk, bool vec, cudaStream_t st, bool persistent) {
    if (ak && bk) return launch_vec<BM, BN, WM, WN, true, true>(p, vec, st, persistent);
    if (ak && !bk) return launch_vec<BM, BN, WM, WN, true, false>(p, vec, st, persistent);
    if (!ak && bk) return launch_vec<BM, BN, WM, WN, false, true>(p, vec, st, persistent);
    return launch_vec<BM, BN, WM, WN, false, false>(p, vec, st, persistent);
}

bool aligned16(const void* ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

template <int BM, int BN, int WM, int WN, bool AK, bool BKM, bool VEC>
cudaError_t launch_grouped_cfg(const GemmF64Args* groups, const int* start, int ngroups, int total, int sm_count,
                               int max_ctas, cudaStream_t st) {
    constexpr int BK = 16, STAGES = 3;
    using Cfg = GemmF64Cfg<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    auto kern = gemm_f64_grouped_kernel<BM, BN, BK, WM, WN, STAGES, AK, BKM, VEC>;
    static std::atomic<unsigned long long> attr_mask{0};
    static std::atomic<int> per_sm_cached{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::THREADS, Cfg::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        per_sm_cached.store(per_sm < 1 ? 1 : per_sm, std::memory_order_release);
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    long long grid = (long long)per_sm_cached.load(std::memory_order_acquire) * sm_count;
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid > total) grid = total;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(groups, start, ngroups); count_launch();
    return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN>
cudaError_t launch_grouped_layout(const GemmF64Args* groups, const int* start, int ngroups, int total, int sm,
                                  int max_ctas, bool ak, bool bk, bool vec, cudaStream_t st) {
#define DONOF_GL(A_, B_)                                                                                       \
    return vec ? launch_grouped_cfg<BM, BN, WM, WN, A_, B_, true>(groups, start, ngroups, total, sm, max_ctas, st) \
               : launch_grouped_cfg<BM, BN, WM, WN, A_, B_, false>(groups, start, ngroups, total, sm, max_ctas, st)
    if (ak && bk) DONOF_GL(true, true);
    if (ak && !bk) DONOF_GL(true, false);
    if (!ak && bk) DONOF_GL(false, true);
    DONOF_GL(false, false);
#undef DONOF_GL
}

}  // namespace

bool gemm_f64_vec_ok(bool a_kmajor, bool b_kmajor, const GemmF64Args& p) {
    int splits = p.splits < 1 ? 1 : p.splits;
    const int kchunk = (splits == 1 || p.kchunk <= 0) ? p.K : p.kchunk;
    const bool va = aligned16(p.A) && (p.lda % 2 == 0) && (p.strideA % 2 == 0) &&
                    (a_kmajor ? (p.K % 2 == 0 && kchunk % 2 == 0) : (p.M % 2 == 0));
    const bool vb = aligned16(p.B) && (p.ldb % 2 == 0) && (p.strideB % 2 == 0) &&
                    (b_kmajor ? (p.K % 2 == 0 && kchunk % 2 == 0) : (p.N % 2 == 0));
    return va && vb;
}

int gemm_f64_tiles(const GemmF64Args& p, GemmTile tile) {
    const int bm = tile == GemmTile::Large ? 128 : (tile == GemmTile::Tiny ? 32 : 64);
    const int bn = tile == GemmTile::Tiny ? 32 : 64;
    if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return 0;
    return ((p.M + bm - 1) / bm) * ((p.N + bn - 1) / bn) * p.batch * (p.splits < 1 ? 1 : p.splits);
}

int gemm_f64_grouped(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, bool vec, GemmTile tile,
                     const GemmF64Args* groups, const int* start, int ngroups, int total_tiles, int max_ctas) {
    if (ngroups <= 0 || total_tiles <= 0) return DONOF_OK;
    cudaError_t e;
    if (tile == GemmTile::Large)
        e = launch_grouped_layout<128, 64, 4, 2>(groups, start, ngroups, total_tiles, ctx->sm_count, max_ctas,
                                                 a_kmajor, b_kmajor, vec, st);
    else if (tile == GemmTile::Small)
        e = launch_grouped_layout<64, 64, 2, 2>(groups, start, ngroups, total_tiles, ctx->sm_count, max_ctas,
                                                a_kmajor, b_kmajor, vec, st);
    else if (tile == GemmTile::SmallW8)
        e = launch_grouped_layout<64, 64, 2, 4>(groups, start, ngroups, total_tiles, ctx->sm_count, max_ctas,
                                                a_kmajor, b_kmajor, vec, st);
    else
        e = launch_grouped_layout<32, 32, 2, 2>(groups, start, ngroups, total_tiles, ctx->sm_count, max_ctas,
                                                a_kmajor, b_kmajor, vec, st);
    if (e != cudaSuccess) {
        set_error(ctx, "gemm_f64_grouped launch (%d groups, %d tiles): %s", ngroups, total_tiles,
                  cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    return DONOF_OK;
}

int gemm_f64(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, GemmF64Args p,
             GemmTile tile) {
    return gemm_f64_run(ctx, st, a_kmajor, b_kmajor, p, tile, false);
}

int gemm_f64_run(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, GemmF64Args p,
                 GemmTile tile, bool persistent) {
    if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return DONOF_OK;
    if (p.splits < 1) p.splits = 1;
    if (p.splits == 1 || p.kchunk <= 0) p.kchunk = p.K;
    // 16-byte staging needs 16-byte aligned bases and even strides along and
    // across the copied direction, and an even extent along it.
    const bool va = aligned16(p.A) && (p.lda % 2 == 0) && (p.strideA % 2 == 0) &&
                    (a_kmajor ? (p.K % 2 == 0 && p.kchunk % 2 == 0) : (p.M % 2 == 0));
    const bool vb = aligned16(p.B) && (p.ldb % 2 == 0) && (p.strideB % 2 == 0) &&
                    (b_kmajor ? (p.K % 2 == 0 && p.kchunk % 2 == 0) : (p.N % 2 == 0));
    const bool vec = va && vb;
    cudaError_t e;
    if (tile == GemmTile::Large)
        e = launch_layout<128, 64, 4, 2>(p, a_kmajor, b_kmajor, vec, st, persistent);
    else if (tile == GemmTile::Small)
        e = launch_layout<64, 64, 2, 2>(p, a_kmajor, b_kmajor, vec, st, persistent);
    else if (tile == GemmTile::SmallW8)
        e = launch_layout<64, 64, 2, 4>(p, a_kmajor, b_kmajor, vec, st, persistent);
    else
        e = launch_layout<32, 32, 2, 2>(p, a_kmajor, b_kmajor, vec, st, persistent);
    if (e != cudaSuccess) {
        set_error(ctx, "gemm_f64 launch (M=%d N=%d K=%d batch=%d splits=%d): %s", p.M, p.N, p.K,
                  p.batch, p.splits, cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    return DONOF_OK;
}

GemmTile pick_tile(donof_ctx* ctx, int M, int N, int K, bool can_split, int* splits_out) {
    struct Cand { GemmTile t; int bm, bn; };
    const Cand cands[3] = {{GemmTile::Large, 128, 64}, {GemmTile::Small, 64, 64}, {GemmTile::Tiny, 32, 32}};
    const int want = 2 * ctx->sm_count;
    for (int c = 0; c < 3; ++c) {
        const long long tiles = (long long)((M + cands[c].bm - 1) / cands[c].bm) * ((N + cands[c].bn - 1) / cands[c].bn);
        int splits = 1;
        if (can_split && tiles < want) {
            const int max_splits = K / 64 > 1 ? K / 64 : 1;  // keep every split >= 64 deep
            long long s = (want + tiles - 1) / tiles;
            splits = (int)(s < max_splits ? s : max_splits);
        }
        if (tiles * splits >= ctx->sm_count || c == 2) {
            *splits_out = splits;
            return cands[c].t;
        }
    }
    *splits_out = 1;
    return GemmTile::Tiny;
}

int gemm_f64_auto(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N,
                  int K, const double* A, long long lda, const double* B, long long ldb,
                  double* C, long long ldc, double alpha, double beta, DevBuf* part) {
    GemmF64Args p{};
    p.M = M; p.N = N; p.K = K;
    p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
    p.alpha = alpha; p.beta = beta; p.batch = 1; p.splits = 1; p.kchunk = K;
    int splits = 1, kchunk = K;
    const GemmTile tile = pick_tile(ctx, M, N, K, part != nullptr, &splits);
    if (splits > 1) {
        kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
        splits = (K + kchunk - 1) / kchunk;
    }
    if (splits > 1) {
        const long long per = (long long)M * N;
        DONOF_CHECK(part->ensure(ctx, sizeof(double) * per * splits));
        GemmF64Args q = p;
        q.C = part->as<double>(); q.ldc = M; q.splits = splits;
        q.kchunk = kchunk;
        q.strideSplit = per; q.beta = 0.0;
        DONOF_CHECK(gemm_f64(ctx, st, a_kmajor, b_kmajor, q, tile));
        if (ldc == M) return splitk_reduce(ctx, st, q.C, per, splits, per, C, beta);
        // strided destination: reduce column by column
        for (int j = 0; j < N; ++j)
            DONOF_CHECK(splitk_reduce(ctx, st, q.C + (long long)j * M, per, splits, M,
                                      C + (long long)j * ldc, beta));
        return DONOF_OK;
    }
    return gemm_f64(ctx, st, a_kmajor, b_kmajor, p, tile);
}

// ---------------------------------------------------------------------------
// Autotuner.  The first call of a GEMM shape (per device, outside stream
// capture) times every candidate configuration on the call's own operands with
// CUDA events and keeps the fastest; later calls of that shape, captured graphs
// included, launch it directly.  Without split-K every tile shape sums each
// output element over K in the same order, so the candidates write identical
// results; with split-K the chosen partition is fixed once per process, so a
// shape gives the same rounding in every later call.
namespace {

struct TuneKey {
    int dev, M, N, K, batch, ak, bk, kind;
    bool operator<(const TuneKey& o) const {
        return std::tie(dev, M, N, K, batch, ak, bk, kind) < std::tie(o.dev, o.M, o.N, o.K, o.batch, o.ak, o.bk, o.kind);
    }
};
struct TuneVal {
    GemmTile tile;
    int splits;
    bool persistent = false;  // gemm_f64_persistent_kernel instead of one CTA per tile
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
}

bool tune_lookup(const TuneKey& k, TuneVal* v) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(k);
    if (it == g_tune.end()) return false;
    *v = it->second;
    return true;
}

void tune_store(const TuneKey& k, const TuneVal& v) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune.emplace(k, v);
}

// Time run(candidate) for each candidate (one warm-up, two timed runs); returns
// the index of the fastest, or -1 if a launch failed.
template <class Run>
int time_candidates(donof_ctx* ctx, cudaStream_t st, int count, Run run) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return -1;
    }
    int best = -1;
    float best_ms = 0.f;
    for (int c = 0; c < count; ++c) {
        if (run(c) != DONOF_OK) { best = -1; break; }
        cudaEventRecord(e0, st);
        int rc = run(c);
        if (rc == DONOF_OK) rc = run(c);
        cudaEventRecord(e1, st);
        if (rc != DONOF_OK || cudaEventSynchronize(e1) != cudaSuccess) { best = -1; break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best < 0 || ms < best_ms) { best = c; best_ms = ms; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best < 0) set_error(ctx, "GEMM autotuning failed: %s", cudaGetErrorString(cudaGetLastError()));
    return best;
}

constexpr int kNT = 4;
const GemmTile kTiles[kNT] = {GemmTile::Large, GemmTile::Small, GemmTile::Tiny, GemmTile::SmallW8};
const int kTileBM[kNT] = {128, 64, 32, 64}, kTileBN[kNT] = {64, 64, 32, 64};

}  // namespace

int gemm_f64_tuned(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, const GemmF64Args& p,
                   GemmTile heuristic) {
    const bool tunable = p.splits == 1 && p.beta == 0.0 && p.skip_le == nullptr && p.skip_nz == nullptr &&
                         p.B_ptr == nullptr;
    if (!tunable) return gemm_f64(ctx, st, a_kmajor, b_kmajor, p, heuristic);
    const TuneKey key{ctx->device, p.M, p.N, p.K, p.batch, a_kmajor, b_kmajor, 0};
    TuneVal v;
    if (tune_lookup(key, &v)) return gemm_f64_run(ctx, st, a_kmajor, b_kmajor, p, v.tile, v.persistent);
    if (capturing(st)) return gemm_f64(ctx, st, a_kmajor, b_kmajor, p, heuristic);
    // every tile shape, one CTA per tile and persistent
    const int best = time_candidates(ctx, st, 2 * kNT, [&](int c) {
        return gemm_f64_run(ctx, st, a_kmajor, b_kmajor, p, kTiles[c % kNT], c >= kNT);
    });
    if (best < 0) return DONOF_ERR_CUDA;
    tune_store(key, TuneVal{kTiles[best % kNT], 1, best >= kNT});
    return DONOF_OK;  // every candidate wrote the same C
}

namespace {

// The (tile, split) configuration gemm_f64_partials uses for a shape: the
// cached autotuner choice, else (outside stream capture) timed now on the
// given operands, else (while capturing) the heuristic.  *splits_out: the
// number of partial products that configuration writes.
int partials_choice(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K,
                    const double* A, long long lda, const double* B, long long ldb, DevBuf* part, TuneVal* out,
                    GemmF64Args* q_out, int* splits_out) {
    GemmF64Args p{};
    p.M = M; p.N = N; p.K = K;
    p.A = A; p.lda = lda; p.B = B; p.ldb = ldb;
    p.alpha = 1.0; p.beta = 0.0; p.batch = 1; p.splits = 1; p.kchunk = K;
    // candidates: each tile shape with about one and about two CTAs per SM
    std::vector<TuneVal> cands;
    {
        int sp = 1;
        const GemmTile h = pick_tile(ctx, M, N, K, true, &sp);
        cands.push_back(TuneVal{h, sp});
        const int max_splits = K / 64 > 1 ? K / 64 : 1;
        for (int t = 0; t < kNT; ++t) {
            const long long tiles = (long long)((M + kTileBM[t] - 1) / kTileBM[t]) * ((N + kTileBN[t] - 1) / kTileBN[t]);
            for (int f = 1; f <= 2; ++f) {
                long long s = (f * (long long)ctx->sm_count + tiles - 1) / tiles;
                if (s > max_splits) s = max_splits;
                if (s < 1) s = 1;
                bool dup = false;
                for (const TuneVal& c : cands) dup = dup || (c.tile == kTiles[t] && c.splits == (int)s);
                if (!dup) cands.push_back(TuneVal{kTiles[t], (int)s});
            }
        }
        const size_t nplain = cands.size();
        for (size_t c = 0; c < nplain; ++c) cands.push_back(TuneVal{cands[c].tile, cands[c].splits, true});
    }
    auto config = [&](const TuneVal& c, GemmF64Args* q, int* ns) {
        *q = p;
        int splits = c.splits, kchunk = K;
        if (splits > 1) {
            kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
            splits = (K + kchunk - 1) / kchunk;
        }
        q->C = part->as<double>(); q->ldc = M;
        if (splits > 1) {
            q->splits = splits;
            q->kchunk = kchunk;
            q->strideSplit = (long long)M * N;
        }
        *ns = splits;
    };
    const TuneKey key{ctx->device, M, N, K, 1, a_kmajor, b_kmajor, 1};
    TuneVal v = cands[0];
    const bool known = tune_lookup(key, &v);
    if (!known && !capturing(st)) {
        int most = 1;
        for (const TuneVal& c : cands) most = c.splits > most ? c.splits : most;
        DONOF_CHECK(part->ensure(ctx, sizeof(double) * (size_t)M * N * most));
        const int best = time_candidates(ctx, st, (int)cands.size(), [&](int c) {
            GemmF64Args q;
            int ns;
            config(cands[c], &q, &ns);
            return gemm_f64_run(ctx, st, a_kmajor, b_kmajor, q, cands[c].tile, cands[c].persistent);
        });
        if (best < 0) return DONOF_ERR_CUDA;
        v = cands[best];
        tune_store(key, v);
    }
    DONOF_CHECK(part->ensure(ctx, sizeof(double) * (size_t)M * N * (v.splits > 1 ? v.splits : 1)));
    *out = v;
    config(v, q_out, splits_out);
    return DONOF_OK;
}

}  // namespace

int gemm_f64_partials(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K,
                      const double* A, long long lda, const double* B, long long ldb, DevBuf* part,
                      const double** out, int* nparts) {
    TuneVal v;
    GemmF64Args q;
    int splits = 1;
    DONOF_CHECK(partials_choice(ctx, st, a_kmajor, b_kmajor, M, N, K, A, lda, B, ldb, part, &v, &q, &splits));
    DONOF_CHECK(gemm_f64_run(ctx, st, a_kmajor, b_kmajor, q, v.tile, v.persistent));
    *out = part->as<double>();
    *nparts = splits;
    return DONOF_OK;
}

int gemm_f64_partials_splits(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K,
                             const double* A, long long lda, const double* B, long long ldb, DevBuf* part,
                             int* splits, int* kchunk) {
    TuneVal v;
    GemmF64Args q;
    DONOF_CHECK(partials_choice(ctx, st, a_kmajor, b_kmajor, M, N, K, A, lda, B, ldb, part, &v, &q, splits));
    *kchunk = (*splits > 1) ? q.kchunk : K;
    return DONOF_OK;
}

__global__ void splitk_reduce_kernel(const double* __restrict__ part, long long stride, int splits,
                                     long long count, double* __restrict__ out, double beta) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < splits; ++k) s += part[i + k * stride];
        out[i] = (beta != 0.0) ? s + beta * out[i] : s;
    }
}

int splitk_reduce(donof_ctx* ctx, cudaStream_t st, const double* part, long long stride,
                  int splits, long long count, double* out, double beta) {
    const int threads = 256;
    long long blocks = (count + threads - 1) / threads;
    if (blocks > 4 * (long long)ctx->sm_count) blocks = 4 * (long long)ctx->sm_count;
    if (blocks < 1) blocks = 1;
    splitk_reduce_kernel<<<(unsigned)blocks, threads, 0, st>>>(part, stride, splits, count, out, beta); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

}  // namespace donof

extern "C" int donof_autotune_entries(void) {
    std::lock_guard<std::mutex> g(donof::g_tune_mu);
    return (int)donof::g_tune.size();
}
