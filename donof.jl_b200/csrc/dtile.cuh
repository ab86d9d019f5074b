// FP64 tile products for the single-launch (cooperative) kernels of the
// orbital step: the exponential of the rotation generator and the Lagrangian
// tail.  Their matrices are small (nbf <= a few hundred), so every GEMM of a
// stage is split into 32 x TN output tiles spread over the SMs.  A tile
// streams 64-deep K panels of both operands into a ring of shared-memory
// buffers with cp.async (two panels in flight while one is multiplied); each
// of the eight warps multiplies an eighth of every panel on the FP64 tensor
// cores (mma.sync m16n8k4 .f64), and the eight partial tiles are summed
// through shared memory.  A bounded grid barrier separates the stages.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "gemm_f64.cuh"

namespace donof {
namespace dtile {

constexpr int TM = 32;        // tile rows
constexpr int KC = 64;        // K panel depth
constexpr int NBUF = 3;       // panel buffers (ring)
constexpr int AS = 36;        // A panel stride, [k][i] layout (doubles): conflict-free fragment reads
constexpr int ATS = KC + 4;   // A panel stride, [i][k] layout (transposed A)
constexpr int BS = KC + 4;    // B panel stride, [j][k] layout
constexpr int THREADS = 256;  // 8 warps, each on an eighth of every K panel
constexpr int WARPS = THREADS / 32;
constexpr int APANEL = (KC * AS > TM * ATS) ? KC * AS : TM * ATS;  // doubles of one A panel

// Shared memory (doubles) of one tile product with TN output columns: the ring
// of A and B panels, which also holds the final cross-warp sum.
template <int TN>
constexpr int smem_doubles() {
    return (NBUF * (APANEL + TN * BS) > THREADS * TN) ? NBUF * (APANEL + TN * BS) : THREADS * TN;
}

// C(i, j) for i < M, j < N of one GEMM: C = alpha opA(A) opB(B) (+ C when accumulate)
//   opA(i, k) = ta ? A[k + i lda] : A[i + k lda]
//   opB(k, j) = tb ? B[j + k ldb] : B[k + j ldb]
struct Gemm {
    const double* A;
    int lda;
    bool ta;
    const double* B;
    int ldb;
    bool tb;
    double* C;
    int ldc;
    int M, N, K;
    double alpha;
    bool accumulate;
};

template <int TN>
__device__ __forceinline__ int tiles(const Gemm& g) {
    return ((g.M + TM - 1) / TM) * ((g.N + TN - 1) / TN);
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared-memory offset of A element (i, k) of a panel: [k][i] for A as stored,
// [i][k] for a transposed A (both contiguous along the stored fast index).
template <bool TA>
__device__ __forceinline__ int aoff(int i, int k) { return TA ? i * ATS + k : k * AS + i; }

// Stage the K panel [k0, k0 + KC) of the tile (i0, j0) into the A and B panel
// buffers (zeros outside the matrices) as one cp.async group; the general
// path, used at the edges of the matrices and for unaligned operands.
template <int TN, bool TA>
__device__ __forceinline__ void load_panel(const Gemm& g, int i0, int j0, int k0, double* As, double* Bs) {
    const int tid = threadIdx.x;
    for (int e = tid; e < TM * KC; e += THREADS) {
        int i, k;
        if (TA) { k = e % KC; i = e / KC; }  // consecutive threads: consecutive k (contiguous in A)
        else { i = e % TM; k = e / TM; }     // consecutive threads: consecutive i
        double* dst = As + aoff<TA>(i, k);
        const int gi = i0 + i, gk = k0 + k;
        if (gi < g.M && gk < g.K)
            cp_async8(dst, TA ? g.A + gk + (long long)gi * g.lda : g.A + gi + (long long)gk * g.lda);
        else
            *dst = 0.0;
    }
    for (int e = tid; e < KC * TN; e += THREADS) {
        int j, k;
        if (g.tb) { j = e % TN; k = e / TN; }  // consecutive j contiguous in B
        else { k = e % KC; j = e / KC; }       // consecutive k contiguous in B
        double* dst = Bs + j * BS + k;
        const int gj = j0 + j, gk = k0 + k;
        if (gj < g.N && gk < g.K)
            cp_async8(dst, g.tb ? g.B + gj + (long long)gk * g.ldb : g.B + gk + (long long)gj * g.ldb);
        else
            *dst = 0.0;
    }
    cp_async_commit();
}

// Copies of the K panels of one tile, set up once per tile.  Interior tiles of
// 16-byte aligned operands with even leading dimensions (B not transposed)
// take a precomputed per-thread pointer: every thread copies the same pair of
// doubles, contiguous in memory and in the panel, at fixed strides in every
// panel.  Everything else, and the last panel when K is not a multiple of KC,
// goes through load_panel.
template <int TN, bool TA>
struct PanelLoader {
    // A as stored: pairs (i, i+1) along a k row; transposed A: pairs (k, k+1) along a row i
    static constexpr int APER = TA ? KC / 2 : TM / 2;           // pairs per line
    static constexpr int ALINES = THREADS / APER;                // lines per pass
    static constexpr int APASS = (TA ? TM : KC) / ALINES;        // passes
    static constexpr int BPER = KC / 2, BJSTEP = THREADS / BPER;  // B: pairs per column, columns per pass

    bool fast;
    const double* a_src;  // this thread's first A pair of panel 0
    const double* b_src;  // this thread's first B pair of panel 0
    long long a_line;     // A elements between two lines copied by this thread
    long long a_panel;    // A elements between panels
    long long b_jstep;    // B elements between two columns copied by this thread
    int a_dst, b_dst;     // offsets in the panel buffers

    __device__ __forceinline__ PanelLoader(const Gemm& g, int i0, int j0) {
        const int tid = threadIdx.x;
        fast = !g.tb && (g.lda & 1) == 0 && (g.ldb & 1) == 0 &&
               ((reinterpret_cast<uintptr_t>(g.A) | reinterpret_cast<uintptr_t>(g.B)) & 15) == 0 &&
               i0 + TM <= g.M && j0 + TN <= g.N;
        const int ap = 2 * (tid % APER), al = tid / APER;  // pair offset within the line, line
        if (TA) {  // line = row i (k contiguous)
            a_src = g.A + ap + (long long)(i0 + al) * g.lda;
            a_panel = KC;
            a_dst = aoff<true>(al, ap);
        } else {   // line = k row (i contiguous)
            a_src = g.A + (i0 + ap) + (long long)al * g.lda;
            a_panel = (long long)KC * g.lda;
            a_dst = aoff<false>(ap, al);
        }
        a_line = (long long)ALINES * g.lda;
        const int bk = 2 * (tid % BPER), bj = tid / BPER;
        b_src = g.B + bk + (long long)(j0 + bj) * g.ldb;
        b_jstep = (long long)BJSTEP * g.ldb;
        b_dst = bj * BS + bk;
    }

    __device__ __forceinline__ void load(const Gemm& g, int i0, int j0, int p, double* As, double* Bs) const {
        if (fast && (p + 1) * KC <= g.K) {
            const double* sa = a_src + p * a_panel;
            const double* sb = b_src + p * KC;
            constexpr int ADST = TA ? ALINES * ATS : ALINES * AS;  // panel offset between passes
#pragma unroll
            for (int r = 0; r < APASS; ++r) cp_async16(As + a_dst + r * ADST, sa + r * a_line);
#pragma unroll
            for (int r = 0; r < TN / BJSTEP; ++r) cp_async16(Bs + b_dst + r * BJSTEP * BS, sb + r * b_jstep);
            cp_async_commit();
        } else {
            load_panel<TN, TA>(g, i0, j0, p * KC, As, Bs);
        }
    }
};

// One 32 x TN output tile (index t of the GEMM's tiles, column-major over the
// tile grid) with A read as stored (TA = false) or transposed (TA = true; must
// equal g.ta).  sm holds smem_doubles<TN>() doubles.  The caller's CTA has
// THREADS threads; every thread must call this.
template <int TN, bool TA>
__device__ void tile_t(const Gemm& g, int t, double* sm) {
    static_assert(TN == 16 || TN == 32, "tile width");
    constexpr int NI = TN / 8;      // n8 blocks
    constexpr int MI = TM / 16;     // m16 blocks
    constexpr int KW = KC / WARPS;  // K per warp per panel
    static_assert(KW % 4 == 0, "k steps");
    const int mt = (g.M + TM - 1) / TM;
    const int i0 = (t % mt) * TM, j0 = (t / mt) * TN;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    double acc[MI][NI][4];
#pragma unroll
    for (int a = 0; a < MI; ++a)
#pragma unroll
        for (int b = 0; b < NI; ++b)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.0;
    auto As = [&](int buf) { return sm + buf * (APANEL + TN * BS); };
    auto Bs = [&](int buf) { return sm + buf * (APANEL + TN * BS) + APANEL; };

    const int npan = (g.K + KC - 1) / KC;
    const PanelLoader<TN, TA> ld(g, i0, j0);
    __syncthreads();  // the buffers may still be read by the previous tile
    // prologue: the first NBUF - 1 panels in flight (one commit group each, empty ones too)
#pragma unroll
    for (int p = 0; p < NBUF - 1; ++p) {
        if (p < npan) ld.load(g, i0, j0, p, As(p), Bs(p));
        else cp_async_commit();
    }
    for (int p = 0; p < npan; ++p) {
        // panel p has landed once at most NBUF - 2 newer groups are pending
        cp_async_wait<NBUF - 2>();
        __syncthreads();  // panel p visible to all; buffer (p - 1) % NBUF no longer read
        const int pn = p + NBUF - 1;
        if (pn < npan) ld.load(g, i0, j0, pn, As(pn % NBUF), Bs(pn % NBUF));
        else cp_async_commit();
        const double* A_ = As(p % NBUF);
        const double* B_ = Bs(p % NBUF);
        const int kbeg = warp * KW;
        const int kend = min(kbeg + KW, g.K - p * KC);
        for (int kk = kbeg; kk < kend; kk += 4) {
            double af[MI][2], bf[NI];
#pragma unroll
            for (int mi = 0; mi < MI; ++mi) {
                af[mi][0] = A_[aoff<TA>(mi * 16 + gq, kk + tq)];
                af[mi][1] = A_[aoff<TA>(mi * 16 + gq + 8, kk + tq)];
            }
#pragma unroll
            for (int ni = 0; ni < NI; ++ni) bf[ni] = B_[(ni * 8 + gq) * BS + kk + tq];
#pragma unroll
            for (int mi = 0; mi < MI; ++mi)
#pragma unroll
                for (int ni = 0; ni < NI; ++ni) gemm_detail::mma_f64_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
        }
    }
    cp_async_wait<0>();
    // Thread (warp, lane) finishes the values v = warp + WARPS u of lane's
    // fragment; their destinations (and, when accumulating, old values) are
    // read before the reduction.
    constexpr int V = MI * NI * 4;
    constexpr int U = V / WARPS;
    static_assert(V % WARPS == 0, "fragment split");
    double old[U];
    bool inb[U];
    double* dst[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int v = warp + WARPS * u;
        const int mi = v / (NI * 4), ni = (v / 4) % NI, e = v % 4;
        const int i = i0 + mi * 16 + gq + ((e >= 2) ? 8 : 0);
        const int j = j0 + ni * 8 + 2 * tq + (e & 1);
        inb[u] = i < g.M && j < g.N;
        dst[u] = g.C + i + (long long)j * g.ldc;
        old[u] = (inb[u] && g.accumulate) ? *dst[u] : 0.0;
    }
    __syncthreads();  // every warp is done with the panels: the ring becomes the reduction buffer
    double* red = sm;  // red[(v * WARPS + warp) * 32 + lane]: lane-contiguous, conflict-free
#pragma unroll
    for (int mi = 0; mi < MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < NI; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) red[(((mi * NI + ni) * 4 + e) * WARPS + warp) * 32 + lane] = acc[mi][ni][e];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int v = warp + WARPS * u;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) s += red[(v * WARPS + w) * 32 + lane];
        if (inb[u]) *dst[u] = old[u] + g.alpha * s;
    }
}

// One output tile of g (see tile_t).
template <int TN>
__device__ __forceinline__ void tile(const Gemm& g, int t, double* sm) {
    if (g.ta) tile_t<TN, true>(g, t, sm);
    else tile_t<TN, false>(g, t, sm);
}

// ---------------------------------------------------------------------------
// Bounded grid barrier for a cooperatively launched grid: a monotonic arrival
// counter (zeroed before the launch); barrier number e completes when the
// counter reaches (e + 1) * members.  On a timeout (or when another CTA gave
// up) it records the error -- in the GridSync and, once per launch, in the
// context's failure word -- and returns false; callers then return without
// touching their outputs further.
struct GridSync {
    unsigned count;
    int err;
    unsigned pad[2];
};

constexpr long long BARRIER_CYCLES = 2000000000LL;  // ~1 s

// How a launch's grid barriers wait: the cycle budget (<= 0: BARRIER_CYCLES)
// and the failure word to set on a timeout (may be null).
struct WaitCtl {
    long long cycles;
    int* fail;
};
// The WaitCtl of a context's launches.
inline WaitCtl wait_ctl(const donof_ctx* ctx) {
    return WaitCtl{ctx->wait_limit, ctx->fail_dev ? ctx->fail_dev + FAIL_BARRIER : nullptr};
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// epoch: barriers this CTA has passed (the same in every CTA); incremented here.
// members: the CTAs that take part (gridDim.x for the whole grid; a grouped
// launch gives each job its own GridSync and CTA range).
__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned& epoch, unsigned members, const WaitCtl& w) {
    __shared__ int fail;
    __syncthreads();
    if (threadIdx.x == 0) {
        fail = 0;
        red_release_add(&gs->count, 1u);
        const unsigned target = (epoch + 1) * members;
        const long long budget = w.cycles > 0 ? w.cycles : BARRIER_CYCLES;
        const long long t0 = clock64();
        while (ld_acquire(&gs->count) < target) {
            if (clock64() - t0 > budget || *(volatile int*)&gs->err) {
                // the CTA that gives up first reports it (plain store: the word may be host memory)
                if (atomicExch(&gs->err, 1) == 0 && w.fail) *reinterpret_cast<volatile int*>(w.fail) = 1;
                fail = 1;
                break;
            }
        }
    }
    __syncthreads();
    ++epoch;
    return fail == 0;
}

}  // namespace dtile
}  // namespace donof
