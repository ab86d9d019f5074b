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

#include "gemm_f64.cuh"

namespace donof {
namespace dtile {

constexpr int TM = 32;        // tile rows
constexpr int KC = 64;        // K panel depth
constexpr int NBUF = 3;       // panel buffers (ring)
constexpr int AS = 36;        // A panel stride ([k][i], doubles): conflict-free fragment reads
constexpr int BS = KC + 4;    // B panel stride ([j][k], doubles): conflict-free fragment reads
constexpr int THREADS = 256;  // 8 warps, each on an eighth of every K panel
constexpr int WARPS = THREADS / 32;

// Shared memory (doubles) of one tile product with TN output columns: the ring
// of A and B panels, which also holds the final cross-warp sum.
template <int TN>
constexpr int smem_doubles() {
    return (NBUF * (KC * AS + TN * BS) > THREADS * TN) ? NBUF * (KC * AS + TN * BS) : THREADS * TN;
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

// Stage the K panel [k0, k0 + KC) of the tile (i0, j0) into As[k][i], Bs[j][k]
// (zeros outside the matrices) as one cp.async group.  Non-transposed operands
// with an even leading dimension and a 16-byte aligned base move two doubles
// per copy; interior panels skip the bounds checks.
template <int TN>
__device__ __forceinline__ void load_panel(const Gemm& g, int i0, int j0, int k0, double* As, double* Bs) {
    const int tid = threadIdx.x;
    const bool full_k = k0 + KC <= g.K;
    const bool a16 = !g.ta && (g.lda & 1) == 0 && (reinterpret_cast<uintptr_t>(g.A) & 15) == 0;
    const bool b16 = !g.tb && (g.ldb & 1) == 0 && (reinterpret_cast<uintptr_t>(g.B) & 15) == 0;
    // A: TM x KC elements
    if (a16 && full_k && i0 + TM <= g.M) {
        // every thread copies the same row pair (i, i+1) of every KSTEP-th k row
        constexpr int PER = TM / 2;           // pairs per k row
        constexpr int KSTEP = THREADS / PER;  // k rows per pass
        const int i = 2 * (tid % PER), k = tid / PER;
        const double* src = g.A + (i0 + i) + (long long)(k0 + k) * g.lda;
        double* dst = As + k * AS + i;
#pragma unroll
        for (int r = 0; r < KC / KSTEP; ++r) cp_async16(dst + r * KSTEP * AS, src + (long long)r * KSTEP * g.lda);
    } else if (a16) {
        for (int e = tid; e < TM * KC / 2; e += THREADS) {
            const int i = 2 * (e % (TM / 2)), k = e / (TM / 2);  // pairs (i, i+1), contiguous in A and in As
            double* dst = As + k * AS + i;
            const int gi = i0 + i, gk = k0 + k;
            if (gk < g.K && gi + 1 < g.M) {
                cp_async16(dst, g.A + gi + (long long)gk * g.lda);
            } else {
                dst[0] = (gk < g.K && gi < g.M) ? g.A[gi + (long long)gk * g.lda] : 0.0;
                dst[1] = 0.0;
            }
        }
    } else {
        for (int e = tid; e < TM * KC; e += THREADS) {
            int i, k;
            if (g.ta) { k = e % KC; i = e / KC; }  // consecutive threads: consecutive k (contiguous in A)
            else { i = e % TM; k = e / TM; }       // consecutive threads: consecutive i
            double* dst = As + k * AS + i;
            const int gi = i0 + i, gk = k0 + k;
            if (gi < g.M && gk < g.K)
                cp_async8(dst, g.ta ? g.A + gk + (long long)gi * g.lda : g.A + gi + (long long)gk * g.lda);
            else
                *dst = 0.0;
        }
    }
    // B: KC x TN elements
    if (b16 && full_k && j0 + TN <= g.N) {
        // every thread copies the same k pair of every JSTEP-th column
        constexpr int PER = KC / 2;           // pairs per column
        constexpr int JSTEP = THREADS / PER;  // columns per pass
        const int k = 2 * (tid % PER), j = tid / PER;
        const double* src = g.B + (k0 + k) + (long long)(j0 + j) * g.ldb;
        double* dst = Bs + j * BS + k;
#pragma unroll
        for (int r = 0; r < TN / JSTEP; ++r) cp_async16(dst + r * JSTEP * BS, src + (long long)r * JSTEP * g.ldb);
    } else if (b16) {
        for (int e = tid; e < KC * TN / 2; e += THREADS) {
            const int k = 2 * (e % (KC / 2)), j = e / (KC / 2);  // pairs (k, k+1), contiguous in B and in Bs
            double* dst = Bs + j * BS + k;
            const int gj = j0 + j, gk = k0 + k;
            if (gj < g.N && gk + 1 < g.K) {
                cp_async16(dst, g.B + gk + (long long)gj * g.ldb);
            } else {
                dst[0] = (gj < g.N && gk < g.K) ? g.B[gk + (long long)gj * g.ldb] : 0.0;
                dst[1] = 0.0;
            }
        }
    } else {
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
    }
    cp_async_commit();
}

// Copies of the K panels of one tile, set up once per tile: interior tiles of
// non-transposed, 16-byte aligned operands with even leading dimensions take
// a precomputed per-thread pointer (every thread copies the same row pair of
// A and the same k pair of B in every panel); everything else, and the last
// panel when K is not a multiple of KC, goes through load_panel.
template <int TN>
struct PanelLoader {
    bool fast;
    const double* a_src;  // this thread's first A pair of panel 0
    const double* b_src;  // this thread's first B pair of panel 0
    long long a_kstep;    // A elements between two k rows copied by this thread
    long long b_jstep;    // B elements between two columns copied by this thread
    long long a_panel;    // A elements between panels (KC k rows)
    int a_dst, b_dst;     // offsets in the panel buffers

    static constexpr int APER = TM / 2, AKSTEP = THREADS / APER;  // A: pairs per k row, k rows per pass
    static constexpr int BPER = KC / 2, BJSTEP = THREADS / BPER;  // B: pairs per column, columns per pass

    __device__ __forceinline__ PanelLoader(const Gemm& g, int i0, int j0) {
        const int tid = threadIdx.x;
        fast = !g.ta && !g.tb && (g.lda & 1) == 0 && (g.ldb & 1) == 0 &&
               ((reinterpret_cast<uintptr_t>(g.A) | reinterpret_cast<uintptr_t>(g.B)) & 15) == 0 &&
               i0 + TM <= g.M && j0 + TN <= g.N;
        const int ai = 2 * (tid % APER), ak = tid / APER;
        const int bk = 2 * (tid % BPER), bj = tid / BPER;
        a_src = g.A + (i0 + ai) + (long long)ak * g.lda;
        b_src = g.B + bk + (long long)(j0 + bj) * g.ldb;
        a_kstep = (long long)AKSTEP * g.lda;
        b_jstep = (long long)BJSTEP * g.ldb;
        a_panel = (long long)KC * g.lda;
        a_dst = ak * AS + ai;
        b_dst = bj * BS + bk;
    }

    __device__ __forceinline__ void load(const Gemm& g, int i0, int j0, int p, double* As, double* Bs) const {
        if (fast && (p + 1) * KC <= g.K) {
            const double* sa = a_src + p * a_panel;
            const double* sb = b_src + p * KC;
#pragma unroll
            for (int r = 0; r < KC / AKSTEP; ++r) cp_async16(As + a_dst + r * AKSTEP * AS, sa + r * a_kstep);
#pragma unroll
            for (int r = 0; r < TN / BJSTEP; ++r) cp_async16(Bs + b_dst + r * BJSTEP * BS, sb + r * b_jstep);
            cp_async_commit();
        } else {
            load_panel<TN>(g, i0, j0, p * KC, As, Bs);
        }
    }
};

// One 32 x TN output tile (index t of the GEMM's tiles, column-major over the
// tile grid).  sm holds smem_doubles<TN>() doubles.  The caller's CTA has
// THREADS threads; every thread must call this.
template <int TN>
__device__ void tile(const Gemm& g, int t, double* sm) {
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
    auto As = [&](int buf) { return sm + buf * (KC * AS + TN * BS); };
    auto Bs = [&](int buf) { return sm + buf * (KC * AS + TN * BS) + KC * AS; };

    const int npan = (g.K + KC - 1) / KC;
    const PanelLoader<TN> ld(g, i0, j0);
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
                af[mi][0] = A_[(kk + tq) * AS + mi * 16 + gq];
                af[mi][1] = A_[(kk + tq) * AS + mi * 16 + gq + 8];
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

// ---------------------------------------------------------------------------
// Bounded grid barrier for a cooperatively launched grid: a monotonic arrival
// counter (zeroed before the launch); barrier number e completes when the
// counter reaches (e + 1) * gridDim.x.  On a timeout (or when another CTA gave
// up) it records the error and returns false; callers then return without
// touching their outputs further.
struct GridSync {
    unsigned count;
    int err;
    unsigned pad[2];
};

constexpr long long BARRIER_CYCLES = 2000000000LL;  // ~1 s

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// epoch: barriers this CTA has passed (the same in every CTA); incremented here.
__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned& epoch) {
    __shared__ int fail;
    __syncthreads();
    if (threadIdx.x == 0) {
        fail = 0;
        red_release_add(&gs->count, 1u);
        const unsigned target = (epoch + 1) * gridDim.x;
        const long long t0 = clock64();
        while (ld_acquire(&gs->count) < target) {
            if (clock64() - t0 > BARRIER_CYCLES || *(volatile int*)&gs->err) {
                atomicExch(&gs->err, 1);
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
