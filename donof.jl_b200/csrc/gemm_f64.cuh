// FP64 tensor-core GEMM for sm_100a (DMMA, mma.sync m16n8k4 .f64).
//
// tcgen05.mma has no f64 kind, so the plain FP64 form of the hot path runs on
// the FP64 MMA pipe through warp-level mma.sync.  The kernel is a strided,
// batched, optionally split-K GEMM
//     C_z(i,j) = alpha * sum_k A_z(i,k) B_z(k,j) + beta * C_z(i,j)
// with either operand K-contiguous or M/N-contiguous, so every contraction of
// the path (three-index transforms, the Lagrangian GEMM, the small C^T X
// products, the exponential of the rotation generator) uses the same kernel
// without transposing copies in HBM.
//
// Operand addressing (0-based):
//   A(i,k) = AK ? A[i*lda + k] : A[i + k*lda]
//   B(k,j) = BK ? B[k + j*ldb] : B[k*ldb + j]
//   C(i,j) = C[i + j*ldc]                  (column-major output)
// Batch z = blockIdx.z / splits adds z*stride{A,B,C}; split s = blockIdx.z %
// splits covers K range [s*kchunk, min(K, (s+1)*kchunk)) and, when splits > 1,
// writes its partial result to C + s*strideSplit (beta is then ignored).
//
// Staging: a STAGES-deep cp.async ring (16-byte copies when the operand is
// 16-byte aligned with even strides, 8-byte otherwise), zero-filled outside
// the matrix; shared-memory rows are padded so the fragment reads of a warp
// hit every bank pair exactly twice (the minimum for 256 bytes): row strides
// are 4 (mod 16) doubles.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace donof {

struct GemmF64Args {
    int M, N, K;
    const double* A;
    long long lda, strideA;
    const double* B;
    long long ldb, strideB;
    double* C;
    long long ldc, strideC;
    double alpha, beta;
    int batch;
    int splits;
    int kchunk;
    long long strideSplit;
    // Optional device-side gates, read at kernel start (so that data-dependent
    // control flow needs no host round trip and survives graph capture):
    //   skip when skip_le != nullptr and *skip_le <= skip_level
    //   skip when skip_nz != nullptr and *skip_nz != 0
    const int* skip_le;
    int skip_level;
    const int* skip_nz;
    // Optional indirect B operand: when B_ptr != nullptr, B = *B_ptr.
    const double* const* B_ptr;
};

namespace gemm_detail {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src, bool valid) {
    const uint32_t d = smem_u32(dst);
    const int sz = valid ? BYTES : 0;  // src-size 0 zero-fills the destination
    if constexpr (BYTES == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(sz));
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz));
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void mma_f64_16x8x4(double (&c)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// K depth of one FP64 MMA instruction (4, 8 or 16); sm_90 and later have the
// m16n8k8 and m16n8k16 shapes, which move the same work in fewer instructions.
constexpr int kMmaK = 8;

// Fragment layouts (g = lane / 4, t = lane % 4), element e of a thread:
//   A (16 x K, row):  row g + 8 (e % 2), column t + 4 (e / 2),  e < K / 2
//   B (K x 8,  col):  row t + 4 e,       column g,              e < K / 4
//   C/D (16 x 8):     row g + 8 (e / 2), column 2 t + e % 2,    e < 4
template <int K>
__device__ __forceinline__ void mma_f64(double (&c)[4], const double (&a)[K / 2], const double (&b)[K / 4]) {
    if constexpr (K == 4) {
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(b[0]));
    } else if constexpr (K == 8) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
    } else {
        static_assert(K == 16, "FP64 MMA depth must be 4, 8 or 16");
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
            "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
              "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
    }
}

}  // namespace gemm_detail

template <int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, bool AK, bool BKM, bool VEC>
struct GemmF64Cfg {
    static constexpr int THREADS = 32 * WARPS_M * WARPS_N;
    static constexpr int WTM = BM / WARPS_M;  // warp tile rows
    static constexpr int WTN = BN / WARPS_N;  // warp tile cols
    static constexpr int MI = WTM / 16;
    static constexpr int NI = WTN / 8;
    // padded shared-memory strides (in doubles)
    // (both forms: a half-warp's 16 fragment reads land on 16 distinct bank pairs,
    // since the 4 threads of a group step the row by 4 doubles mod 16)
    static constexpr int SA = AK ? (BK + 4) : (BM + 4);
    static constexpr int SB = BKM ? (BK + 4) : (BN + 4);
    static constexpr int A_ELEMS = AK ? BM * SA : BK * SA;
    static constexpr int B_ELEMS = BKM ? BN * SB : BK * SB;
    static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS;
    static constexpr size_t SMEM_BYTES = sizeof(double) * (size_t)STAGES * STAGE_ELEMS;
    static constexpr int VW = VEC ? 2 : 1;  // doubles per copy
    static_assert(WTM % 16 == 0 && WTN % 8 == 0, "warp tile must be a multiple of 16x8");
    static_assert(BK % 4 == 0, "BK must be a multiple of 4");
};

// One output tile (bx, by) of batch/split index bz = z * splits + split, in
// four steps that a kernel can interleave across tiles: init (operands,
// extents, gates), prologue (the first STAGES - 1 cp.async stages, one commit
// group each), mainloop (acc += A B over the tile's K range) and epilogue
// (alpha, beta, column-major store).  gemm_f64_kernel runs them in order for
// its one tile; the grouped persistent kernel issues the next tile's prologue
// before the current tile's epilogue.  Both use the same staging and MMA order,
// so they write identical results.
template <int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, bool AK, bool BKM, bool VEC>
struct GemmTileF64 {
    using Cfg = GemmF64Cfg<BM, BN, BK, WARPS_M, WARPS_N, STAGES, AK, BKM, VEC>;
    static constexpr int KS = gemm_detail::kMmaK;
    static_assert(BK % KS == 0, "BK must be a multiple of the MMA depth");
    using Acc = double[Cfg::MI][Cfg::NI][4];

    const double* A;
    const double* B;
    double* Cout;
    long long lda, ldb, ldc;
    double alpha, beta;
    int M, N, m0, n0, kbeg, kend, nk;
    bool use_beta, skip;

    __device__ __forceinline__ void init(const GemmF64Args& p, int bx, int by, int bz) {
        const int z = bz / p.splits;
        const int split = bz % p.splits;
        m0 = bx * BM;
        n0 = by * BN;
        kbeg = split * p.kchunk;
        kend = min(p.K, kbeg + p.kchunk);
        nk = (kend > kbeg) ? (kend - kbeg + BK - 1) / BK : 0;
        A = p.A + (long long)z * p.strideA;
        B = (p.B_ptr != nullptr ? *p.B_ptr : p.B) + (long long)z * p.strideB;
        Cout = p.C + (long long)z * p.strideC + (p.splits > 1 ? (long long)split * p.strideSplit : 0LL);
        lda = p.lda; ldb = p.ldb; ldc = p.ldc;
        M = p.M; N = p.N;
        alpha = p.alpha; beta = p.beta;
        use_beta = (p.splits == 1) && (p.beta != 0.0);
        skip = (p.skip_le != nullptr && *p.skip_le <= p.skip_level) || (p.skip_nz != nullptr && *p.skip_nz != 0);
    }

    static __device__ __forceinline__ double* As(double* smem, int s) { return smem + (size_t)s * Cfg::STAGE_ELEMS; }
    static __device__ __forceinline__ double* Bs(double* smem, int s) {
        return smem + (size_t)s * Cfg::STAGE_ELEMS + Cfg::A_ELEMS;
    }

    __device__ __forceinline__ void load(double* smem, int stage, int k0) const {
        const int tid = threadIdx.x;
        double* as = As(smem, stage);
        double* bs = Bs(smem, stage);
        // ---- A tile: BM x BK
        if constexpr (AK) {
            constexpr int CPR = BK / Cfg::VW;  // copies per row
            for (int c = tid; c < BM * CPR; c += Cfg::THREADS) {
                const int i = c / CPR, kk = (c % CPR) * Cfg::VW;
                const int gi = m0 + i, gk = k0 + kk;
                const bool ok = (gi < M) && (gk < kend);
                const double* src = ok ? (A + (long long)gi * lda + gk) : A;
                gemm_detail::cp_async<8 * Cfg::VW>(as + i * Cfg::SA + kk, src, ok);
            }
        } else {
            constexpr int CPR = BM / Cfg::VW;
            for (int c = tid; c < BK * CPR; c += Cfg::THREADS) {
                const int kk = c / CPR, i = (c % CPR) * Cfg::VW;
                const int gi = m0 + i, gk = k0 + kk;
                const bool ok = (gi < M) && (gk < kend);
                const double* src = ok ? (A + gi + (long long)gk * lda) : A;
                gemm_detail::cp_async<8 * Cfg::VW>(as + kk * Cfg::SA + i, src, ok);
            }
        }
        // ---- B tile: BK x BN
        if constexpr (BKM) {
            constexpr int CPR = BK / Cfg::VW;
            for (int c = tid; c < BN * CPR; c += Cfg::THREADS) {
                const int j = c / CPR, kk = (c % CPR) * Cfg::VW;
                const int gj = n0 + j, gk = k0 + kk;
                const bool ok = (gj < N) && (gk < kend);
                const double* src = ok ? (B + gk + (long long)gj * ldb) : B;
                gemm_detail::cp_async<8 * Cfg::VW>(bs + j * Cfg::SB + kk, src, ok);
            }
        } else {
            constexpr int CPR = BN / Cfg::VW;
            for (int c = tid; c < BK * CPR; c += Cfg::THREADS) {
                const int kk = c / CPR, j = (c % CPR) * Cfg::VW;
                const int gj = n0 + j, gk = k0 + kk;
                const bool ok = (gj < N) && (gk < kend);
                const double* src = ok ? (B + (long long)gk * ldb + gj) : B;
                gemm_detail::cp_async<8 * Cfg::VW>(bs + kk * Cfg::SB + j, src, ok);
            }
        }
    }

    __device__ __forceinline__ void prologue(double* smem) const {
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) {
            if (s < nk) load(smem, s, kbeg + s * BK);
            gemm_detail::cp_async_commit();
        }
    }

    __device__ __forceinline__ void mainloop(double* smem, Acc& acc) const {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int g = lane >> 2;  // groupID
        const int t = lane & 3;   // threadID_in_group
        const int wrow = (warp % WARPS_M) * Cfg::WTM;
        const int wcol = (warp / WARPS_M) * Cfg::WTN;
#pragma unroll
        for (int a = 0; a < Cfg::MI; ++a)
#pragma unroll
            for (int b = 0; b < Cfg::NI; ++b)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.0;
        for (int kt = 0; kt < nk; ++kt) {
            gemm_detail::cp_async_wait<STAGES - 2>();
            __syncthreads();
            {
                const int nt = kt + STAGES - 1;
                if (nt < nk) load(smem, nt % STAGES, kbeg + nt * BK);
                gemm_detail::cp_async_commit();
            }
            const double* as = As(smem, kt % STAGES);
            const double* bs = Bs(smem, kt % STAGES);
#pragma unroll
            for (int kk = 0; kk < BK; kk += KS) {
                double af[Cfg::MI][KS / 2];
                double bf[Cfg::NI][KS / 4];
#pragma unroll
                for (int a = 0; a < Cfg::MI; ++a) {
#pragma unroll
                    for (int e = 0; e < KS / 2; ++e) {
                        const int r = wrow + a * 16 + g + 8 * (e & 1);
                        const int k = kk + t + 4 * (e >> 1);
                        af[a][e] = AK ? as[r * Cfg::SA + k] : as[k * Cfg::SA + r];
                    }
                }
#pragma unroll
                for (int b = 0; b < Cfg::NI; ++b) {
                    const int cidx = wcol + b * 8 + g;
#pragma unroll
                    for (int e = 0; e < KS / 4; ++e) {
                        const int k = kk + t + 4 * e;
                        bf[b][e] = BKM ? bs[cidx * Cfg::SB + k] : bs[k * Cfg::SB + cidx];
                    }
                }
#pragma unroll
                for (int a = 0; a < Cfg::MI; ++a)
#pragma unroll
                    for (int b = 0; b < Cfg::NI; ++b) gemm_detail::mma_f64<KS>(acc[a][b], af[a], bf[b]);
            }
        }
    }

    __device__ __forceinline__ void epilogue(const Acc& acc) const {
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int g = lane >> 2;
        const int t = lane & 3;
        const int wrow = (warp % WARPS_M) * Cfg::WTM;
        const int wcol = (warp / WARPS_M) * Cfg::WTN;
#pragma unroll
        for (int a = 0; a < Cfg::MI; ++a) {
#pragma unroll
            for (int b = 0; b < Cfg::NI; ++b) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int i = m0 + wrow + a * 16 + g + ((e >= 2) ? 8 : 0);
                    const int j = n0 + wcol + b * 8 + 2 * t + (e & 1);
                    if (i < M && j < N) {
                        double* dst = Cout + i + (long long)j * ldc;
                        double v = alpha * acc[a][b][e];
                        if (use_beta) v += beta * (*dst);
                        *dst = v;
                    }
                }
            }
        }
    }
};

template <int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, bool AK, bool BKM, bool VEC>
__global__ void __launch_bounds__(32 * WARPS_M * WARPS_N)
gemm_f64_kernel(const GemmF64Args p) {
    extern __shared__ __align__(16) double smem[];
    using Tile = GemmTileF64<BM, BN, BK, WARPS_M, WARPS_N, STAGES, AK, BKM, VEC>;
    Tile T;
    T.init(p, blockIdx.x, blockIdx.y, blockIdx.z);
    if (T.skip) return;
    typename Tile::Acc acc;
    T.prologue(smem);
    T.mainloop(smem, acc);
    gemm_detail::cp_async_wait<0>();
    T.epilogue(acc);
}

// Grouped persistent form: `ngroups` independent GEMMs (one per job of a
// batch; every group with its own sizes, operands, batch count, split-K and
// device-side gates) share one launch.  Group g owns the tiles
// [start[g], start[g + 1]) of a flat work list (tile t of a group is
// (bx, by, bz) = (t % gx, (t / gx) % gy, t / (gx gy)) as in the 3-D grid of
// gemm_f64_kernel); each CTA walks the list with stride gridDim.x and starts
// the cp.async prologue of its next tile before it stores the current one, so
// the loads of the next tile are in flight during the epilogue (the tiles of
// the batch's jobs have short K ranges, where the prologue is a large share).
// CTAs per SM the grouped kernel is compiled for (a register cap): as many as
// fit without spills: 6 (32 x 32), 3 (64 x 64 over 4 warps), 2 (64 x 64 over 8
// warps, 128 x 64).
template <int BM, int BN, int WARPS_M, int WARPS_N>
constexpr int grouped_min_ctas() {
    return BM * BN <= 32 * 32 ? 6 : ((BM * BN <= 64 * 64 && WARPS_M * WARPS_N <= 4) ? 3 : 2);
}

// Persistent form of one GEMM: a grid of about one wave of CTAs walks the
// tiles of gemm_f64_kernel's 3-D grid (in its order, x fastest) and starts the
// cp.async prologue of its next tile before it stores the current one.  Same
// tile routine, so it writes what gemm_f64_kernel writes; the autotuner picks
// between the two.  The device-side gates hold for the whole launch.
template <int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, bool AK, bool BKM, bool VEC>
__global__ void __launch_bounds__(32 * WARPS_M * WARPS_N, (grouped_min_ctas<BM, BN, WARPS_M, WARPS_N>()))
gemm_f64_persistent_kernel(const GemmF64Args p) {
    extern __shared__ __align__(16) double smem[];
    using Tile = GemmTileF64<BM, BN, BK, WARPS_M, WARPS_N, STAGES, AK, BKM, VEC>;
    const int gx = (p.M + BM - 1) / BM, gy = (p.N + BN - 1) / BN;
    const int total = gx * gy * p.batch * p.splits;
    int t = blockIdx.x;
    if (t >= total) return;
    Tile cur;
    cur.init(p, t % gx, (t / gx) % gy, t / (gx * gy));
    if (cur.skip) return;
    cur.prologue(smem);
    typename Tile::Acc acc;
    while (true) {
        cur.mainloop(smem, acc);
        const int tn = t + gridDim.x;
        const bool more = tn < total;
        Tile nxt;
        if (more) {
            nxt.init(p, tn % gx, (tn / gx) % gy, tn / (gx * gy));
            __syncthreads();  // every warp is done with the stages the prologue overwrites
            nxt.prologue(smem);
        }
        cur.epilogue(acc);
        if (!more) break;
        cur = nxt;
        t = tn;
    }
    gemm_detail::cp_async_wait<0>();
}


template <int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, bool AK, bool BKM, bool VEC>
__global__ void __launch_bounds__(32 * WARPS_M * WARPS_N, (grouped_min_ctas<BM, BN, WARPS_M, WARPS_N>()))
gemm_f64_grouped_kernel(const GemmF64Args* __restrict__ groups, const int* __restrict__ start, int ngroups) {
    extern __shared__ __align__(16) double smem[];
    using Tile = GemmTileF64<BM, BN, BK, WARPS_M, WARPS_N, STAGES, AK, BKM, VEC>;
    const int total = start[ngroups];
    int g = 0;
    // next tile at or after t that is not gated off; returns its index (total if none)
    auto next = [&](int t, Tile& T) {
        for (; t < total; t += gridDim.x) {
            while (g + 1 < ngroups && start[g + 1] <= t) ++g;  // t only grows: advance the group
            const GemmF64Args& p = groups[g];
            const int lt = t - start[g];
            const int gx = (p.M + BM - 1) / BM, gy = (p.N + BN - 1) / BN;
            T.init(p, lt % gx, (lt / gx) % gy, lt / (gx * gy));
            if (!T.skip) break;
        }
        return t;
    };
    Tile cur;
    int t = next(blockIdx.x, cur);
    if (t >= total) return;
    cur.prologue(smem);
    typename Tile::Acc acc;
    while (true) {
        cur.mainloop(smem, acc);
        Tile nxt;
        const int tn = next(t + gridDim.x, nxt);
        const bool more = tn < total;
        if (more) {
            __syncthreads();  // every warp is done with the stages the prologue overwrites
            nxt.prologue(smem);
        }
        cur.epilogue(acc);
        if (!more) break;
        cur = nxt;
        t = tn;
    }
    gemm_detail::cp_async_wait<0>();
}

}  // namespace donof
