// FP64-accurate T1 (tmp_l = B_l C5, the first half of the b_mnP -> b_pqP
// transform of src/utils.jl:19-20 and src/integrals.jl:150-152) on the
// 5th-generation tensor cores, by exact integer products (the Ozaki scheme:
// K. Ozaki, T. Ogita, S. Oishi, S. M. Rump, "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication and
// its applications", Numer. Algorithms 59 (2012) 95-118).
//
// Every row m of B_l (over the contraction index n) and every column q of C5
// is written as S = 7 signed 7-bit digits times a power of two,
//     x = 2^e sum_{i<S} d_i 2^(-7(i+1)),   d_i in [-127, 127],
// with 2^e the smallest power of two above the row's (column's) largest |x|:
// d_i = trunc(128 r_i), r_(i+1) = 128 r_i - d_i, all exact in FP64, and the
// residual is below 2^(-7S) 2^e.  Then
//     tmp_l[m, q] = 2^(ea_m + eb_q) sum_g 2^(-7(g+2)) sum_{i+j=g} (D_i E_j)[m, q]
// where each D_i E_j is an s8 x s8 GEMM whose int32 sums are exact
// (tcgen05.mma kind::i8; |sum| <= 7 * 127^2 * nbf < 2^31 for nbf <= 16384).
// The products with i + j >= S are dropped: they lie below the truncation
// error.  That leaves 28 digit products in 7 int32 TMEM accumulators (one per
// g, 64 columns each), combined in FP64 by the epilogue (exact int32 -> double,
// Horner in 2^-7) and scaled by powers of two.  Since the C5 slices are adjacent in shared memory,
// the products of one b slice with several C5 slices are one MMA of N = 64 x
// (slices) <= 256: 10 MMAs per 32-wide step of n instead of 28.  The result differs from an FP64 GEMM by ~1e-13 of
// the largest |tmp| (tests/test_gpu_ozaki.py states the bound).
//
// b's digit slices are made once per job (it is constant); C5's per call.
// One persistent kernel (ozaki_t1_kernel): a work unit is (aux index l,
// 128-row tile of m); warp 8 streams b's slices (16 KB TMA boxes, no
// multicast) through a ring, warp 9 issues the MMAs, warps 0-7 drain TMEM and
// write tmp in FP64 in the layout the FP64 GEMM path writes.  Every wait is
// bounded; on a timeout the CTA records the failure in the context's failure
// word, drains its copies and MMAs, frees TMEM and exits.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include <atomic>

#include "kernels.cuh"
#include "sm100.cuh"

namespace donof {

namespace oz {

constexpr int S = 7;                        // digit slices per operand
constexpr int EPI_WARPS = 8;                // two per TMEM lane quarter, 32 columns each
constexpr int PRODUCER = EPI_WARPS;         // warp 8: TMA producer
constexpr int ISSUER = EPI_WARPS + 1;       // warp 9: TMEM allocator + MMA issuer
constexpr int NTHREADS = 32 * (EPI_WARPS + 2);
constexpr int KC = 128;                     // n per stage: one 128-byte swizzle row of int8
constexpr int MT = 128;                     // m rows per tile (MMA M)
constexpr int QT = 64;                      // q columns per tile (MMA N per C5 slice)
constexpr int A_BYTES = MT * KC;            // 16 KB: one slice of b over (m tile, n chunk)
constexpr int BS_BYTES = QT * KC;           // 8 KB: one slice of C5 over (q tile, n chunk)
constexpr int B_BYTES = S * BS_BYTES;       // 56 KB: every slice of C5 over (q tile, n chunk)
constexpr int RING = 6;                     // b stages in flight (96 KB)
constexpr int OFF_B = 0;                    // two C5 stages
constexpr int OFF_RING = OFF_B + 2 * B_BYTES;
constexpr int OFF_BAR = OFF_RING + RING * A_BYTES;
constexpr int NBAR = 32;
constexpr int OFF_MISC = OFF_BAR + NBAR * 8;  // tmem base, abort flag
constexpr int SMEM_USED = OFF_MISC + 64;
constexpr int SMEM_ALLOC = SMEM_USED + 1024;  // slack for 1024-B alignment
static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory budget");
static_assert(S * QT <= 512, "TMEM columns");

// barrier indices
constexpr int A_FULL = 0;               // +s (RING): b stage landed
constexpr int A_EMPTY = RING;           // +s: b stage consumed by the MMAs
constexpr int B_FULL = 2 * RING;        // +slot (2): C5 stage landed
constexpr int B_EMPTY = B_FULL + 2;     // +slot: C5 stage consumed
constexpr int ACC_FULL = B_EMPTY + 2;   // every accumulator of a round (unit, q tile) complete
constexpr int GFREE = ACC_FULL + 1;     // +g (S): accumulator g drained and zeroed (count EPI_WARPS)
constexpr int B_END = GFREE + S;        // every MMA of the CTA complete
static_assert(B_END < NBAR, "barrier count");

struct Params {
    int nbf, nbf5, naux;
    int nmt, nkc, nqt;   // tiles of m (128), chunks of n (128), tiles of q (64)
    int resident;        // nqt * nkc <= 2: every C5 stage is loaded once and kept
    const double* sa;    // 2^ea per (m, l): sa[m + nbf*l]
    const double* sb;    // 2^(eb - 14) per q
    double* tmp;         // tmp[m + nbf*q + nbf*nbf5*l]
    int* fail;           // the context's failure word for mbarrier waits
    long long wait;      // cycle budget of every bounded wait (drains excepted)
};

using namespace sm100;

// Exact int32 -> double: the bits 0x43300000:(x ^ 2^31) are the double
// 2^52 + 2^31 + x, from which 2^52 + 2^31 is subtracted exactly (an integer
// op and an FP64 add instead of a conversion-pipe instruction).
__device__ __forceinline__ double exact_f64(int x) {
    return __hiloint2double(0x43300000, x ^ (int)0x80000000) - 4503601774854144.0;
}

// Round r of a CTA = one (unit, q tile): its MMAs accumulate into the 7
// accumulators, then the epilogue drains them.  The b slices of an n chunk are
// consumed from the least significant (i = 6) to the most (i = 0): slice i
// writes accumulators i .. 6 only, so the first MMAs of round r + 1 need only
// accumulator 6, which the epilogue of round r drains (and zeroes) first.  The
// drain of accumulator g is a TMEM load and a store of zeros; its release
// (GFREE[g]) comes right after, and the FP64 arithmetic of the epilogue runs
// while the next round's MMAs already fill the released columns.
__global__ void __launch_bounds__(NTHREADS, 1)
ozaki_t1_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                const Params P) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = saddr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + OFF_MISC);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + OFF_MISC + 16);
    auto bar = [&](int i) { return saddr(&bars[i]); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = gridDim.x;
    const int nunits = P.naux * P.nmt;
    const int my_units = (nunits - (int)blockIdx.x + G - 1) / G;  // unit w = blockIdx.x + u*G
    const int nbst = P.nqt * P.nkc;

    if (threadIdx.x == 0) {
        *abort_flag = 0;
        for (int i = 0; i <= B_END; ++i) mbar_init(bar(i), (i >= GFREE && i < GFREE + S) ? EPI_WARPS : 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == ISSUER) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(saddr(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == PRODUCER) {
        // ------------------------------------------------------------ producer
        // b's slices in the order the MMAs consume them: with C5 resident, slice
        // i of every n chunk before slice i-1 (i = S-1 .. 0), so that a round
        // needs accumulator 0 only for its last nkc stages; with C5 streamed, per
        // q tile and n chunk the C5 stage, then the slices i = S-1 .. 0
        if (lane == 0 && my_units > 0) {
            int it = 0, bs = 0;
            bool ok = true;
            if (P.resident) {
                for (int b = 0; b < nbst; ++b) {
                    const int qt = b / P.nkc, kc = b - qt * P.nkc;
                    mbar_expect_tx(bar(B_FULL + b), (uint32_t)B_BYTES);
                    tma_load_3d(sbase + OFF_B + b * B_BYTES, &map_b, bar(B_FULL + b), kc * KC, qt * QT, 0);
                }
            }
            for (int u = 0; u < my_units && ok; ++u) {
                const int w = (int)blockIdx.x + u * G;
                const int l = w / P.nmt, mt = w - l * P.nmt;
                for (int qt = 0; qt < P.nqt && ok; ++qt) {
                    if (P.resident) {
                        for (int i = S - 1; i >= 0 && ok; --i)
                            for (int kc = 0; kc < P.nkc; ++kc, ++it) {
                                const int s = it % RING;
                                if (!mbar_wait(bar(A_EMPTY + s), (uint32_t)(((it / RING) & 1) ^ 1), abort_flag, P.wait)) {
                                    ok = false;
                                    break;
                                }
                                mbar_expect_tx(bar(A_FULL + s), (uint32_t)A_BYTES);
                                tma_load_4d(sbase + OFF_RING + s * A_BYTES, &map_a, bar(A_FULL + s), kc * KC, mt * MT, i, l);
                            }
                        continue;
                    }
                    for (int kc = 0; kc < P.nkc && ok; ++kc) {
                        if (!P.resident) {
                            const int slot = bs & 1;
                            if (!mbar_wait(bar(B_EMPTY + slot), (uint32_t)(((bs >> 1) & 1) ^ 1), abort_flag, P.wait)) {
                                ok = false;
                                break;
                            }
                            mbar_expect_tx(bar(B_FULL + slot), (uint32_t)B_BYTES);
                            tma_load_3d(sbase + OFF_B + slot * B_BYTES, &map_b, bar(B_FULL + slot), kc * KC, qt * QT, 0);
                            ++bs;
                        }
                        for (int i = S - 1; i >= 0; --i, ++it) {
                            const int s = it % RING;
                            if (!mbar_wait(bar(A_EMPTY + s), (uint32_t)(((it / RING) & 1) ^ 1), abort_flag, P.wait)) {
                                ok = false;
                                break;
                            }
                            mbar_expect_tx(bar(A_FULL + s), (uint32_t)A_BYTES);
                            tma_load_4d(sbase + OFF_RING + s * A_BYTES, &map_a, bar(A_FULL + s), kc * KC, mt * MT, i, l);
                        }
                    }
                }
            }
            // drain: every issued copy has landed before the CTA exits
            for (int j = (it > RING ? it - RING : 0); j < it; ++j)
                mbar_drain(bar(A_FULL + j % RING), (uint32_t)((j / RING) & 1));
            if (P.resident) {
                for (int b = 0; b < nbst; ++b) mbar_drain(bar(B_FULL + b), 0);
            } else {
                for (int j = (bs > 2 ? bs - 2 : 0); j < bs; ++j) mbar_drain(bar(B_FULL + (j & 1)), (uint32_t)((j >> 1) & 1));
            }
        }
    } else if (warp == ISSUER) {
        // ------------------------------------------------------------ MMA issuer
        // accumulator g (TMEM columns [64 g, 64 g + 64)) collects D_i E_j, i + j = g.
        // The C5 slices lie one after the other in shared memory (slice j = rows
        // [64 j, 64 j + 64) of the stage), so D_i times slices j0 .. j0+c-1 is ONE
        // MMA with N = 64 c whose columns land on accumulators i+j0 .. i+j0+c-1.
        // The epilogue zeroes every accumulator it releases: all MMAs accumulate.
        if (lane == 0 && my_units > 0) {
            int s = 0, bs = 0, rnd = 0;  // ring slot of the next b stage, C5 stages, rounds
            uint32_t aph = 0;            // phase of the ring's current pass
            bool ok = true;
            for (int u = 0; u < my_units && ok; ++u) {
                for (int qt = 0; qt < P.nqt && ok; ++qt, ++rnd) {
                    if (P.resident) {
                        const uint64_t bq = sdesc(sbase + OFF_B + qt * P.nkc * B_BYTES, 16, 1024);
                        if (rnd == 0)
                            for (int b = 0; b < nbst && ok; ++b) ok = mbar_wait(bar(B_FULL + b), 0, abort_flag, P.wait);
                        fence_after();
#pragma unroll
                        for (int ii = 0; ii < S; ++ii) {
                            const int i = S - 1 - ii;
                            for (int kc = 0; kc < P.nkc && ok; ++kc) {
                                const uint64_t bd = bq + (uint64_t)((kc * B_BYTES) >> 4);
                                if (kc == 0 && !mbar_wait(bar(GFREE + i), (uint32_t)(rnd & 1), abort_flag, P.wait)) {
                                    ok = false;
                                    break;
                                }
                                if (!mbar_wait(bar(A_FULL + s), aph, abort_flag, P.wait)) {
                                    ok = false;
                                    break;
                                }
                                fence_after();
                                const uint64_t ad = sdesc(sbase + OFF_RING + s * A_BYTES, 16, 1024);
#pragma unroll
                                for (int k4 = 0; k4 < KC / 32; ++k4) {
#pragma unroll
                                    for (int j0 = 0; j0 < S - i; j0 += 4) {
                                        constexpr int kMax = 4;
                                        const int cnt = (S - i - j0) < kMax ? (S - i - j0) : kMax;
                                        umma_i8(tmem + (uint32_t)((i + j0) * QT), ad + (uint64_t)(2 * k4),
                                                bd + (uint64_t)((j0 * BS_BYTES + k4 * 32) >> 4), idesc_i8(MT, QT * cnt), 1u);
                                    }
                                }
                                umma_commit(bar(A_EMPTY + s));
                                if (++s == RING) {
                                    s = 0;
                                    aph ^= 1u;
                                }
                            }
                            if (!ok) break;
                        }
                        if (!ok) break;
                        umma_commit(bar(ACC_FULL));
                        continue;
                    }
                    for (int kc = 0; kc < P.nkc && ok; ++kc) {
                        const int bslot = P.resident ? qt * P.nkc + kc : (bs & 1);
                        const uint32_t bpar = P.resident ? 0u : (uint32_t)((bs >> 1) & 1);
                        if (!mbar_wait(bar(B_FULL + bslot), bpar, abort_flag, P.wait)) {
                            ok = false;
                            break;
                        }
                        fence_after();
                        // descriptors are linear in the shared-memory address (addr >> 4 in the
                        // low 14 bits, no carry below 256 KB): offsets are plain adds
                        const uint64_t bd = sdesc(sbase + OFF_B + bslot * B_BYTES, 16, 1024);
#pragma unroll
                        for (int ii = 0; ii < S; ++ii) {
                            const int i = S - 1 - ii;
                            // accumulator i (and, released before it, i+1 .. 6) free for this round
                            if (kc == 0 && !mbar_wait(bar(GFREE + i), (uint32_t)(rnd & 1), abort_flag, P.wait)) {
                                ok = false;
                                break;
                            }
                            if (!mbar_wait(bar(A_FULL + s), aph, abort_flag, P.wait)) {
                                ok = false;
                                break;
                            }
                            fence_after();
                            const uint64_t ad = sdesc(sbase + OFF_RING + s * A_BYTES, 16, 1024);
#pragma unroll
                            for (int k4 = 0; k4 < KC / 32; ++k4) {
#pragma unroll
                                for (int j0 = 0; j0 < S - i; j0 += 4) {
                                    constexpr int kMax = 4;  // N = 64 cnt <= 256
                                    const int cnt = (S - i - j0) < kMax ? (S - i - j0) : kMax;
                                    umma_i8(tmem + (uint32_t)((i + j0) * QT), ad + (uint64_t)(2 * k4),
                                            bd + (uint64_t)((j0 * BS_BYTES + k4 * 32) >> 4), idesc_i8(MT, QT * cnt), 1u);
                                }
                            }
                            umma_commit(bar(A_EMPTY + s));
                            if (++s == RING) {
                                s = 0;
                                aph ^= 1u;
                            }
                        }
                        if (!ok) break;
                        if (!P.resident) {
                            umma_commit(bar(B_EMPTY + bslot));
                            ++bs;
                        }
                    }
                    if (!ok) break;
                    umma_commit(bar(ACC_FULL));
                }
            }
            umma_commit(bar(B_END));
            mbar_drain(bar(B_END), 0);  // every MMA of this CTA has completed
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 0-7)
        // warp w reads TMEM lanes [32 (w % 4), +32) = rows m = 128 mt + 32 (w % 4) + lane,
        // and columns [32 (w / 4), +32) of every accumulator = q = 64 qt + 32 (w / 4) + k
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t tl = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * 32);
        // zero every accumulator and release it for the first work unit
#pragma unroll
        for (int g = 0; g < S; ++g) tmem_zero32(tl + (uint32_t)(g * QT));
        tmem_wait_st();
        fence_before();
        __syncwarp();
        if (lane == 0)
            for (int g = 0; g < S; ++g) mbar_arrive(bar(GFREE + g));
        int rnd = 0;
        bool ok = true;
        for (int u = 0; u < my_units && ok; ++u) {
            const int w = (int)blockIdx.x + u * G;
            const int l = w / P.nmt, mt = w - l * P.nmt;
            const int m = mt * MT + quarter * 32 + lane;
            const bool mrow = m < P.nbf;
            const double sa = mrow ? P.sa[m + (size_t)P.nbf * l] : 0.0;
            double* dst = P.tmp + (size_t)P.nbf * P.nbf5 * l + m;
            for (int qt = 0; qt < P.nqt; ++qt, ++rnd) {
                int r = 1;
                if (lane == 0) r = mbar_wait(bar(ACC_FULL), (uint32_t)(rnd & 1), abort_flag, P.wait) ? 1 : 0;
                r = __shfl_sync(0xffffffffu, r, 0);
                if (!r) {
                    ok = false;
                    break;
                }
                fence_after();
                // Horner in 2^-7 from the least significant accumulator: v = sum_g acc_g 2^(-7g)
                double v[32];
#pragma unroll
                for (int g = S - 1; g >= 0; --g) {
                    uint32_t a[32];
                    tmem_issue32(tl + (uint32_t)(g * QT), a);
                    tmem_wait_ld();
                    tmem_zero32(tl + (uint32_t)(g * QT));
                    tmem_wait_st();
                    fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(bar(GFREE + g));
#pragma unroll
                    for (int k = 0; k < 32; ++k) {
                        const double x = exact_f64((int)a[k]);
                        v[k] = (g == S - 1) ? x : fma(v[k], 0x1p-7, x);
                    }
                }
                const int q0 = qt * QT + half * 32;
#pragma unroll
                for (int k = 0; k < 32; ++k) {
                    const int q = q0 + k;
                    if (mrow && q < P.nbf5) dst[(size_t)P.nbf * q] = v[k] * sa * P.sb[q];
                }
            }
        }
    }

    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag && P.fail) *reinterpret_cast<volatile int*>(P.fail) = 1;
    if (warp == ISSUER) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// ---------------------------------------------------------------- digit slices
// Row scales of b: sa[m + nbf*l] = 2^e with max_n |b[m, n, l]| < 2^e (1 for a
// zero row); one thread per (m, l), coalesced over m.
__global__ void row_scale_kernel(const double* __restrict__ b, int nbf, long long naux, double* __restrict__ sa) {
    const long long total = (long long)nbf * naux;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long l = i / nbf;
        const int m = (int)(i - l * nbf);
        const double* row = b + (long long)nbf * nbf * l + m;
        double mx = 0.0;
        for (int n = 0; n < nbf; ++n) mx = fmax(mx, fabs(row[(long long)nbf * n]));
        int e = 0;
        if (mx > 0.0) frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1)
        sa[i] = ldexp(1.0, e);
    }
}

// Digits of one value scaled into (-1, 1): d_i = trunc(128 r_i), r_(i+1) = 128 r_i - d_i.
__device__ __forceinline__ void digits(double y, int8_t (&d)[S]) {
#pragma unroll
    for (int i = 0; i < S; ++i) {
        y *= 128.0;
        const double t = trunc(y);
        d[i] = (int8_t)(int)t;
        y -= t;
    }
}

// b's slices, transposed so that n is contiguous: out[n + ldn*(m + nbf*(i + S*l))].
// 32 x 32 (m, n) tiles through shared memory: reads coalesced over m, writes over n.
__global__ void __launch_bounds__(256) split_b_kernel(const double* __restrict__ b, const double* __restrict__ sa,
                                                      int nbf, int ldn, long long naux, int8_t* __restrict__ out) {
    __shared__ double tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int tn = (nbf + 31) / 32;
    const long long tiles = (long long)tn * tn * naux;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        const long long l = t / ((long long)tn * tn);
        const int r = (int)(t - l * tn * tn);
        const int m0 = 32 * (r % tn), n0 = 32 * (r / tn);
        const double* B = b + (long long)nbf * nbf * l;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int m = m0 + tx, n = n0 + ty + 8 * k;
            tile[ty + 8 * k][tx] = (m < nbf && n < nbf) ? B[m + (long long)nbf * n] : 0.0;  // tile[n][m]
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int m = m0 + ty + 8 * k, n = n0 + tx;
            if (m >= nbf || n >= nbf) continue;
            int8_t d[S];
            digits(tile[tx][ty + 8 * k] / sa[m + (long long)nbf * l], d);
#pragma unroll
            for (int i = 0; i < S; ++i) out[n + (long long)ldn * (m + (long long)nbf * (i + S * l))] = d[i];
        }
    }
}

// C5's slices (one block per column q): sb[q] = 2^(e - 14) with max_n |C[n, q]| < 2^e,
// out[n + ldn*(q + nbf5*i)].
__global__ void __launch_bounds__(256) split_c_kernel(const double* __restrict__ C, int nbf, int nbf5, int ldn,
                                                      double* __restrict__ sb, int8_t* __restrict__ out) {
    __shared__ double red[8];
    __shared__ double inv_s;
    const int q = blockIdx.x;
    const double* col = C + (long long)nbf * q;
    double mx = 0.0;
    for (int n = threadIdx.x; n < nbf; n += blockDim.x) mx = fmax(mx, fabs(col[n]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        int e = 0;
        if (m > 0.0) frexp(m, &e);
        sb[q] = ldexp(1.0, e - 14);  // 2^-14: the weight 2^(-7(i+1) - 7(j+1)) of digit pair (0, 0)
        inv_s = ldexp(1.0, -e);
    }
    __syncthreads();
    const double inv = inv_s;
    for (int n = threadIdx.x; n < nbf; n += blockDim.x) {
        int8_t d[S];
        digits(col[n] * inv, d);
#pragma unroll
        for (int i = 0; i < S; ++i) out[n + (long long)ldn * (q + (long long)nbf5 * i)] = d[i];
    }
}

}  // namespace oz

namespace {

int ldn_of(int nbf) { return (nbf + 15) / 16 * 16; }  // 16-byte row pitch (TMA stride rule)
size_t slice_bytes(int nbf, int naux) { return (size_t)naux * oz::S * nbf * ldn_of(nbf); }
size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

bool ozaki_shape_ok(int nbf) { return nbf >= 1 && nbf <= 16384; }

size_t ozaki_bytes(int nbf, int naux) {
    return align256(slice_bytes(nbf, naux)) + sizeof(double) * (size_t)nbf * naux;
}

// Digit slices and row scales of the job's b (kept until ozaki_free).
int ozaki_build(donof_job* job) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    if (job->oz_b) return DONOF_OK;
    if (!ozaki_shape_ok(nbf)) {
        set_error(ctx, "the tensor-core FP64 transform needs nbf <= 16384 (got %d)", nbf);
        return DONOF_ERR_ARG;
    }
    void* buf = nullptr;
    DONOF_CHECK(dev_alloc(ctx, &buf, ozaki_bytes(nbf, naux)));
    int8_t* slices = static_cast<int8_t*>(buf);
    double* sa = reinterpret_cast<double*>(static_cast<char*>(buf) + align256(slice_bytes(nbf, naux)));
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemsetAsync(slices, 0, slice_bytes(nbf, naux), st);
    if (e == cudaSuccess) {
        oz::row_scale_kernel<<<8 * ctx->sm_count, 256, 0, st>>>(job->b, nbf, (long long)naux, sa); count_launch();
        oz::split_b_kernel<<<16 * ctx->sm_count, 256, 0, st>>>(job->b, sa, nbf, ldn_of(nbf), (long long)naux, slices);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        dev_free(ctx, buf);
        set_error(ctx, "digit slices of b: %s", cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    job->oz_b = buf;
    job->oz_sa = sa;
    ++job->oz_gen;
    return DONOF_OK;
}

void ozaki_free(donof_job* job) {
    if (!job->oz_b) return;
    cudaStreamSynchronize(job->ctx->stream);
    dev_free(job->ctx, job->oz_b);
    job->oz_b = nullptr;
    job->oz_sa = nullptr;
    job->oz_c.release(job->ctx);
    ++job->oz_gen;
}

// tmp_l = B_l C5 for every l (FP64 result, tmp[m + nbf*q + nbf*nbf5*l]).
int t1_ozaki(donof_job* job, cudaStream_t st, const double* C, int nbf5, double* tmp) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux, ldn = ldn_of(nbf);
    const size_t cbytes = align256((size_t)oz::S * nbf5 * ldn);
    DONOF_CHECK(job->oz_c.ensure(ctx, cbytes + sizeof(double) * (size_t)nbf5));
    int8_t* c8 = job->oz_c.as<int8_t>();
    double* sb = reinterpret_cast<double*>(job->oz_c.as<char>() + cbytes);
    oz::split_c_kernel<<<nbf5, 256, 0, st>>>(C, nbf, nbf5, ldn, sb, c8); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());

    CUtensorMap ma, mb;
    {
        cuuint64_t dims[4] = {(cuuint64_t)nbf, (cuuint64_t)nbf, (cuuint64_t)oz::S, (cuuint64_t)naux};
        cuuint64_t strides[3] = {(cuuint64_t)ldn, (cuuint64_t)ldn * nbf, (cuuint64_t)ldn * nbf * oz::S};
        cuuint32_t box[4] = {oz::KC, oz::MT, 1, 1};
        DONOF_CHECK(make_tmap_u8(ctx, &ma, job->oz_b, 4, dims, strides, box));
    }
    {
        cuuint64_t dims[3] = {(cuuint64_t)nbf, (cuuint64_t)nbf5, (cuuint64_t)oz::S};
        cuuint64_t strides[2] = {(cuuint64_t)ldn, (cuuint64_t)ldn * nbf5};
        cuuint32_t box[3] = {oz::KC, oz::QT, oz::S};
        DONOF_CHECK(make_tmap_u8(ctx, &mb, c8, 3, dims, strides, box));
    }
    oz::Params P{};
    P.nbf = nbf; P.nbf5 = nbf5; P.naux = naux;
    P.nmt = (nbf + oz::MT - 1) / oz::MT;
    P.nkc = (nbf + oz::KC - 1) / oz::KC;
    P.nqt = (nbf5 + oz::QT - 1) / oz::QT;
    P.resident = P.nqt * P.nkc <= 2;
    P.sa = job->oz_sa; P.sb = sb; P.tmp = tmp;
    P.fail = ctx->fail_dev ? ctx->fail_dev + FAIL_MBAR : nullptr;
    P.wait = sm100::wait_budget(ctx->wait_limit);
    const long long units = (long long)naux * P.nmt;
    const int grid = (int)(units < ctx_ctas(ctx) ? units : ctx_ctas(ctx));
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(oz::ozaki_t1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             oz::SMEM_ALLOC));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    prof_begin(ctx, st);
    oz::ozaki_t1_kernel<<<grid, oz::NTHREADS, oz::SMEM_ALLOC, st>>>(ma, mb, P); count_launch();
    prof_end(ctx, st);
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

}  // namespace donof
