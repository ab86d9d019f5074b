// Mixed-precision form for every shape (any nbf, nbf5): the contractions of the
// RI hot path as 3 x bf16 split products on the 5th-generation tensor cores.
//
// The fused kernel of mixed.cu keeps one aux index entirely on chip, which
// limits it to nbf <= 256 and nbf5 <= 64 (TMEM holds T1, T2 and the Y
// accumulator at once).  Larger jobs (n-octane, water clusters, alkanes) run
// the same arithmetic as a short pipeline of one persistent tcgen05 GEMM kernel
// (mg_gemm_kernel) with three epilogues, plus two small kernels:
//
//   T1  tmp_l[m, q]  = sum_n C5[n, q] b_l[n, m]       D[q, m]; tmp written as a
//                                                      bf16 hi/lo split tmpQ[l][q][m]
//   T2  b_pq^l[p, q] = sum_m C5[m, p] tmp_l[m, q]     D[p, q]; FP32 out
//   W   W_l[q, b] = delta_qb (n'_b d_b + sum_q' cj12[b, q'] d_q') - ck12[b, q] b_bq^l
//                                                      (mg_wdiag_kernel + mg_w_kernel, FP32, split out)
//   Y   Y[m, b] = sum_l sum_q W_l[q, b] tmp_l[m, q]    D[b, m]; FP32 partial per aux chunk
//
// and the FP64 tail (tail.cu) forms H_mat, elag and E_elec from the Y
// partials, as for the other forms (src/utils.jl:1-59 restructured:
// elag[:, :nbf5] = C^T Y + n o H_mat).
//
// b is the RI tensor, symmetric in (m, n) like every tensor Iaux produces;
// the W builder reads b_pq^l through the symmetry that follows from it.
//
// Every product is  A_hi B_hi + A_hi B_lo + A_lo B_hi  (the lo x lo term is
// below FP32 rounding) with FP32 accumulation in TMEM.  Operands are staged by
// TMA (no multicast) in 128-byte swizzled tiles: A always K-major (128 rows x
// 64 k), B either K-major (T2: tmpQ rows q, contiguous m) or MN-major in
// 64-column chunks (T1: the quarter-major bf16 split of b; Y: tmpQ read with m
// contiguous).  One CTA per SM walks its work items (aux index or aux chunk x
// row tile x column tile) with a 2-stage ring of 96 KB stages and two 256-column
// TMEM accumulators, so the epilogue of one item overlaps the MMAs of the next.
//
// Warp roles (192 threads): warps 0-3 epilogue (TMEM lane quarters), warp 4
// TMA producer, warp 5 TMEM allocator + MMA issuer.  Every mbarrier wait is
// bounded (sm100.cuh); a wait that runs out sets the CTA's abort flag, the
// roles stop, in-flight copies and MMAs are drained with bounded waits, TMEM is
// freed and the context's failure word records the failure.
#include <atomic>
#include <cuda.h>
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "sm100.cuh"

namespace donof {

namespace mg {

using namespace sm100;

constexpr int NTHREADS = 192;
constexpr int BM = 128;                          // output rows per tile (TMEM lanes)
constexpr int BN = 256;                          // output columns per tile (TMEM columns per accumulator)
constexpr int BK = 64;                           // k per stage: one 128-byte swizzle row of bf16
constexpr int A_BYTES = BM * BK * 2;             // 16 KB per part (hi, lo)
constexpr int B_BYTES = BN * BK * 2;             // 32 KB per part
constexpr int CHUNK_BYTES = 64 * BK * 2;         // 8 KB: MN-major box of 64 columns x 64 k
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 96 KB
constexpr int RING = 2;
constexpr int OFF_BAR = RING * STAGE_BYTES;
constexpr int NBAR = 16;
constexpr int OFF_MISC = OFF_BAR + NBAR * 8;     // abort flag, TMEM base, epilogue vote
constexpr int SMEM_USED = OFF_MISC + 64;
constexpr int SMEM_ALLOC = SMEM_USED + 1024;     // slack for 1024-B alignment
static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory budget");

// barriers
constexpr int B_FULL = 0;              // +s: stage s landed
constexpr int B_EMPTY = RING;          // +s: stage s consumed by the MMAs
constexpr int B_ACC = 2 * RING;        // +buf: accumulator buf complete
constexpr int B_ACCFREE = B_ACC + 2;   // +buf: the four epilogue warps drained buf (count 4)
constexpr int B_END = B_ACCFREE + 2;   // every MMA of the CTA complete
static_assert(B_END < NBAR, "barrier count");

enum : int { MODE_T1 = 1, MODE_T2 = 2, MODE_Y = 3 };

struct Params {
    int mode;
    int Mv, Nv;            // valid rows / columns of the output
    int mtiles, ntiles;    // 128-row and 256-column tiles
    int kb;                // 64-wide k blocks per aux index
    int naux, lchunk, nchunks;
    int kbox_rows;         // T2: rows of the K-major B box (<= 256)
    int nbf, nbf5, ldm;
    __nv_bfloat16* tq_hi;  // T1 out: tmpQ[m + ldm q + ldm nbf5 l]
    __nv_bfloat16* tq_lo;
    float* out;            // T2: b_pq[p + nbf5 q + nbf5^2 l]; Y: part[m + nbf b + nbf nbf5 chunk]
    int* fail;             // the context's failure word for mbarrier waits (set to 1 on a timeout)
    long long wait;        // cycle budget of every bounded wait (drains excepted)
};

struct Item {
    int chunk, mt, nt, l0, l1, ncol;
};

__device__ __forceinline__ Item decode(const Params& P, int item) {
    Item it;
    const int per = P.mtiles * P.ntiles;
    it.chunk = item / per;
    const int r = item - it.chunk * per;
    it.mt = r % P.mtiles;
    it.nt = r / P.mtiles;
    it.l0 = it.chunk * P.lchunk;
    it.l1 = min(P.naux, it.l0 + P.lchunk);
    it.ncol = min(BN, P.Nv - BN * it.nt);
    return it;
}

// MMA width of a tile: whole 64-column chunks for MN-major B, a multiple of 16 for K-major B
__device__ __forceinline__ int mma_n(const Params& P, int ncol) {
    return P.mode == MODE_T2 ? (ncol + 15) / 16 * 16 : (ncol + 63) / 64 * 64;
}

__global__ void __launch_bounds__(NTHREADS, 1)
mg_gemm_kernel(const __grid_constant__ CUtensorMap ma_hi, const __grid_constant__ CUtensorMap ma_lo,
               const __grid_constant__ CUtensorMap mb_hi, const __grid_constant__ CUtensorMap mb_lo, const Params P) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = saddr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + OFF_MISC);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + OFF_MISC + 16);
    auto bar = [&](int i) { return saddr(&bars[i]); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = gridDim.x;
    const int nitems = P.nchunks * P.mtiles * P.ntiles;
    const int my_count = ((int)blockIdx.x < nitems) ? (nitems - (int)blockIdx.x + G - 1) / G : 0;

    if (threadIdx.x == 0) {
        *abort_flag = 0;
        for (int i = 0; i <= B_END; ++i) mbar_init(bar(i), (i == B_ACCFREE || i == B_ACCFREE + 1) ? 4 : 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(saddr(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 4) {
        // ------------------------------------------------------------ producer
        if (lane == 0 && my_count > 0) {
            int it = 0;
            bool ok = true;
            for (int k = 0; k < my_count && ok; ++k) {
                const Item w = decode(P, (int)blockIdx.x + k * G);
                const int nch = (w.ncol + 63) / 64;
                const uint32_t bbytes =
                    P.mode == MODE_T2 ? (uint32_t)(2 * P.kbox_rows * BK * 2) : (uint32_t)(2 * nch * CHUNK_BYTES);
                for (int l = w.l0; l < w.l1 && ok; ++l) {
                    for (int kbi = 0; kbi < P.kb; ++kbi, ++it) {
                        const int s = it % RING;
                        if (!mbar_wait(bar(B_EMPTY + s), (uint32_t)(((it / RING) & 1) ^ 1), abort_flag, P.wait)) {
                            ok = false;
                            break;
                        }
                        const uint32_t fb = bar(B_FULL + s);
                        mbar_expect_tx(fb, (uint32_t)(2 * A_BYTES) + bbytes);
                        const uint32_t st = sbase + s * STAGE_BYTES;
                        const uint32_t bh = st + 2 * A_BYTES, bl = bh + B_BYTES;
                        const int k0 = kbi * BK;
                        if (P.mode == MODE_Y) {
                            tma_load_3d(st, &ma_hi, fb, k0, BM * w.mt, l);
                            tma_load_3d(st + A_BYTES, &ma_lo, fb, k0, BM * w.mt, l);
                        } else {
                            tma_load_2d(st, &ma_hi, fb, k0, BM * w.mt);
                            tma_load_2d(st + A_BYTES, &ma_lo, fb, k0, BM * w.mt);
                        }
                        if (P.mode == MODE_T1) {
                            // quarter-major b split: coordinates (mi, n, quarter, l)
                            for (int c = 0; c < nch; ++c) {
                                tma_load_4d(bh + c * CHUNK_BYTES, &mb_hi, fb, 0, k0, 4 * w.nt + c, l);
                                tma_load_4d(bl + c * CHUNK_BYTES, &mb_lo, fb, 0, k0, 4 * w.nt + c, l);
                            }
                        } else if (P.mode == MODE_T2) {
                            // tmpQ as K-major rows q: coordinates (m, q, l)
                            tma_load_3d(bh, &mb_hi, fb, k0, BN * w.nt, l);
                            tma_load_3d(bl, &mb_lo, fb, k0, BN * w.nt, l);
                        } else {
                            // tmpQ as MN-major chunks of 64 m over 64 q: coordinates (m, q, l)
                            for (int c = 0; c < nch; ++c) {
                                tma_load_3d(bh + c * CHUNK_BYTES, &mb_hi, fb, BN * w.nt + 64 * c, k0, l);
                                tma_load_3d(bl + c * CHUNK_BYTES, &mb_lo, fb, BN * w.nt + 64 * c, k0, l);
                            }
                        }
                    }
                }
            }
            // every issued stage must have landed before the CTA exits
            const int issued = it;
            for (int j = (issued > RING ? issued - RING : 0); j < issued; ++j)
                mbar_drain(bar(B_FULL + j % RING), (uint32_t)((j / RING) & 1));
        }
    } else if (warp == 5) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0 && my_count > 0) {
            const int b_mn = (P.mode == MODE_T2) ? 0 : 1;
            int it = 0;
            bool ok = true;
            for (int k = 0; k < my_count && ok; ++k) {
                const Item w = decode(P, (int)blockIdx.x + k * G);
                const int buf = k & 1;
                if (!mbar_wait(bar(B_ACCFREE + buf), (uint32_t)(((k >> 1) & 1) ^ 1), abort_flag, P.wait)) break;
                fence_after();
                const uint32_t d = tmem + (uint32_t)(BN * buf);
                const uint32_t id = idesc(BM, mma_n(P, w.ncol), 0, b_mn);
                bool first = true;
                for (int l = w.l0; l < w.l1 && ok; ++l) {
                    for (int kbi = 0; kbi < P.kb; ++kbi, ++it) {
                        const int s = it % RING;
                        if (!mbar_wait(bar(B_FULL + s), (uint32_t)((it / RING) & 1), abort_flag, P.wait)) {
                            ok = false;
                            break;
                        }
                        fence_after();
                        const uint32_t st = sbase + s * STAGE_BYTES;
                        const uint32_t bh = st + 2 * A_BYTES, bl = bh + B_BYTES;
#pragma unroll
                        for (int ks = 0; ks < BK / 16; ++ks) {
                            const uint64_t ah = sdesc(st + ks * 32, 16, 1024);
                            const uint64_t al = sdesc(st + A_BYTES + ks * 32, 16, 1024);
                            uint64_t dbh, dbl;
                            if (b_mn) {
                                dbh = sdesc(bh + ks * 2048, CHUNK_BYTES, 1024);
                                dbl = sdesc(bl + ks * 2048, CHUNK_BYTES, 1024);
                            } else {
                                dbh = sdesc(bh + ks * 32, 16, 1024);
                                dbl = sdesc(bl + ks * 32, 16, 1024);
                            }
                            umma(d, ah, dbh, id, (first && ks == 0) ? 0u : 1u);
                            umma(d, ah, dbl, id, 1u);
                            umma(d, al, dbh, id, 1u);
                        }
                        first = false;
                        umma_commit(bar(B_EMPTY + s));
                    }
                }
                if (!ok) break;
                umma_commit(bar(B_ACC + buf));
            }
            umma_commit(bar(B_END));
            mbar_drain(bar(B_END), 0);  // every MMA of this CTA has completed
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 0-3)
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        for (int k = 0; k < my_count; ++k) {
            const Item w = decode(P, (int)blockIdx.x + k * G);
            const int buf = k & 1;
            int r = 1;
            if (lane == 0) r = mbar_wait(bar(B_ACC + buf), (uint32_t)((k >> 1) & 1), abort_flag, P.wait) ? 1 : 0;
            r = __shfl_sync(0xffffffffu, r, 0);
            if (!r) break;
            fence_after();
            const int row = BM * w.mt + 32 * warp + lane;  // output row of this thread
            const uint32_t src = tmem + (uint32_t)(BN * buf) + lane_addr;
            const int ncols = mma_n(P, w.ncol);
            for (int c = 0; c < ncols / 32 + ((ncols & 31) ? 1 : 0); ++c) {
                float v[32];
                tmem_ld32(src + 32 * c, v);
                const int col0 = BN * w.nt + 32 * c;  // output column of v[0]
                if (P.mode == MODE_T1) {
                    // row = q, columns = m, l = the item's aux index
                    if (row < P.nbf5) {
                        const size_t base = (size_t)P.ldm * row + (size_t)P.ldm * P.nbf5 * w.l0;
#pragma unroll
                        for (int g8 = 0; g8 < 4; ++g8) {
                            const int m8 = col0 + 8 * g8;
                            __align__(16) __nv_bfloat16 h[8], lo[8];
#pragma unroll
                            for (int e = 0; e < 8; ++e) split_bf16(v[8 * g8 + e], h[e], lo[e]);
                            if (m8 + 8 <= P.nbf) {
                                *reinterpret_cast<uint4*>(P.tq_hi + base + m8) = *reinterpret_cast<const uint4*>(h);
                                *reinterpret_cast<uint4*>(P.tq_lo + base + m8) = *reinterpret_cast<const uint4*>(lo);
                            } else {
#pragma unroll
                                for (int e = 0; e < 8; ++e)
                                    if (m8 + e < P.nbf) {
                                        P.tq_hi[base + m8 + e] = h[e];
                                        P.tq_lo[base + m8 + e] = lo[e];
                                    }
                            }
                        }
                    }
                } else if (P.mode == MODE_T2) {
                    // row = p, columns = q
                    if (row < P.nbf5) {
                        float* dst = P.out + (size_t)P.nbf5 * P.nbf5 * w.l0 + row;
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (col0 + i < P.nbf5) dst[(size_t)P.nbf5 * (col0 + i)] = v[i];
                    }
                } else {
                    // row = b, columns = m
                    if (row < P.nbf5) {
                        float* dst = P.out + (size_t)P.nbf * P.nbf5 * w.chunk + (size_t)P.nbf * row;
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (col0 + i < P.nbf) dst[col0 + i] = v[i];
                    }
                }
            }
            // the accumulator can take the next item
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(B_ACCFREE + buf));
        }
    }

    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag && P.fail) *reinterpret_cast<volatile int*>(P.fail) = 1;
    if (warp == 5) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// Cs_x[n + ldm q] = C_x[n, q] (C5 transposed, rows q; zero for n >= nbf), and
// the functional's n, cj12 and ck12 in FP32 (coefficients only when n != null):
// n32[q], cj32[b + nbf5 q] = cj12[b, q], ckT[q + nbf5 b] = ck12[b, q].
__global__ void mg_prep_kernel(const double* __restrict__ C, int nbf, int nbf5, int ldm,
                               __nv_bfloat16* __restrict__ cs_hi, __nv_bfloat16* __restrict__ cs_lo,
                               const double* __restrict__ n, const double* __restrict__ cj12,
                               const double* __restrict__ ck12, float* __restrict__ n32, float* __restrict__ cj32,
                               float* __restrict__ ckT) {
    const long long ncs = (long long)ldm * nbf5, n55 = (long long)nbf5 * nbf5;
    const long long total = ncs > n55 ? ncs : n55;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < ncs) {
            const int k = (int)(i % ldm), q = (int)(i / ldm);
            const double v = (k < nbf) ? C[k + (long long)nbf * q] : 0.0;
            const __nv_bfloat16 h = __double2bfloat16(v);
            cs_hi[i] = h;
            cs_lo[i] = __double2bfloat16(v - (double)__bfloat162float(h));
        }
        if (n != nullptr && i < n55) {
            const int b = (int)(i % nbf5), q = (int)(i / nbf5);
            cj32[i] = (float)cj12[i];
            ckT[q + (long long)nbf5 * b] = (float)ck12[i];
            if (i < nbf5) n32[i] = (float)n[i];
        }
    }
}

// W (FP32), written as the bf16 split W_x[q + ldq b + ldq nbf5 l] (rows b,
// contiguous q: the K-major A operand of Y):
//   W[q, b] = delta_qb (n'_b d_b + sum_q' cj12[b, q'] d_q') - ck12[b, q] b_pq[q, b]
// with d_q = b_pq[q, q] and n'_b = n_b for b < nbeta or b >= nalpha (0 when
// nbeta = 0); b_pq is symmetric, so its row b is read as column b.  mg_wdiag
// forms the diagonal terms (one thread per (b, l)), mg_w the elements (one
// thread per element, reads and writes along q).
__global__ void mg_wdiag_kernel(const float* __restrict__ bpq, const float* __restrict__ n32,
                                const float* __restrict__ cj32, int nbf5, int naux, int nalpha, int nbeta,
                                float* __restrict__ tv) {
    const long long n55 = (long long)nbf5 * nbf5, total = (long long)nbf5 * naux;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i % nbf5);
        const float* B = bpq + n55 * (i / nbf5);
        float s = 0.f;
        for (int q = 0; q < nbf5; ++q) s += cj32[b + (long long)nbf5 * q] * B[(long long)q * (nbf5 + 1)];
        const bool dj = (nbeta > 0) && (b < nbeta || b >= nalpha);
        tv[i] = (dj ? n32[b] * B[(long long)b * (nbf5 + 1)] : 0.f) + s;
    }
}

__global__ void mg_w_kernel(const float* __restrict__ bpq, const float* __restrict__ ckT,
                            const float* __restrict__ tv, int nbf5, int ldq, int naux,
                            __nv_bfloat16* __restrict__ w_hi, __nv_bfloat16* __restrict__ w_lo) {
    const long long n55 = (long long)nbf5 * nbf5, total = (long long)ldq * nbf5 * naux;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i % ldq);
        const long long r = i / ldq;  // b + nbf5 l
        const int b = (int)(r % nbf5);
        const long long l = r / nbf5;
        float v = 0.f;
        if (q < nbf5) {
            v = -ckT[q + (long long)nbf5 * b] * bpq[q + (long long)nbf5 * b + n55 * l];
            if (q == b) v += tv[r];
        }
        __nv_bfloat16 h, lo;
        split_bf16(v, h, lo);
        w_hi[i] = h;
        w_lo[i] = lo;
    }
}

// J and K partial sums over an aux chunk from FP32 b_pq, accumulated in FP64:
// part[c][0][p + nbf5 q] = sum_l d_p d_q,  part[c][1][p + nbf5 q] = sum_l b_pq^2
__global__ void mg_jk_partial_kernel(const float* __restrict__ bpq, int nbf5, int naux, int lchunk,
                                     double* __restrict__ part) {
    const long long n55 = (long long)nbf5 * nbf5;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (idx >= n55) return;
    const int p = (int)(idx % nbf5), q = (int)(idx / nbf5);
    const int l0 = c * lchunk, l1 = min(naux, l0 + lchunk);
    double sj = 0.0, sk = 0.0;
    for (int l = l0; l < l1; ++l) {
        const float* B = bpq + n55 * l;
        const double v = B[idx];
        sj += (double)B[(long long)p * (nbf5 + 1)] * (double)B[(long long)q * (nbf5 + 1)];
        sk += v * v;
    }
    part[(long long)c * 2 * n55 + idx] = sj;
    part[(long long)c * 2 * n55 + n55 + idx] = sk;
}

// tmp[m + nbf q + nbf nbf5 l] = tmpQ_hi + tmpQ_lo (FP32, for checks of T1)
__global__ void mg_tq_to_f32(const __nv_bfloat16* __restrict__ hi, const __nv_bfloat16* __restrict__ lo, int nbf,
                             int nbf5, int ldm, long long naux, float* __restrict__ out) {
    const long long total = (long long)nbf * nbf5 * naux;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(i % nbf);
        const long long r = i / nbf;  // q + nbf5 l
        const long long src = m + (long long)ldm * r;
        out[i] = __bfloat162float(hi[src]) + __bfloat162float(lo[src]);
    }
}

__global__ void f32_to_f64_kernel(const float* __restrict__ a, long long count, double* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)a[i];
}

}  // namespace mg

namespace {

int round8(int x) { return (x + 7) / 8 * 8; }

// Scratch of the general mixed form.  job->tmp: tmpQ hi | lo; job->W:
// Cs hi | Cs lo | n32 | cj32 | ckT | b_pq (FP32) | W hi | W lo | Y partials.
struct GenScratch {
    __nv_bfloat16 *cs_hi, *cs_lo, *tq_hi, *tq_lo, *w_hi, *w_lo;
    float *n32, *cj32, *ckT, *bpq, *ypart, *tv;
    int ldm, ldq, nchunks, lchunk;
};

void y_chunks(donof_job* job, int nbf5, int* nchunks, int* lchunk) {
    const int mtiles = (nbf5 + mg::BM - 1) / mg::BM, ntiles = (job->nbf + mg::BN - 1) / mg::BN;
    int nc = ctx_ctas(job->ctx) / (mtiles * ntiles);
    if (nc < 1) nc = 1;
    if (nc > job->naux) nc = job->naux;
    const int lc = (job->naux + nc - 1) / nc;
    *lchunk = lc;
    *nchunks = (job->naux + lc - 1) / lc;
}

int gen_prepare(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* cj12,
                const double* ck12, int nbf5, bool with_w, GenScratch* S) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    S->ldm = round8(nbf);
    S->ldq = round8(nbf5);
    y_chunks(job, nbf5, &S->nchunks, &S->lchunk);
    const size_t tq = (size_t)S->ldm * nbf5 * naux;
    DONOF_CHECK(job->tmp.ensure(ctx, 2 * sizeof(__nv_bfloat16) * tq));
    S->tq_hi = job->tmp.as<__nv_bfloat16>();
    S->tq_lo = S->tq_hi + tq;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_cs = take(2 * sizeof(__nv_bfloat16) * (size_t)S->ldm * nbf5);
    const size_t o_n = take(sizeof(float) * (size_t)nbf5);
    const size_t o_cj = take(sizeof(float) * (size_t)nbf5 * nbf5);
    const size_t o_ck = take(sizeof(float) * (size_t)nbf5 * nbf5);
    const size_t o_bpq = take(sizeof(float) * (size_t)nbf5 * nbf5 * naux);
    const size_t wsz = with_w ? (size_t)S->ldq * nbf5 * naux : 0;
    const size_t o_w = take(2 * sizeof(__nv_bfloat16) * wsz);
    const size_t o_y = take(with_w ? sizeof(float) * (size_t)S->nchunks * nbf * nbf5 : 0);
    const size_t o_tv = take(with_w ? sizeof(float) * (size_t)nbf5 * naux : 0);
    DONOF_CHECK(job->W.ensure(ctx, off));
    char* base = job->W.as<char>();
    S->cs_hi = reinterpret_cast<__nv_bfloat16*>(base + o_cs);
    S->cs_lo = S->cs_hi + (size_t)S->ldm * nbf5;
    S->n32 = reinterpret_cast<float*>(base + o_n);
    S->cj32 = reinterpret_cast<float*>(base + o_cj);
    S->ckT = reinterpret_cast<float*>(base + o_ck);
    S->bpq = reinterpret_cast<float*>(base + o_bpq);
    S->w_hi = reinterpret_cast<__nv_bfloat16*>(base + o_w);
    S->w_lo = S->w_hi + wsz;
    S->ypart = reinterpret_cast<float*>(base + o_y);
    S->tv = reinterpret_cast<float*>(base + o_tv);
    const long long work = (long long)S->ldm * nbf5 > (long long)nbf5 * nbf5 ? (long long)S->ldm * nbf5
                                                                             : (long long)nbf5 * nbf5;
    long long blocks = (work + 255) / 256;
    if (blocks > 4LL * ctx->sm_count) blocks = 4LL * ctx->sm_count;
    mg::mg_prep_kernel<<<(int)blocks, 256, 0, st>>>(C, nbf, nbf5, S->ldm, S->cs_hi, S->cs_lo, with_w ? n : nullptr,
                                                    cj12, ck12, S->n32, S->cj32, S->ckT); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int launch_gemm(donof_job* job, cudaStream_t st, const mg::Params& P, const CUtensorMap& a_hi, const CUtensorMap& a_lo,
                const CUtensorMap& b_hi, const CUtensorMap& b_lo) {
    donof_ctx* ctx = job->ctx;
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(mg::mg_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             mg::SMEM_ALLOC));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    const int nitems = P.nchunks * P.mtiles * P.ntiles;
    const int grid = nitems < ctx_ctas(ctx) ? nitems : ctx_ctas(ctx);
    mg::mg_gemm_kernel<<<grid, mg::NTHREADS, mg::SMEM_ALLOC, st>>>(a_hi, a_lo, b_hi, b_lo, P); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

mg::Params base_params(donof_job* job, int nbf5, const GenScratch& S) {
    mg::Params P{};
    P.naux = job->naux;
    P.nbf = job->nbf;
    P.nbf5 = nbf5;
    P.ldm = S.ldm;
    P.fail = job->ctx->fail_dev ? job->ctx->fail_dev + FAIL_MBAR : nullptr;
    P.wait = sm100::wait_budget(job->ctx->wait_limit);
    P.lchunk = 1;
    P.nchunks = job->naux;
    return P;
}

// T1 and T2: tmpQ (split) in job->tmp, b_pq (FP32) in the scratch
int gen_transforms(donof_job* job, cudaStream_t st, int nbf5, const GenScratch& S) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux, ldm = S.ldm;
    CUtensorMap cs_hi, cs_lo, bq_hi, bq_lo, tk_hi, tk_lo;
    {   // C5 transposed, rows q: (k, q)
        cuuint64_t dims[2] = {(cuuint64_t)nbf, (cuuint64_t)nbf5};
        cuuint64_t strides[1] = {(cuuint64_t)ldm * 2};
        cuuint32_t box[2] = {64, 128};
        DONOF_CHECK(make_tmap_bf16(ctx, &cs_hi, S.cs_hi, 2, dims, strides, box));
        DONOF_CHECK(make_tmap_bf16(ctx, &cs_lo, S.cs_lo, 2, dims, strides, box));
    }
    {   // quarter-major b split: (mi, n, quarter, l)
        const int nb = (nbf + 63) / 64;
        cuuint64_t dims[4] = {64, (cuuint64_t)nbf, (cuuint64_t)nb, (cuuint64_t)naux};
        cuuint64_t strides[3] = {128, (cuuint64_t)128 * nbf, (cuuint64_t)128 * nbf * nb};
        cuuint32_t box[4] = {64, 64, 1, 1};
        DONOF_CHECK(make_tmap_bf16(ctx, &bq_hi, job->b16hi, 4, dims, strides, box));
        DONOF_CHECK(make_tmap_bf16(ctx, &bq_lo, job->b16lo, 4, dims, strides, box));
    }
    const int kbox = nbf5 >= mg::BN ? mg::BN : (nbf5 + 15) / 16 * 16;
    {   // tmpQ as K-major rows q: (m, q, l)
        cuuint64_t dims[3] = {(cuuint64_t)nbf, (cuuint64_t)nbf5, (cuuint64_t)naux};
        cuuint64_t strides[2] = {(cuuint64_t)ldm * 2, (cuuint64_t)ldm * nbf5 * 2};
        cuuint32_t box[3] = {64, (cuuint32_t)kbox, 1};
        DONOF_CHECK(make_tmap_bf16(ctx, &tk_hi, S.tq_hi, 3, dims, strides, box));
        DONOF_CHECK(make_tmap_bf16(ctx, &tk_lo, S.tq_lo, 3, dims, strides, box));
    }
    mg::Params P = base_params(job, nbf5, S);
    P.mode = mg::MODE_T1;
    P.Mv = nbf5; P.Nv = nbf;
    P.mtiles = (nbf5 + mg::BM - 1) / mg::BM; P.ntiles = (nbf + mg::BN - 1) / mg::BN;
    P.kb = (nbf + mg::BK - 1) / mg::BK;
    P.tq_hi = S.tq_hi; P.tq_lo = S.tq_lo;
    prof_begin(ctx, st);
    DONOF_CHECK(launch_gemm(job, st, P, cs_hi, cs_lo, bq_hi, bq_lo));
    prof_end(ctx, st);
    P.mode = mg::MODE_T2;
    P.Mv = nbf5; P.Nv = nbf5;
    P.mtiles = (nbf5 + mg::BM - 1) / mg::BM; P.ntiles = (nbf5 + mg::BN - 1) / mg::BN;
    P.kb = (nbf + mg::BK - 1) / mg::BK;
    P.kbox_rows = kbox;
    P.out = S.bpq;
    return launch_gemm(job, st, P, cs_hi, cs_lo, tk_hi, tk_lo);
}

}  // namespace

bool mixed_general_needed(int nbf, int nbf5) { return !(nbf <= 256 && nbf5 <= 64); }

int lagrange2_mixed_general(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* H,
                            const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta, double* elag,
                            double* Hmat, double* E) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    GenScratch S;
    DONOF_CHECK(gen_prepare(job, st, C, n, cj12, ck12, nbf5, true, &S));
    DONOF_CHECK(gen_transforms(job, st, nbf5, S));
    {
        const long long nd = (long long)nbf5 * naux, nw = (long long)S.ldq * nbf5 * naux;
        long long blocks = (nd + 255) / 256;
        if (blocks > 8LL * ctx->sm_count) blocks = 8LL * ctx->sm_count;
        mg::mg_wdiag_kernel<<<(int)blocks, 256, 0, st>>>(S.bpq, S.n32, S.cj32, nbf5, naux, nalpha, nbeta,
                                                         S.tv); count_launch();
        blocks = (nw + 255) / 256;
        if (blocks > 16LL * ctx->sm_count) blocks = 16LL * ctx->sm_count;
        mg::mg_w_kernel<<<(int)blocks, 256, 0, st>>>(S.bpq, S.ckT, S.tv, nbf5, S.ldq, naux, S.w_hi,
                                                     S.w_lo); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
    }
    CUtensorMap w_hi, w_lo, tm_hi, tm_lo;
    {   // W, rows b, contiguous q: (q, b, l)
        cuuint64_t dims[3] = {(cuuint64_t)nbf5, (cuuint64_t)nbf5, (cuuint64_t)naux};
        cuuint64_t strides[2] = {(cuuint64_t)S.ldq * 2, (cuuint64_t)S.ldq * nbf5 * 2};
        cuuint32_t box[3] = {64, 128, 1};
        DONOF_CHECK(make_tmap_bf16(ctx, &w_hi, S.w_hi, 3, dims, strides, box));
        DONOF_CHECK(make_tmap_bf16(ctx, &w_lo, S.w_lo, 3, dims, strides, box));
    }
    {   // tmpQ as MN-major chunks: (m, q, l), boxes of 64 m x 64 q
        cuuint64_t dims[3] = {(cuuint64_t)nbf, (cuuint64_t)nbf5, (cuuint64_t)naux};
        cuuint64_t strides[2] = {(cuuint64_t)S.ldm * 2, (cuuint64_t)S.ldm * nbf5 * 2};
        cuuint32_t box[3] = {64, 64, 1};
        DONOF_CHECK(make_tmap_bf16(ctx, &tm_hi, S.tq_hi, 3, dims, strides, box));
        DONOF_CHECK(make_tmap_bf16(ctx, &tm_lo, S.tq_lo, 3, dims, strides, box));
    }
    mg::Params P = base_params(job, nbf5, S);
    P.mode = mg::MODE_Y;
    P.Mv = nbf5; P.Nv = nbf;
    P.mtiles = (nbf5 + mg::BM - 1) / mg::BM; P.ntiles = (nbf + mg::BN - 1) / mg::BN;
    P.kb = (nbf5 + mg::BK - 1) / mg::BK;
    P.lchunk = S.lchunk; P.nchunks = S.nchunks;
    P.out = S.ypart;
    DONOF_CHECK(launch_gemm(job, st, P, w_hi, w_lo, tm_hi, tm_lo));
    return elag_tail_f64(job, st, C, H, n, nbf5, S.ypart, true, S.nchunks, (long long)nbf * nbf5, Hmat, elag, E);
}

int transforms_mixed_general(donof_job* job, cudaStream_t st, const double* C, int nbf5) {
    donof_ctx* ctx = job->ctx;
    GenScratch S;
    DONOF_CHECK(gen_prepare(job, st, C, nullptr, nullptr, nullptr, nbf5, false, &S));
    DONOF_CHECK(gen_transforms(job, st, nbf5, S));
    const long long cnt = (long long)nbf5 * nbf5 * job->naux;
    DONOF_CHECK(job->bpq.ensure(ctx, sizeof(double) * (size_t)cnt));
    mg::f32_to_f64_kernel<<<4 * ctx->sm_count, 256, 0, st>>>(S.bpq, cnt, job->bpq.as<double>()); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int jkh_mo_mixed_general(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5, double* J,
                         double* K, double* Hcore) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    GenScratch S;
    DONOF_CHECK(gen_prepare(job, st, C, nullptr, nullptr, nullptr, nbf5, false, &S));
    DONOF_CHECK(gen_transforms(job, st, nbf5, S));
    const long long n55 = (long long)nbf5 * nbf5;
    const int xblocks = (int)((n55 + 255) / 256);
    int chunks = (2 * ctx->sm_count + xblocks - 1) / xblocks;
    if (chunks > naux) chunks = naux;
    if (chunks < 1) chunks = 1;
    const int lchunk = (naux + chunks - 1) / chunks;
    chunks = (naux + lchunk - 1) / lchunk;
    DONOF_CHECK(job->part.ensure(ctx, sizeof(double) * (size_t)chunks * 2 * n55));
    double* part = job->part.as<double>();
    mg::mg_jk_partial_kernel<<<dim3(xblocks, chunks), 256, 0, st>>>(S.bpq, nbf5, naux, lchunk, part); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(splitk_reduce(ctx, st, part, 2 * n55, chunks, n55, J, 0.0));
    DONOF_CHECK(splitk_reduce(ctx, st, part + n55, 2 * n55, chunks, n55, K, 0.0));
    DONOF_CHECK(job->small.ensure(ctx, sizeof(double) * (size_t)nbf * nbf5 * 2));
    double* HC = job->small.as<double>();
    DONOF_CHECK(gemm_f64_auto(ctx, st, false, true, nbf, nbf5, nbf, H, nbf, C, nbf, HC, nbf, 1.0, 0.0, nullptr));
    return hcore_f64(job, st, C, HC, nbf5, Hcore);
}

int mixed_t1_general(donof_job* job, cudaStream_t st, const double* C, int nbf5, float* tmp_out) {
    donof_ctx* ctx = job->ctx;
    GenScratch S;
    DONOF_CHECK(gen_prepare(job, st, C, nullptr, nullptr, nullptr, nbf5, false, &S));
    DONOF_CHECK(gen_transforms(job, st, nbf5, S));
    mg::mg_tq_to_f32<<<4 * ctx->sm_count, 256, 0, st>>>(S.tq_hi, S.tq_lo, job->nbf, nbf5, S.ldm, job->naux, tmp_out); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

}  // namespace donof
