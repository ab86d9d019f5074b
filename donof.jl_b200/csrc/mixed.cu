// Mixed-precision form of the RI hot path on the 5th-generation tensor cores.
//
// b is kept on the device as two bf16 arrays, b = b_hi + b_lo (both rounded
// to nearest, 16 significant bits together); C5, the intermediates and the
// functional weights are split the same way, and every product is formed from
// all four hi/lo pairs with FP32 accumulation in tensor memory (TMEM).  The
// hi and lo halves of the small operand are stacked as the 128 rows of one
// MMA, so one tcgen05.mma (M = 128) yields both partial products; the row of
// part x (0 hi, 1 lo) of index q is prow(q, x) = 32 (q / 16) + 16 x + q % 16,
// which puts both parts of q in one warp's TMEM lanes (i and i + 16), so the
// hi + lo sums are warp shuffles.
//
// One persistent kernel (lag_mixed_kernel) walks the aux index l and, per l,
// without leaving the SM:
//   T1  D1[j, m] = sum_n Cs[j, n] b_x[n, m]      (x = hi, lo; j = prow(q, x)),
//       one 64-column quarter of m at a time into two ping-pong TMEM slots
//       tmp[m, q] = D1[prow(q, 0), m] + D1[prow(q, 1), m]
//   T2  D2[j, j'] = sum_m tmp_x[m, q] Cs[j', m]  -> b_pq = sum of 4 quadrants
//   W   W[q, b] = delta_qb (n'_b d_b + sum_q' cj12[b,q'] d_q') - ck12[b,q] b_bq
//   Y   D3[j, m] += sum_q W_x[q, b] tmp_y[m, q]   (accumulated over all l of the CTA)
// and emits d_q^l = b_qq^l (for J_MO = D D^T) and per-CTA partial sums of
// K_MO[p,q] = sum_l (b_pq^l)^2 and of Y.  b is read from HBM exactly once.
//
// Warp roles (192 threads): warps 0-3 epilogue (TMEM lane quarters), warp 4
// TMA producer, warp 5 TMEM allocator + MMA issuer.  Operands are staged by
// TMA (cp.async.bulk.tensor, no multicast) with 128-byte swizzle; every wait
// on an mbarrier is bounded by a clock budget after which the CTA records an
// error in its context's failure word, drains its in-flight copies, frees TMEM
// and exits.
//
// Shapes: nbf <= 256, nbf5 <= 64 (one MMA tile per aux index); larger jobs
// run the general-shape pipeline of mixed_general.cu.
#include <atomic>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <math.h>

#include "kernels.cuh"
#include "sm100.cuh"

namespace donof {

namespace mx {

constexpr int NTHREADS = 192;
constexpr int KB = 64;                // n rows per b stage (8 KB TMA boxes)
constexpr int BOX_M = 64;             // m per TMA box (128 B of bf16) = one T1 quarter
constexpr int BOX_BYTES = KB * BOX_M * 2;           // 8 KB
constexpr int STAGE_BYTES = 2 * BOX_BYTES;          // hi + lo, 16 KB
constexpr int RING = 5;                             // b stages in shared memory (80 KB)
constexpr int CS_BOX_BYTES = 128 * 64 * 2;          // 16 KB: 128 rows x 64 k
constexpr int CS_BYTES = 4 * CS_BOX_BYTES;          // K up to 256 -> 64 KB
constexpr int A2_BYTES = 4 * CS_BOX_BYTES;          // tmp split, 64 KB
constexpr int A3_BYTES = CS_BOX_BYTES;              // W split, 16 KB
// shared-memory map (offsets from a 1024-aligned base)
constexpr int OFF_CS = 0;
constexpr int OFF_RING = OFF_CS + CS_BYTES;
constexpr int OFF_A2 = OFF_RING + RING * STAGE_BYTES;
constexpr int OFF_A3 = OFF_A2 + A2_BYTES;
constexpr int OFF_DS = OFF_A3 + A3_BYTES;            // 64 floats d
constexpr int OFF_BAR = OFF_DS + 256;
constexpr int NBAR = 32;
constexpr int OFF_MISC = OFF_BAR + NBAR * 8;         // tmem base, abort flag
constexpr int SMEM_USED = OFF_MISC + 64;
constexpr int SMEM_ALLOC = SMEM_USED + 1024;         // slack for 1024-B alignment
static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory budget");

// barrier indices
constexpr int B_FULL = 0;          // +s, RING of them: stage s landed
constexpr int B_EMPTY = RING;      // +s: stage s consumed by the MMAs
constexpr int B_CS = 2 * RING;     // Cs landed
constexpr int B_T1 = B_CS + 1;     // +slot (2): T1 quarter in TMEM slot complete
constexpr int B_T1FREE = B_T1 + 2; // +slot (2): the four epilogue warps read the slot (count 4)
constexpr int B_A2 = B_T1FREE + 2; // tmp split of the aux index written (one phase per index)
constexpr int B_T2 = B_A2 + 1;     // T2 complete
constexpr int B_A3 = B_T2 + 1;     // W split written, T2 region drained
constexpr int B_Y = B_A3 + 1;      // Y MMAs of the aux index complete
constexpr int B_END = B_Y + 1;     // every MMA of the CTA complete
static_assert(B_END < NBAR, "barrier count");

// TMEM columns (512 allocated): Y accumulator [0, 256), two T1 quarter slots
// of 64 columns [256, 384), T2 [384, 512)
constexpr int TM_Y = 0;
constexpr int TM_T1 = 256;
constexpr int TM_T2 = 384;

struct Params {
    int nbf, nbf5, naux, nalpha, nbeta;
    int nb;                  // 64-wide m boxes (N = 64 * nb)
    int nkb;                 // b stages per quarter of m (ceil(nbf / KB))
    int ncs;                 // 64-wide k boxes of Cs (ceil(nbf / 64))
    int mode;                // 1: write tmp; 2: write b_pq; 3: full Lagrangian
    const float* n32;        // n (nbf5)
    const float* cj32;       // cj12 zero-padded to 64 x 64: cj32[q + 64*c] = cj12[q, c]
    const float* ck32t;      // ck12 transposed, zero-padded: ck32t[q + 64*b] = ck12[b, q]
    float* tmp_out;          // mode 1: tmp[m + nbf*q + nbf*nbf5*l]
    float* bpq_out;          // mode 2: b_pq[p + nbf5*q + nbf5^2*l]
    float* d_out;            // d[q + nbf5*l]
    float* y_part;           // per CTA: Y[m + nbf*b]
    float* k_part;           // per CTA: K[p + nbf5*q]
    int* fail;               // the context's failure word for mbarrier waits (set to 1 on a timeout)
    long long wait;          // cycle budget of every bounded wait (drains excepted)
};

using namespace sm100;

// Row of the stacked (hi, lo) operands and accumulators that holds part x
// (0 hi, 1 lo) of index q: r = 32 (q / 16) + 16 x + q % 16, so that a warp's
// 32 TMEM lanes hold the hi and lo rows of the same 16 indices.
__device__ __forceinline__ int prow(int q, int x) { return 32 * (q >> 4) + 16 * x + (q & 15); }

// Finish columns m0 .. m0+15 of tmp row q: mode 1 writes FP32 to global,
// otherwise the bf16 hi/lo split goes to A2 (rows prow(q, 0), prow(q, 1)).
__device__ __forceinline__ void finish_tmp16(const Params& P, unsigned char* sm, const float (&v)[16], int q, int m0,
                                             int l) {
    if (P.mode == 1) {
        if (q < P.nbf5) {
            float* dst = P.tmp_out + (size_t)P.nbf * P.nbf5 * l + (size_t)P.nbf * q + m0;
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (m0 + i < P.nbf) dst[i] = v[i];
        }
        return;
    }
    unsigned char* box = sm + OFF_A2 + (m0 >> 6) * CS_BOX_BYTES;
    const int kin = m0 & 63;
    const int rh = prow(q, 0), rl = prow(q, 1);
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        __align__(16) __nv_bfloat16 h[8], lo[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) split_bf16(v[cc * 8 + e], h[e], lo[e]);
        *reinterpret_cast<uint4*>(box + sw128(rh, kin + cc * 8)) = *reinterpret_cast<const uint4*>(h);
        *reinterpret_cast<uint4*>(box + sw128(rl, kin + cc * 8)) = *reinterpret_cast<const uint4*>(lo);
    }
}

// The kernel's work on CTA `cta` of `G` CTAs for one job (its aux indices
// l = cta + k G): lag_mixed_kernel runs it for one job on the whole grid,
// lag_mixed_grouped_kernel for each job of a batch on its own CTA range.  The
// tensor maps and P live in the launch's parameter space (__grid_constant__).
__device__ __forceinline__ void lag_mixed_body(const CUtensorMap& map_bhi, const CUtensorMap& map_blo,
                                               const CUtensorMap& map_cs, const Params& P, const int cta,
                                               const int G) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = saddr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + OFF_MISC);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + OFF_MISC + 16);
    auto bar = [&](int i) { return saddr(&bars[i]); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int my_count = (P.naux - cta + G - 1) / G;  // l = cta + k*G
    const int ncol = 64 * P.nb;

    if (threadIdx.x == 0) {
        *abort_flag = 0;
        for (int i = 0; i <= B_END; ++i) mbar_init(bar(i), (i == B_T1FREE || i == B_T1FREE + 1) ? 4 : 1);
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
    const uint32_t RY = tmem + TM_Y, RT1 = tmem + TM_T1, RT2 = tmem + TM_T2;

    if (warp == 4) {
        // ------------------------------------------------------------ producer
        // stages in the order the MMAs consume them: per aux index, per 64-column
        // quarter of m, per 32 rows of n (hi and lo box of the same rows)
        if (lane == 0 && my_count > 0) {
            mbar_expect_tx(bar(B_CS), (uint32_t)(P.ncs * CS_BOX_BYTES));
            for (int kb = 0; kb < P.ncs; ++kb)
                tma_load_2d(sbase + OFF_CS + kb * CS_BOX_BYTES, &map_cs, bar(B_CS), kb * 64, 0);
            int it = 0;
            bool ok = true;
            for (int li = 0; li < my_count && ok; ++li) {
                const int l = cta + li * G;
                for (int qb = 0; qb < P.nb && ok; ++qb) {
                    for (int kb = 0; kb < P.nkb; ++kb, ++it) {
                        const int s = it % RING;
                        const uint32_t ph = (uint32_t)((it / RING) & 1);
                        if (!mbar_wait(bar(B_EMPTY + s), ph ^ 1u, abort_flag, P.wait)) { ok = false; break; }
                        mbar_expect_tx(bar(B_FULL + s), (uint32_t)STAGE_BYTES);
                        const uint32_t st = sbase + OFF_RING + s * STAGE_BYTES;
                        tma_load_4d(st, &map_bhi, bar(B_FULL + s), 0, kb * KB, qb, l);
                        tma_load_4d(st + BOX_BYTES, &map_blo, bar(B_FULL + s), 0, kb * KB, qb, l);
                    }
                }
            }
            // drain: every issued stage must have landed before the CTA exits
            const int issued = it;
            for (int j = (issued > RING ? issued - RING : 0); j < issued; ++j) {
                const int s = j % RING;
                mbar_drain(bar(B_FULL + s), (uint32_t)((j / RING) & 1));
            }
            mbar_drain(bar(B_CS), 0);
        }
    } else if (warp == 5) {
        // ------------------------------------------------------------ MMA issuer
        // Issue order per aux index l: its T1 quarters, T2(l), then (while the
        // epilogue drains T2(l) and builds W(l)) up to two T1 quarters of l+1 into
        // the free slots, and Y(l) as soon as W(l) is ready.
        if (lane == 0 && my_count > 0) {
            const uint32_t id_t1 = idesc(128, BOX_M, 0, 1);
            const uint32_t id_t2 = idesc(128, 128, 0, 0);
            const uint32_t id_y = idesc(128, ncol, 0, 1);
            bool ok = mbar_wait(bar(B_CS), 0, abort_flag, P.wait);
            fence_after();
            int it = 0;          // ring stages consumed
            int tq = 0;          // T1 quarters issued (slot = tq & 1)
            int y_li = -1;       // aux index whose Y MMAs are still to be issued
            // Shared-memory descriptors are linear in the address (addr >> 4 in the low 14
            // bits, no carry below 256 KB): the fixed bases are built once, offsets are adds.
            const uint64_t dA3 = sdesc(sbase + OFF_A3, 16, 1024);
            const uint64_t dA2k = sdesc(sbase + OFF_A2, 16, 1024);            // A2 as a K-major operand
            const uint64_t dA2m = sdesc(sbase + OFF_A2, CS_BOX_BYTES, 1024);  // A2 as an MN-major operand
            const uint64_t dCS = sdesc(sbase + OFF_CS, 16, 1024);
            auto issue_y = [&]() {
                // Y: RY[j, m] += sum_q A3[j, q] tmp_x[q, m]  (A2 read as an MN-major operand)
                // K rows q = 16 ks + i of the hi part are A2 rows 32 ks + i, the lo part 32 ks + 16 + i
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {
                    umma(RY, dA3 + (uint64_t)(2 * ks), dA2m + (uint64_t)(256 * ks), id_y, (y_li | ks) ? 1u : 0u);
                    umma(RY, dA3 + (uint64_t)(2 * ks), dA2m + (uint64_t)(256 * ks + 128), id_y, 1u);
                }
                umma_commit(bar(B_Y));
                y_li = -1;
            };
            // Bounded wait that issues the pending Y MMAs as soon as W is ready.
            auto wait_poll = [&](uint32_t b, uint32_t parity) -> bool {
                const long long t0 = clock64();
                while (!mbar_test(b, parity)) {
                    if (y_li >= 0 && mbar_test(bar(B_A3), (uint32_t)(y_li & 1))) {
                        fence_after();
                        issue_y();
                    }
                    if (*abort_flag) return false;
                    if (clock64() - t0 > P.wait) { *abort_flag = 1; return false; }
                    __nanosleep(32);  // leave issue slots to the epilogue warp on this SM sub-partition
                }
                return true;
            };
            // T1 quarter: slot[j, m'] = sum_n Cs[j, n] b_x[n, m'] over one 64-column box of m
            auto t1_quarter = [&]() -> bool {
                const int slot = tq & 1;
                if (!wait_poll(bar(B_T1FREE + slot), (uint32_t)(((tq >> 1) & 1) ^ 1))) return false;
                fence_after();
                const uint32_t d = RT1 + slot * BOX_M;
                for (int kb = 0; kb < P.nkb; ++kb, ++it) {
                    const int s = it % RING;
                    if (y_li >= 0 && mbar_test(bar(B_A3), (uint32_t)(y_li & 1))) {
                        fence_after();
                        issue_y();
                    }
                    if (!wait_poll(bar(B_FULL + s), (uint32_t)((it / RING) & 1))) return false;
                    fence_after();
                    // n rows kb*64 + 16 ks of Cs: box kb (KB = 64 = one box), 32 bytes per ks
                    const uint64_t a0 = dCS + (uint64_t)((kb * CS_BOX_BYTES) >> 4);
                    const uint64_t bh0 = sdesc(sbase + OFF_RING + s * STAGE_BYTES, BOX_BYTES, 1024);
                    const uint64_t bl0 = bh0 + (uint64_t)(BOX_BYTES >> 4);
#pragma unroll
                    for (int ks = 0; ks < KB / 16; ++ks) {
                        umma(d, a0 + (uint64_t)(2 * ks), bh0 + (uint64_t)(128 * ks), id_t1, (kb | ks) ? 1u : 0u);
                        umma(d, a0 + (uint64_t)(2 * ks), bl0 + (uint64_t)(128 * ks), id_t1, 1u);
                    }
                    umma_commit(bar(B_EMPTY + s));
                }
                umma_commit(bar(B_T1 + slot));
                ++tq;
                return true;
            };
            const int ahead_max = P.nb < 2 ? P.nb : 2;
            int ahead = 0;  // quarters of the current index issued early
            for (int li = 0; li < my_count && ok; ++li) {
                const uint32_t lph = (uint32_t)(li & 1);
                for (int qb = ahead; qb < P.nb && ok; ++qb) ok = t1_quarter();
                ahead = 0;
                if (!ok) break;
                if (P.mode == 1) continue;
                // T2: RT2[j, j'] = sum_m A2[j, m] Cs[j', m]
                if (!wait_poll(bar(B_A2), lph)) { ok = false; break; }
                fence_after();
                for (int ks = 0; ks < ncol / 16; ++ks) {
                    // m offset 16 ks: box ks / 4, 32 bytes per ks inside it
                    const uint64_t off = (uint64_t)((ks >> 2) * (CS_BOX_BYTES >> 4) + 2 * (ks & 3));
                    umma(RT2, dA2k + off, dCS + off, id_t2, ks ? 1u : 0u);
                }
                umma_commit(bar(B_T2));
                if (P.mode == 3) y_li = li;
                // T1 of the next index into the slots the epilogue has already drained
                if (li + 1 < my_count)
                    for (; ahead < ahead_max && ok; ++ahead) ok = t1_quarter();
                if (!ok) break;
                // W(l) ready (and the T2 region drained)
                if (!mbar_wait(bar(B_A3), lph, abort_flag, P.wait)) { ok = false; break; }
                fence_after();
                if (y_li >= 0) issue_y();
            }
            umma_commit(bar(B_END));
            mbar_drain(bar(B_END), 0);  // every MMA of this CTA has completed
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 0-3)
        // Accumulator rows are stacked as prow(q, x): warp g holds q in [16 g, 16 g + 16),
        // the hi part in lanes 0-15 and the lo part in lanes 16-31, so every hi + lo sum
        // is a shuffle between lanes i and i + 16 of one warp.
        const int q = 16 * warp + (lane & 15);  // q (T1/T2 rows) or b (Y rows)
        const int x = lane >> 4;                 // 0: hi row, 1: lo row
        const int off = 32 * x;                  // T2/W: this thread finishes p (or b) in [off, off + 32)
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        volatile int* epi_ok = reinterpret_cast<volatile int*>(sm + OFF_MISC + 32);
        // one thread waits, the 128 epilogue threads agree on the outcome
        auto epi_wait = [&](int b, uint32_t parity) -> bool {
            if (threadIdx.x == 0) *epi_ok = mbar_wait(bar(b), parity, abort_flag, P.wait) ? 1 : 0;
            epi_sync();
            const bool r = *epi_ok != 0;
            epi_sync();
            if (r) fence_after();
            return r;
        };
        // one warp waits on its own (lane 0 polls, the warp agrees)
        auto warp_wait = [&](int b, uint32_t parity) -> bool {
            int r = 1;
            if (lane == 0) r = mbar_wait(bar(b), parity, abort_flag, P.wait) ? 1 : 0;
            r = __shfl_sync(0xffffffffu, r, 0);
            if (r) fence_after();
            return r != 0;
        };
        // the four warps agree to go on unless a wait failed somewhere (every failed
        // wait sets the abort flag)
        auto agree = [&](bool mine) -> bool {
            if (!mine) *abort_flag = 1;
            epi_sync();
            if (threadIdx.x == 0) *epi_ok = *abort_flag ? 0 : 1;
            epi_sync();
            const bool r = *epi_ok != 0;
            epi_sync();
            return r;
        };
        // ck12 (transposed, 16 KB) is read through L1 where W is built: the shared
        // memory it would take holds a fifth stage of the b ring instead.
        // row q of cj12 restricted to this thread's half of the columns, kept in registers
        float cjr[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) cjr[i] = __ldg(P.cj32 + q + 64 * (off + i));
        epi_sync();
        float* ds = reinterpret_cast<float*>(sm + OFF_DS);

        // columns 32 c .. 32 c + 31 of tmp row q: the hi lane finishes the first 16,
        // the lo lane the last 16
        auto drain32 = [&](const uint32_t (&r)[32], int c, int l) {
            float v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float send = __uint_as_float(x ? r[i] : r[16 + i]);
                const float keep = __uint_as_float(x ? r[16 + i] : r[i]);
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
            }
            finish_tmp16(P, sm, v, q, 32 * c + 16 * x, l);
        };

        bool ok = true;
        int tq = 0;  // T1 quarters drained (slot = tq & 1)
        for (int li = 0; li < my_count && ok; ++li) {
            const int l = cta + li * G;
            const uint32_t lph = (uint32_t)(li & 1);
            // ---- T1 drain, one 64-column quarter of m at a time, each warp on its own:
            // tmp[m, q] = D1[prow(q, 0), m] + D1[prow(q, 1), m]
            bool wok = true;
            for (int qb = 0; qb < P.nb; ++qb) {
                const int t = tq + qb, slot = t & 1;
                if (!warp_wait(B_T1 + slot, (uint32_t)((t >> 1) & 1))) { wok = false; break; }
                // A2 is read by the Y MMAs of the previous index
                if (qb == 0 && li > 0 && P.mode == 3 && !warp_wait(B_Y, (uint32_t)((li - 1) & 1))) { wok = false; break; }
                const uint32_t src = RT1 + slot * BOX_M + lane_addr;
                uint32_t ra[32], rb[32];
                tmem_issue32(src, ra);
                tmem_issue32(src + 32, rb);
                tmem_wait_ld();
                // the slot can take the next quarter while this one is finished
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(bar(B_T1FREE + slot));
                drain32(ra, 2 * qb, l);
                drain32(rb, 2 * qb + 1, l);
            }
            tq += P.nb;
            if (P.mode != 1) fence_async_smem();  // A2 written by the generic proxy, read by the MMAs
            if (!agree(wok)) { ok = false; break; }
            if (P.mode == 1) continue;
            if (threadIdx.x == 0) mbar_arrive(bar(B_A2));
            // ---- T2 drain: b_pq[p, q] = sum over x, x' of D2[prow(q, x), prow(p, x')]
            if (!epi_wait(B_T2, lph)) { ok = false; break; }
            float bq[32];  // b_pq for p = off + i
            {
                float lowp[32], highp[32];  // this row's sums over x' for p in [0, 32) and [32, 64)
                uint32_t r0[32], r1[32];
                tmem_issue32(RT2 + lane_addr + 0, r0);
                tmem_issue32(RT2 + lane_addr + 32, r1);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    lowp[i] = __uint_as_float(r0[i]) + __uint_as_float(r0[16 + i]);
                    lowp[16 + i] = __uint_as_float(r1[i]) + __uint_as_float(r1[16 + i]);
                }
                tmem_issue32(RT2 + lane_addr + 64, r0);
                tmem_issue32(RT2 + lane_addr + 96, r1);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    highp[i] = __uint_as_float(r0[i]) + __uint_as_float(r0[16 + i]);
                    highp[16 + i] = __uint_as_float(r1[i]) + __uint_as_float(r1[16 + i]);
                }
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const float send = x ? lowp[i] : highp[i];
                    bq[i] = (x ? highp[i] : lowp[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
                }
            }
            // the T2 region is free again once every thread's loads are done
            fence_before();
            const bool own_diag = (q >= off) && (q < off + 32);  // this thread holds b_pq[q, q]
            {
                float dq = 0.f;
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (off + i == q) dq = bq[i];
                if (own_diag) {
                    if (q >= P.nbf5) dq = 0.f;
                    ds[q] = dq;
                    if (q < P.nbf5 && P.mode == 2) P.d_out[q + (size_t)P.nbf5 * l] = dq;
                }
                if (q < P.nbf5 && P.mode == 2) {  // J/K ingredients are only needed by JKH_MO
                    float* dst = P.bpq_out + (size_t)P.nbf5 * P.nbf5 * l + (size_t)P.nbf5 * q + off;
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (off + i < P.nbf5) dst[i] = bq[i];
                    // K_MO partial sums of this CTA, stored transposed (kp[q + nbf5*p]) so that
                    // the reductions of a warp are coalesced; each address has one writer
                    float* kp = P.k_part + (size_t)cta * P.nbf5 * P.nbf5 + q;
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (off + i < P.nbf5) atomicAdd(kp + (size_t)P.nbf5 * (off + i), bq[i] * bq[i]);
                }
            }
            epi_sync();
            if (P.mode != 2) {
                // W[q, b] = delta_qb (n'_q d_q + t_q) - ck12[b, q] b_pq[b, q],  t_q = sum_q' cj12[q, q'] d_q'
                float tpart = 0.f;
#pragma unroll
                for (int i = 0; i < 32; ++i) tpart += cjr[i] * ds[off + i];
                const float t = tpart + __shfl_xor_sync(0xffffffffu, tpart, 16);
                float diag = 0.f;
                if (own_diag && q < P.nbf5) {
                    const bool dj = (P.nbeta > 0) && (q < P.nbeta || q >= P.nalpha);
                    diag = (dj ? P.n32[q] * ds[q] : 0.f) + t;
                }
                // This thread builds part of A3 row b = q (hi: prow(q, 0), lo: prow(q, 1)) over
                // K = k in [off, off + 32), using the symmetry of b_pq (bq[i] = b_pq[off + i, q]):
                // W[k, q] = delta_kq (n'_q d_q + t_q) - ck12[q, k] b_pq[q, k]
                const float4* ckrow = reinterpret_cast<const float4*>(P.ck32t + q * 64 + off);  // ck12[q, off + i]
                const int rh = prow(q, 0), rl = prow(q, 1);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float4 k0 = __ldg(ckrow + 2 * c), k1 = __ldg(ckrow + 2 * c + 1);
                    const float ck8[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
                    __align__(16) __nv_bfloat16 h[8], lo[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int i = 8 * c + e, k = off + i;
                        float w = 0.f;
                        if (q < P.nbf5 && k < P.nbf5) w = -ck8[e] * bq[i] + (k == q ? diag : 0.f);
                        split_bf16(w, h[e], lo[e]);
                    }
                    *reinterpret_cast<uint4*>(sm + OFF_A3 + sw128(rh, off + 8 * c)) = *reinterpret_cast<const uint4*>(h);
                    *reinterpret_cast<uint4*>(sm + OFF_A3 + sw128(rl, off + 8 * c)) = *reinterpret_cast<const uint4*>(lo);
                }
            }
            fence_async_smem();
            fence_before();
            epi_sync();
            if (threadIdx.x == 0) mbar_arrive(bar(B_A3));
        }
        // ---- final: Y partial (mode 3): Y[m, b] = D3[prow(b, 0), m] + D3[prow(b, 1), m]
        if (ok && my_count > 0 && P.mode == 3) {
            if (epi_wait(B_Y, (uint32_t)((my_count - 1) & 1))) {
                for (int c = 0; c < ncol / 32; ++c) {
                    uint32_t r[32];
                    tmem_issue32(RY + lane_addr + c * 32, r);
                    tmem_wait_ld();
                    const int m0 = 32 * c + 16 * x;
                    float* dst = P.y_part + (size_t)cta * P.nbf * P.nbf5 + (size_t)P.nbf * q + m0;
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const float send = __uint_as_float(x ? r[i] : r[16 + i]);
                        const float v = __uint_as_float(x ? r[16 + i] : r[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
                        if (q < P.nbf5 && m0 + i < P.nbf) dst[i] = v;
                    }
                }
            }
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

__global__ void __launch_bounds__(NTHREADS, 1)
lag_mixed_kernel(const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo,
                 const __grid_constant__ CUtensorMap map_cs, const Params P) {
    lag_mixed_body(map_bhi, map_blo, map_cs, P, (int)blockIdx.x, (int)gridDim.x);
}

// Several jobs in one launch: job j owns the CTAs [cta0[j], cta0[j + 1]) and
// runs lag_mixed_body on them with its own tensor maps and parameters.
constexpr int GROUP_MAX = 48;  // 48 jobs' maps and parameters fit the 32 KB of kernel parameters
struct GroupParams {
    CUtensorMap maps[GROUP_MAX][3];  // b_hi, b_lo, Cs
    Params P[GROUP_MAX];
    int cta0[GROUP_MAX + 1];
    int njobs;
};
static_assert(sizeof(GroupParams) <= 32000, "kernel parameter space");

__global__ void __launch_bounds__(NTHREADS, 1) lag_mixed_grouped_kernel(const __grid_constant__ GroupParams GP) {
    int j = 0;
    while (j + 1 < GP.njobs && GP.cta0[j + 1] <= (int)blockIdx.x) ++j;
    const int cta = (int)blockIdx.x - GP.cta0[j], G = GP.cta0[j + 1] - GP.cta0[j];
    lag_mixed_body(GP.maps[j][0], GP.maps[j][1], GP.maps[j][2], GP.P[j], cta, G);
}

// ---------------------------------------------------------------- helpers
// b = hi + lo in the quarter-major layout the mixed kernel streams: element
// (m, n, l) at [mi + 64 n + 64 nbf qb + 64 nbf nb l] with m = 64 qb + mi, so
// that the 32-row stages of one 64-column quarter are contiguous 4 KB blocks;
// m >= nbf is zero.
__global__ void split_b_kernel(const double* __restrict__ b, int nbf, int nb, long long naux,
                               __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    const long long total = 64LL * nbf * nb * naux;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int mi = (int)(i & 63);
        const long long r = i >> 6;
        const int n = (int)(r % nbf);
        const long long r2 = r / nbf;
        const int qb = (int)(r2 % nb);
        const long long l = r2 / nb;
        const int m = 64 * qb + mi;
        double v = (m < nbf) ? b[m + (long long)nbf * n + (long long)nbf * nbf * l] : 0.0;
        const __nv_bfloat16 h = __double2bfloat16(v);
        const __nv_bfloat16 lw = __double2bfloat16(v - (double)__bfloat162float(h));
        hi[i] = h;
        lo[i] = lw;
    }
}

// split_c_kernel for every job of a batch: job blockIdx.y, its arrays from a device table.
__global__ void split_c_grouped_kernel(const MixedSplitJob* __restrict__ jobs) {
    const MixedSplitJob J = jobs[blockIdx.y];
    const int total = J.ldk * 128;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int k = i % J.ldk, j = i / J.ldk;
        const int q = 16 * (j >> 5) + (j & 15), x = (j >> 4) & 1;  // j = prow(q, x)
        double v = (k < J.nbf && q < J.nbf5) ? J.C[k + (long long)J.nbf * q] : 0.0;
        const __nv_bfloat16 h = __double2bfloat16(v);
        static_cast<__nv_bfloat16*>(J.cs)[i] = (x == 0) ? h : __double2bfloat16(v - (double)__bfloat162float(h));
    }
}

// Cs[k + ldk*j] = C_x[k, q] for j = prow(q, x) (x = 0: bf16 hi, 1: lo); zero beyond nbf5 / nbf.
__global__ void split_c_kernel(const double* __restrict__ C, int nbf, int nbf5, int ldk,
                               __nv_bfloat16* __restrict__ cs) {
    const int total = ldk * 128;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int k = i % ldk, j = i / ldk;
        const int q = 16 * (j >> 5) + (j & 15), x = (j >> 4) & 1;  // j = prow(q, x)
        double v = (k < nbf && q < nbf5) ? C[k + (long long)nbf * q] : 0.0;
        const __nv_bfloat16 h = __double2bfloat16(v);
        cs[i] = (x == 0) ? h : __double2bfloat16(v - (double)__bfloat162float(h));
    }
}

// n, cj12 and ck12 of the functional in FP32, zero-padded to 64:
// n32[q], cj32[q + 64 c] = cj12[q, c], ck32[q + 64 b] = ck12[b, q]
__global__ void prep_coef_kernel(const double* __restrict__ n, const double* __restrict__ cj12,
                                 const double* __restrict__ ck12, int nbf5, float* __restrict__ n32,
                                 float* __restrict__ cj32, float* __restrict__ ck32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 64 * 64; i += gridDim.x * blockDim.x) {
        const int r = i & 63, c = i >> 6;
        const bool in = r < nbf5 && c < nbf5;
        cj32[i] = in ? (float)cj12[r + nbf5 * c] : 0.f;
        ck32[i] = in ? (float)ck12[c + nbf5 * r] : 0.f;
        if (i < 64) n32[i] = (i < nbf5) ? (float)n[i] : 0.f;
    }
}

// Same for an n x n matrix stored transposed in the partials: out[c + n*r] = sum_g part[r + n*c + g*stride]
__global__ void reduce_f32_to_f64_t(const float* __restrict__ part, long long stride, int parts, int n,
                                    double* __restrict__ out) {
    const long long count = (long long)n * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int g = 0; g < parts; ++g) s += (double)part[i + g * stride];
        const long long r = i % n, c = i / n;
        out[c + n * r] = s;
    }
}

__global__ void f32_to_f64(const float* __restrict__ a, long long count, double* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)a[i];
}

}  // namespace mx

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    // looked up once (thread-safe static initialisation)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    }();
    return fn;
}

}  // namespace

// Tensor map with 128-byte swizzle and zero fill outside the tensor (no
// interleave): bf16 for the mixed kernels of this file and mixed_general.cu,
// 8-bit for the digit slices of ozaki.cu.
static int make_tmap(donof_ctx* ctx, CUtensorMap* map, CUtensorMapDataType dtype, const void* base, int rank,
                     const cuuint64_t* dims, const cuuint64_t* strides_bytes, const cuuint32_t* box);

int make_tmap_bf16(donof_ctx* ctx, CUtensorMap* map, const void* base, int rank, const cuuint64_t* dims,
             const cuuint64_t* strides_bytes, const cuuint32_t* box) {
    return make_tmap(ctx, map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, rank, dims, strides_bytes, box);
}

int make_tmap_u8(donof_ctx* ctx, CUtensorMap* map, const void* base, int rank, const cuuint64_t* dims,
                 const cuuint64_t* strides_bytes, const cuuint32_t* box) {
    return make_tmap(ctx, map, CU_TENSOR_MAP_DATA_TYPE_UINT8, base, rank, dims, strides_bytes, box);
}

static int make_tmap(donof_ctx* ctx, CUtensorMap* map, CUtensorMapDataType dtype, const void* base, int rank,
                     const cuuint64_t* dims, const cuuint64_t* strides_bytes, const cuuint32_t* box) {
    auto fn = encode_fn();
    if (!fn) {
        set_error(ctx, "cuTensorMapEncodeTiled is not available");
        return DONOF_ERR_CUDA;
    }
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = fn(map, dtype, rank, const_cast<void*>(base), dims, strides_bytes, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error(ctx, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return DONOF_ERR_CUDA;
    }
    return DONOF_OK;
}

namespace {

int ldm_of(int nbf) { return (nbf + 7) / 8 * 8; }

// Scratch of the mixed form inside the job: [Cs | n32 | cj32 | ck32 | d | y_part | k_part | tmp/bpq out]
struct MixedScratch {
    __nv_bfloat16* cs;
    float *n32, *cj32, *ck32, *d, *ypart, *kpart;
    double *Y, *Kd, *dd;
};

int mixed_prepare(donof_job* job, cudaStream_t st, const double* C, int nbf5, MixedScratch* S, int grid) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    const int ldk = ldm_of(nbf);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_cs = take(sizeof(__nv_bfloat16) * (size_t)ldk * 128);
    const size_t o_n = take(sizeof(float) * 64);
    const size_t o_cj = take(sizeof(float) * 64 * 64);
    const size_t o_ck = take(sizeof(float) * 64 * 64);
    const size_t o_d = take(sizeof(float) * (size_t)nbf5 * naux);
    const size_t o_y = take(sizeof(float) * (size_t)grid * nbf * nbf5);
    const size_t o_k = take(sizeof(float) * (size_t)grid * nbf5 * nbf5);
    const size_t o_Y = take(sizeof(double) * (size_t)nbf * nbf5);
    const size_t o_K = take(sizeof(double) * (size_t)nbf5 * nbf5);
    const size_t o_dd = take(sizeof(double) * (size_t)nbf5 * naux);
    DONOF_CHECK(job->W.ensure(ctx, off));  // the FP64 form's W buffer doubles as the mixed scratch
    char* base = job->W.as<char>();
    S->cs = reinterpret_cast<__nv_bfloat16*>(base + o_cs);
    S->n32 = reinterpret_cast<float*>(base + o_n);
    S->cj32 = reinterpret_cast<float*>(base + o_cj);
    S->ck32 = reinterpret_cast<float*>(base + o_ck);
    S->d = reinterpret_cast<float*>(base + o_d);
    S->ypart = reinterpret_cast<float*>(base + o_y);
    S->kpart = reinterpret_cast<float*>(base + o_k);
    S->Y = reinterpret_cast<double*>(base + o_Y);
    S->Kd = reinterpret_cast<double*>(base + o_K);
    S->dd = reinterpret_cast<double*>(base + o_dd);
    // the kernel accumulates its K_MO partial sums into these
    DONOF_CUDA(ctx, cudaMemsetAsync(S->kpart, 0, sizeof(float) * (size_t)grid * nbf5 * nbf5, st));
    mx::split_c_kernel<<<(ldk * 128 + 255) / 256, 256, 0, st>>>(C, nbf, nbf5, ldk, S->cs); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int launch_mixed(donof_job* job, cudaStream_t st, int nbf5, int nalpha, int nbeta, int mode, const MixedScratch& S,
                 float* tmp_out, float* bpq_out, int grid) {
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux;
    const int ldm = ldm_of(nbf);
    CUtensorMap mhi, mlo, mcs;
    {
        // quarter-major split: [mi + 64 n + 64 nbf qb + 64 nbf nb l], m = 64 qb + mi
        const int nb = (nbf + 63) / 64;
        cuuint64_t dims[4] = {64, (cuuint64_t)nbf, (cuuint64_t)nb, (cuuint64_t)naux};
        cuuint64_t strides[3] = {128, (cuuint64_t)128 * nbf, (cuuint64_t)128 * nbf * nb};
        cuuint32_t box[4] = {mx::BOX_M, mx::KB, 1, 1};
        DONOF_CHECK(make_tmap_bf16(ctx, &mhi, job->b16hi, 4, dims, strides, box));
        DONOF_CHECK(make_tmap_bf16(ctx, &mlo, job->b16lo, 4, dims, strides, box));
    }
    {
        cuuint64_t dims[2] = {(cuuint64_t)nbf, 128};
        cuuint64_t strides[1] = {(cuuint64_t)ldm * 2};
        cuuint32_t box[2] = {64, 128};
        DONOF_CHECK(make_tmap_bf16(ctx, &mcs, S.cs, 2, dims, strides, box));
    }
    mx::Params P{};
    P.nbf = nbf; P.nbf5 = nbf5; P.naux = naux; P.nalpha = nalpha; P.nbeta = nbeta;
    P.nb = (nbf + 63) / 64;
    P.nkb = (nbf + mx::KB - 1) / mx::KB;
    P.ncs = (nbf + 63) / 64;
    P.mode = mode;
    P.n32 = S.n32; P.cj32 = S.cj32; P.ck32t = S.ck32;
    P.tmp_out = tmp_out; P.bpq_out = bpq_out; P.d_out = S.d; P.y_part = S.ypart; P.k_part = S.kpart;
    P.fail = ctx->fail_dev ? ctx->fail_dev + FAIL_MBAR : nullptr;
    P.wait = sm100::wait_budget(ctx->wait_limit);
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(mx::lag_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             mx::SMEM_ALLOC));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    prof_begin(ctx, st);
    mx::lag_mixed_kernel<<<grid, mx::NTHREADS, mx::SMEM_ALLOC, st>>>(mhi, mlo, mcs, P); count_launch();
    prof_end(ctx, st);
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

// One launch of lag_mixed_grouped_kernel per GROUP_MAX jobs (mode 3: the Y
// partials of every job's CTAs into its ypart).
int launch_mixed_grouped_impl(donof_ctx* ctx, cudaStream_t st, const MixedGroupJob* jobs, int njobs) {
    static std::atomic<unsigned long long> attr_mask{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_mask.load(std::memory_order_acquire) & bit)) {
        DONOF_CUDA(ctx, cudaFuncSetAttribute(mx::lag_mixed_grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             mx::SMEM_ALLOC));
        attr_mask.fetch_or(bit, std::memory_order_acq_rel);
    }
    for (int j0 = 0; j0 < njobs; j0 += mx::GROUP_MAX) {
        const int nj = njobs - j0 < mx::GROUP_MAX ? njobs - j0 : mx::GROUP_MAX;
        mx::GroupParams GP;
        memset(&GP, 0, sizeof(GP));
        GP.njobs = nj;
        int cta = 0;
        for (int i = 0; i < nj; ++i) {
            const MixedGroupJob& g = jobs[j0 + i];
            donof_job* job = g.job;
            const int nbf = job->nbf, naux = job->naux, ldm = ldm_of(nbf), nb = (nbf + 63) / 64;
            {
                cuuint64_t dims[4] = {64, (cuuint64_t)nbf, (cuuint64_t)nb, (cuuint64_t)naux};
                cuuint64_t strides[3] = {128, (cuuint64_t)128 * nbf, (cuuint64_t)128 * nbf * nb};
                cuuint32_t box[4] = {mx::BOX_M, mx::KB, 1, 1};
                DONOF_CHECK(make_tmap_bf16(ctx, &GP.maps[i][0], job->b16hi, 4, dims, strides, box));
                DONOF_CHECK(make_tmap_bf16(ctx, &GP.maps[i][1], job->b16lo, 4, dims, strides, box));
            }
            {
                cuuint64_t dims[2] = {(cuuint64_t)nbf, 128};
                cuuint64_t strides[1] = {(cuuint64_t)ldm * 2};
                cuuint32_t box[2] = {64, 128};
                DONOF_CHECK(make_tmap_bf16(ctx, &GP.maps[i][2], g.cs, 2, dims, strides, box));
            }
            mx::Params& P = GP.P[i];
            P.nbf = nbf; P.nbf5 = g.nbf5; P.naux = naux; P.nalpha = g.nalpha; P.nbeta = g.nbeta;
            P.nb = nb;
            P.nkb = (nbf + mx::KB - 1) / mx::KB;
            P.ncs = (nbf + 63) / 64;
            P.mode = 3;
            P.n32 = g.n32; P.cj32 = g.cj32; P.ck32t = g.ck32;
            P.y_part = g.ypart;
            P.fail = ctx->fail_dev ? ctx->fail_dev + FAIL_MBAR : nullptr;
            P.wait = sm100::wait_budget(ctx->wait_limit);
            GP.cta0[i] = cta;
            cta += g.ctas;
        }
        GP.cta0[nj] = cta;
        mx::lag_mixed_grouped_kernel<<<cta, mx::NTHREADS, mx::SMEM_ALLOC, st>>>(GP); count_launch();
        DONOF_CUDA(ctx, cudaGetLastError());
    }
    return DONOF_OK;
}

int mixed_grid(donof_job* job) { return job->naux < ctx_ctas(job->ctx) ? job->naux : ctx_ctas(job->ctx); }

int check_mixed(donof_job* job, int nbf5) {
    if (job->b16hi == nullptr) {
        set_error(job->ctx, "mixed precision requested but the job holds no bf16 split of b");
        return DONOF_ERR_ARG;
    }
    if (nbf5 < 1 || nbf5 > job->nbf) {
        set_error(job->ctx, "nbf5 must be in [1, nbf] (got nbf=%d nbf5=%d)", job->nbf, nbf5);
        return DONOF_ERR_ARG;
    }
    return DONOF_OK;
}

}  // namespace

bool mixed_fused_fits(int nbf, int nbf5) { return !mixed_general_needed(nbf, nbf5); }

int launch_mixed_grouped(donof_ctx* ctx, cudaStream_t st, const MixedGroupJob* jobs, int njobs) {
    return launch_mixed_grouped_impl(ctx, st, jobs, njobs);
}

int split_c_grouped(donof_ctx* ctx, cudaStream_t st, const MixedSplitJob* d_jobs, int njobs, int max_ldk) {
    const int blocks = (max_ldk * 128 + 255) / 256;
    mx::split_c_grouped_kernel<<<dim3(blocks, njobs), 256, 0, st>>>(d_jobs); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int prep_coef(donof_ctx* ctx, cudaStream_t st, const double* n, const double* cj12, const double* ck12, int nbf5,
              float* n32, float* cj32, float* ck32) {
    mx::prep_coef_kernel<<<16, 256, 0, st>>>(n, cj12, ck12, nbf5, n32, cj32, ck32); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int mixed_ldk(int nbf) { return ldm_of(nbf); }

int convert_b_f32(donof_job* job) {
    // b split into bf16 hi + lo (the mixed form's copy of b)
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, nb = (nbf + 63) / 64;
    const size_t count = (size_t)64 * nb * nbf * job->naux;
    void* hi = nullptr;
    void* lo = nullptr;
    DONOF_CHECK(dev_alloc(ctx, &hi, sizeof(__nv_bfloat16) * count));
    int s = dev_alloc(ctx, &lo, sizeof(__nv_bfloat16) * count);
    if (s != DONOF_OK) {
        dev_free(ctx, hi);
        return s;
    }
    mx::split_b_kernel<<<8 * ctx->sm_count, 256, 0, ctx->stream>>>(job->b, nbf, nb, (long long)job->naux,
                                                                   static_cast<__nv_bfloat16*>(hi),
                                                                   static_cast<__nv_bfloat16*>(lo)); count_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        dev_free(ctx, hi);
        dev_free(ctx, lo);
        set_error(ctx, "bf16 split of b: %s", cudaGetErrorString(e));
        return DONOF_ERR_CUDA;
    }
    job->b16hi = hi;
    job->b16lo = lo;
    return DONOF_OK;
}

int transforms_mixed(donof_job* job, cudaStream_t st, const double* C, int nbf5) {
    DONOF_CHECK(check_mixed(job, nbf5));
    if (mixed_general_needed(job->nbf, nbf5)) return transforms_mixed_general(job, st, C, nbf5);
    donof_ctx* ctx = job->ctx;
    const int naux = job->naux, grid = mixed_grid(job);
    MixedScratch S;
    DONOF_CHECK(mixed_prepare(job, st, C, nbf5, &S, grid));
    DONOF_CHECK(job->tmp.ensure(ctx, sizeof(float) * (size_t)nbf5 * nbf5 * naux));
    float* bpq32 = job->tmp.as<float>();
    DONOF_CHECK(launch_mixed(job, st, nbf5, nbf5, nbf5, 2, S, nullptr, bpq32, grid));
    DONOF_CHECK(job->bpq.ensure(ctx, sizeof(double) * (size_t)nbf5 * nbf5 * naux));
    const long long cnt = (long long)nbf5 * nbf5 * naux;
    mx::f32_to_f64<<<4 * ctx->sm_count, 256, 0, st>>>(bpq32, cnt, job->bpq.as<double>()); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

int mixed_t1_debug(donof_job* job, cudaStream_t st, const double* C, int nbf5, float* tmp_out) {
    DONOF_CHECK(check_mixed(job, nbf5));
    if (mixed_general_needed(job->nbf, nbf5)) return mixed_t1_general(job, st, C, nbf5, tmp_out);
    const int grid = mixed_grid(job);
    MixedScratch S;
    DONOF_CHECK(mixed_prepare(job, st, C, nbf5, &S, grid));
    return launch_mixed(job, st, nbf5, nbf5, nbf5, 1, S, tmp_out, nullptr, grid);
}

int lagrange2_mixed(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* H,
                    const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta, double* elag,
                    double* Hmat, double* E) {
    DONOF_CHECK(check_mixed(job, nbf5));
    if (mixed_general_needed(job->nbf, nbf5))
        return lagrange2_mixed_general(job, st, C, n, H, cj12, ck12, nbf5, nalpha, nbeta, elag, Hmat, E);
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, grid = mixed_grid(job);
    MixedScratch S;
    DONOF_CHECK(mixed_prepare(job, st, C, nbf5, &S, grid));
    mx::prep_coef_kernel<<<16, 256, 0, st>>>(n, cj12, ck12, nbf5, S.n32, S.cj32, S.ck32); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(launch_mixed(job, st, nbf5, nalpha, nbeta, 3, S, nullptr, nullptr, grid));
    // Y (FP64) = sum over CTAs of the FP32 partials; H_mat, elag and E_elec in FP64
    return elag_tail_f64(job, st, C, H, n, nbf5, S.ypart, true, grid, (long long)nbf * nbf5, Hmat, elag, E);
}

int jkh_mo_mixed(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5, double* J, double* K,
                 double* Hcore) {
    DONOF_CHECK(check_mixed(job, nbf5));
    if (mixed_general_needed(job->nbf, nbf5)) return jkh_mo_mixed_general(job, st, C, H, nbf5, J, K, Hcore);
    donof_ctx* ctx = job->ctx;
    const int nbf = job->nbf, naux = job->naux, grid = mixed_grid(job);
    MixedScratch S;
    DONOF_CHECK(mixed_prepare(job, st, C, nbf5, &S, grid));
    // mode 2 also emits d and the K partials; b_pq itself goes to a scratch
    DONOF_CHECK(job->tmp.ensure(ctx, sizeof(float) * (size_t)nbf5 * nbf5 * naux));
    DONOF_CHECK(launch_mixed(job, st, nbf5, nbf5, nbf5, 2, S, nullptr, job->tmp.as<float>(), grid));
    const long long n55 = (long long)nbf5 * nbf5;
    mx::reduce_f32_to_f64_t<<<(int)((n55 + 255) / 256), 256, 0, st>>>(S.kpart, n55, grid, nbf5, K); count_launch();
    // J = D D^T with D[p, l] = d_p^l (FP64 GEMM on the FP32 diagonals)
    const long long nd = (long long)nbf5 * naux;
    mx::f32_to_f64<<<4 * ctx->sm_count, 256, 0, st>>>(S.d, nd, S.dd); count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    DONOF_CHECK(gemm_f64_auto(ctx, st, false, false, nbf5, nbf5, naux, S.dd, nbf5, S.dd, nbf5, J, nbf5, 1.0, 0.0,
                              &job->part));
    DONOF_CHECK(job->small.ensure(ctx, sizeof(double) * (size_t)nbf * nbf5 * 2));
    double* HC = job->small.as<double>();
    DONOF_CHECK(gemm_f64_auto(ctx, st, false, true, nbf, nbf5, nbf, H, nbf, C, nbf, HC, nbf, 1.0, 0.0, nullptr));
    DONOF_CHECK(hcore_f64(job, st, C, HC, nbf5, Hcore));
    return DONOF_OK;
}

}  // namespace donof
