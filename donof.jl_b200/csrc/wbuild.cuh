// The W operand of the restructured Lagrangian (lagrange.cu header):
//   W_l[q, b] = delta_qb (n'_b d_b^l + t_b^l) - ck12[b, q] b_pq^l[b, q]
// with d_b^l = b_pq^l[b, b], t_b^l = sum_q cj12[b, q] d_q^l and n'_b = n_b for
// b < nbeta or b >= nalpha (0 when nbeta = 0), stored as W[q + nbf5 l + Kt b]
// (Kt = nbf5 naux).  The per-element and per-tile bodies are shared by the
// single-job kernels (lagrange.cu) and the grouped ones (batch.cu).
#pragma once

namespace donof {
namespace wbuild {

// The arithmetic of W with explicit rounding (no multiply-add contraction left
// to the compiler's choice), so that every kernel that builds W -- single job,
// grouped, fused into T2 or not -- writes the same bits.
// t_b^l accumulation: s + cj12[b, q] d_q^l, one rounding
__device__ __forceinline__ double tv_step(double s, double cj, double d) { return __fma_rn(cj, d, s); }
// n'_b d_b^l + t_b^l
__device__ __forceinline__ double tv_value(bool dj, double nb, double db, double s) {
    return __dadd_rn(dj ? __dmul_rn(nb, db) : 0.0, s);
}
// -ck12[b, q] b_pq^l[b, q]
__device__ __forceinline__ double w_value(double ck, double v) { return __dmul_rn(-ck, v); }
// the diagonal element adds n'_b d_b^l + t_b^l
__device__ __forceinline__ double w_diag(double w, double tv) { return __dadd_rn(w, tv); }

// n'_b d_b^l + t_b^l for element i = b + nbf5 l.
__device__ __forceinline__ double diag_value(const double* __restrict__ bpq, const double* __restrict__ n,
                                             const double* __restrict__ cj12, int nbf5, int nalpha, int nbeta,
                                             long long i) {
    const long long n55 = (long long)nbf5 * nbf5;
    const int b = (int)(i % nbf5);
    const long long l = i / nbf5;
    const double* B = bpq + n55 * l;
    double s = 0.0;
    for (int q = 0; q < nbf5; ++q) s = tv_step(s, cj12[b + (long long)nbf5 * q], B[(long long)q * (nbf5 + 1)]);
    const bool dj = (nbeta > 0) && (b < nbeta || b >= nalpha);
    return tv_value(dj, n[b], B[(long long)b * (nbf5 + 1)], s);
}

// The diagonal terms for a group of aux indices at a time: their diagonals
// d^l staged in shared memory once per block (DIAG_SM doubles), then one
// thread per (b, l) sums over q in the order of diag_value (same result).
constexpr int DIAG_SM = 2048;

// aux indices per group for nbf5 (about one (b, l) per thread of a 256-thread
// block); 0 when nbf5 is too large to stage (diag_value per element instead)
__host__ __device__ __forceinline__ int diag_group(int nbf5) {
    if (nbf5 > DIAG_SM) return 0;
    int g = 256 / nbf5;
    if (g < 1) g = 1;
    if (g * nbf5 > DIAG_SM) g = DIAG_SM / nbf5;
    return g;
}

// Work units for nbf5, naux: groups of diag_group(nbf5) aux indices, or
// 1024-element chunks of the (b, l) list when nbf5 cannot be staged.
__host__ __device__ __forceinline__ long long diag_units(int nbf5, int naux) {
    const int g = diag_group(nbf5);
    return g > 0 ? (naux + g - 1) / g : ((long long)nbf5 * naux + 1023) / 1024;
}

// Unit u of diag_units; sd: DIAG_SM doubles of shared memory.  Starts with a
// block barrier (the previous unit's reads of sd are done).
__device__ __forceinline__ void diag_unit(const double* __restrict__ bpq, const double* __restrict__ n,
                                          const double* __restrict__ cj12, int nbf5, int naux, int nalpha, int nbeta,
                                          double* __restrict__ tv, long long u, double* sd) {
    const int g = diag_group(nbf5);
    if (g == 0) {
        const long long k0 = u * 1024, k1 = min((long long)nbf5 * naux, k0 + 1024);
        for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x)
            tv[k] = diag_value(bpq, n, cj12, nbf5, nalpha, nbeta, k);
        return;
    }
    const long long n55 = (long long)nbf5 * nbf5, l0 = u * g;
    const int items = g * nbf5;
    __syncthreads();
    for (int i = threadIdx.x; i < items; i += blockDim.x) {
        const int li = i / nbf5, q = i - li * nbf5;
        const long long l = l0 + li;
        sd[i] = (l < naux) ? bpq[n55 * l + (long long)q * (nbf5 + 1)] : 0.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < items; i += blockDim.x) {
        const int li = i / nbf5, b = i - li * nbf5;
        const long long l = l0 + li;
        if (l >= naux) continue;
        const double* d = sd + li * nbf5;
        double s = 0.0;
        for (int q = 0; q < nbf5; ++q) s = tv_step(s, cj12[b + (long long)nbf5 * q], d[q]);
        const bool dj = (nbeta > 0) && (b < nbeta || b >= nalpha);
        tv[b + (long long)nbf5 * l] = tv_value(dj, n[b], d[b], s);
    }
}

// Aux indices per tile: a tile covers 32 x 32 (b, q) for LT consecutive l.
constexpr int LT = 4;

// Number of tiles for nbf5, naux.
__host__ __device__ __forceinline__ long long tiles(int nbf5, int naux) {
    const long long nt = (nbf5 + 31) / 32;
    return nt * nt * ((naux + LT - 1) / LT);
}

// Tile t of the (b, q, l-group) tile list: 32 x 32 (b, q) for the aux indices
// l0 .. l0 + LT - 1; 256 threads (tx = threadIdx.x % 32, ty = threadIdx.x / 32).
// Every load of the tile (ck12 once, b_pq^l for each l) is issued before the
// first barrier; the transpose through shared memory makes b_pq^l and ck12 read
// along b and W written along q.  Starts with a block barrier (the previous
// tile's reads of tb are done).
__device__ __forceinline__ void tile(const double* __restrict__ bpq, const double* __restrict__ ck12,
                                     const double* __restrict__ tv, int nbf5, int naux, double* __restrict__ W,
                                     long long t, double (*tb)[32][33]) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const long long n55 = (long long)nbf5 * nbf5, Kt = (long long)nbf5 * naux;
    const int nt = (nbf5 + 31) / 32;
    const int b0 = (int)(t % nt) * 32, q0 = (int)((t / nt) % nt) * 32;
    const long long l0 = (t / ((long long)nt * nt)) * LT;
    const int b = b0 + tx;
    double ck[4], v[LT][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int q = q0 + ty + 8 * r;
        ck[r] = (b < nbf5 && q < nbf5) ? ck12[b + (long long)nbf5 * q] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < LT; ++k) {
        const long long l = l0 + k;
        const double* B = bpq + n55 * l;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = q0 + ty + 8 * r;
            v[k][r] = (l < naux && b < nbf5 && q < nbf5) ? B[b + (long long)nbf5 * q] : 0.0;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < LT; ++k) {
        const long long l = l0 + k;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = q0 + ty + 8 * r;
            double w = w_value(ck[r], v[k][r]);
            if (q == b && l < naux && b < nbf5) w = w_diag(w, tv[b + (long long)nbf5 * l]);
            tb[k][ty + 8 * r][tx] = w;  // [l - l0][q - q0][b - b0]
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < LT; ++k) {
        const long long l = l0 + k;
        if (l >= naux) break;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = q0 + tx, bb = b0 + ty + 8 * r;
            if (bb < nbf5 && q < nbf5) W[q + (long long)nbf5 * l + Kt * bb] = tb[k][tx][ty + 8 * r];
        }
    }
}

}  // namespace wbuild
}  // namespace donof
