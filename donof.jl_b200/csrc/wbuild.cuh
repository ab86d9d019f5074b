// The W operand of the restructured Lagrangian (lagrange.cu header):
//   W_l[q, b] = delta_qb (n'_b d_b^l + t_b^l) - ck12[b, q] b_pq^l[b, q]
// with d_b^l = b_pq^l[b, b], t_b^l = sum_q cj12[b, q] d_q^l and n'_b = n_b for
// b < nbeta or b >= nalpha (0 when nbeta = 0), stored as W[q + nbf5 l + Kt b]
// (Kt = nbf5 naux).  The per-element and per-tile bodies are shared by the
// single-job kernels (lagrange.cu) and the grouped ones (batch.cu).
#pragma once

namespace donof {
namespace wbuild {

// n'_b d_b^l + t_b^l for element i = b + nbf5 l.
__device__ __forceinline__ double diag_value(const double* __restrict__ bpq, const double* __restrict__ n,
                                             const double* __restrict__ cj12, int nbf5, int nalpha, int nbeta,
                                             long long i) {
    const long long n55 = (long long)nbf5 * nbf5;
    const int b = (int)(i % nbf5);
    const long long l = i / nbf5;
    const double* B = bpq + n55 * l;
    double s = 0.0;
    for (int q = 0; q < nbf5; ++q) s += cj12[b + (long long)nbf5 * q] * B[(long long)q * (nbf5 + 1)];
    const bool dj = (nbeta > 0) && (b < nbeta || b >= nalpha);
    return (dj ? n[b] * B[(long long)b * (nbf5 + 1)] : 0.0) + s;
}

// Tile t of the (b, q, l) tile list, 32 x 32 (b, q) per tile and nt = ceil(nbf5 / 32)
// tiles per side; 256 threads (tx = threadIdx.x % 32, ty = threadIdx.x / 32),
// transposed through shared memory so that b_pq^l and ck12 are read along b and
// W is written along q.  Starts with a block barrier (the previous tile's reads
// of tb are done).
__device__ __forceinline__ void tile(const double* __restrict__ bpq, const double* __restrict__ ck12,
                                     const double* __restrict__ tv, int nbf5, int naux, double* __restrict__ W,
                                     long long t, double (*tb)[33]) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const long long n55 = (long long)nbf5 * nbf5, Kt = (long long)nbf5 * naux;
    const int nt = (nbf5 + 31) / 32;
    const int b0 = (int)(t % nt) * 32, q0 = (int)((t / nt) % nt) * 32;
    const long long l = t / ((long long)nt * nt);
    const double* B = bpq + n55 * l;
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int b = b0 + tx, q = q0 + r;
        double v = 0.0;
        if (b < nbf5 && q < nbf5) {
            const long long e = b + (long long)nbf5 * q;
            v = -ck12[e] * B[e];
            if (q == b) v += tv[b + (long long)nbf5 * l];
        }
        tb[r][tx] = v;  // [q - q0][b - b0]
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int q = q0 + tx, b = b0 + r;
        if (b < nbf5 && q < nbf5) W[q + (long long)nbf5 * l + Kt * b] = tb[tx][r];
    }
}

}  // namespace wbuild
}  // namespace donof
