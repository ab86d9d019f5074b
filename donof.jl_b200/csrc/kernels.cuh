// Internal (non-exported) entry points shared between the translation units.
#pragma once

#include "common.cuh"
#include "gemm_f64.cuh"

namespace donof {

enum class GemmTile { Large /*128x64*/, Small /*64x64*/, Tiny /*32x32*/ };

// C = alpha*op(A)op(B) + beta*C on stream st (see gemm_f64.cuh for addressing).
int gemm_f64(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, GemmF64Args p,
             GemmTile tile);

// out[i] = sum_s part[i + s*stride] (+ beta*out[i]), i < count
int splitk_reduce(donof_ctx* ctx, cudaStream_t st, const double* part, long long stride,
                  int splits, long long count, double* out, double beta);

// Tile shape (and split count, when can_split) that puts >= one CTA per SM.
GemmTile pick_tile(donof_ctx* ctx, int M, int N, int K, bool can_split, int* splits_out);

// Convenience: plain column-major GEMM with a split-K heuristic that fills the
// SMs; partial results go to the job/context scratch `part`.
int gemm_f64_auto(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N,
                  int K, const double* A, long long lda, const double* B, long long ldb,
                  double* C, long long ldc, double alpha, double beta, DevBuf* part);

// FP64 pipelines (lagrange.cu)
int transforms_f64(donof_job* job, cudaStream_t st, const double* C, int nbf5);
int lagrange2_f64(donof_job* job, cudaStream_t st, const double* C, const double* n,
                  const double* H, const double* cj12, const double* ck12, int nbf5, int nalpha,
                  int nbeta, double* elag, double* Hmat, double* E);
int jkh_mo_f64(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5,
               double* J, double* K, double* Hcore);

// Shared tails of the Lagrangian / JKH_MO (lagrange.cu): elag = n o H_mat + C^T Y
// (columns >= nbf5 zero) and E_elec; H_core from HC = H C5.
int elag_finish_f64(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* Hmat,
                    const double* Y, int nbf5, double* elag, double* E);
int hcore_f64(donof_job* job, cudaStream_t st, const double* C, const double* HC, int nbf5, double* Hcore);

// Mixed-precision pipelines (mixed.cu)
int transforms_mixed(donof_job* job, cudaStream_t st, const double* C, int nbf5);
int lagrange2_mixed(donof_job* job, cudaStream_t st, const double* C, const double* n,
                    const double* H, const double* cj12, const double* ck12, int nbf5,
                    int nalpha, int nbeta, double* elag, double* Hmat, double* E);
int jkh_mo_mixed(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5,
                 double* J, double* K, double* Hcore);

// Rotation C_new = C exp(Y(y)) (rotate.cu)
int rotate_f64(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
               const double* C, double* Cnew);
// Same, every launch gated by *done (skipped when nonzero; done may be null).
int rotate_f64_gated(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
                     const double* C, double* Cnew, const int* done, DevBuf* part);
size_t rotate_scratch_bytes(int nbf);

// Orbital-gradient helpers (optim.cu): g = pack(4 elag - 4 elag^T); when
// maxabs != nullptr also atomically max-reduces |g| into it (must be zeroed).
int pack_grad(donof_ctx* ctx, cudaStream_t st, const double* elag, int nbf, int nbf5, double* g,
              unsigned long long* maxabs_bits);
inline long long nvar_of(int nbf, int nbf5) {
    return (long long)nbf5 * nbf - (long long)nbf5 * (nbf5 + 1) / 2;
}

}  // namespace donof
