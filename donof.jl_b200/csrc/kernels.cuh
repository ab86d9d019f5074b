// Internal (non-exported) entry points shared between the translation units.
#pragma once

#include <atomic>

#include <cuda.h>

#include "common.cuh"
#include "gemm_f64.cuh"

namespace donof {

// Tile shapes of the FP64 GEMM.  SmallW8 (64 x 64 over 8 warps of 32 x 16):
// more warps per SM for short-K products.
enum class GemmTile { Large /*128x64*/, Small /*64x64*/, Tiny /*32x32*/, SmallW8 /*64x64, 8 warps*/ };

// C = alpha*op(A)op(B) + beta*C on stream st (see gemm_f64.cuh for addressing).
int gemm_f64(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, GemmF64Args p,
             GemmTile tile);
// Same; persistent: one wave of CTAs walks the tiles (gemm_f64_persistent_kernel),
// which writes the same result.
int gemm_f64_run(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, GemmF64Args p,
                 GemmTile tile, bool persistent);

// out[i] = sum_s part[i + s*stride] (+ beta*out[i]), i < count
int splitk_reduce(donof_ctx* ctx, cudaStream_t st, const double* part, long long stride,
                  int splits, long long count, double* out, double beta);

// gemm_f64 with the tile shape chosen by the autotuner (gemm_f64.cu): the first
// call of a shape outside stream capture times the candidates and caches the
// fastest; heuristic is used while capturing and for calls with beta != 0,
// split-K or device-side gates.
int gemm_f64_tuned(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, const GemmF64Args& p,
                   GemmTile heuristic);

// Grouped persistent GEMM (gemm_f64.cuh, gemm_f64_grouped_kernel): ngroups
// GEMMs of one operand layout in one launch.  groups and start live in device
// memory: group g owns tiles [start[g], start[g+1]) of the flat work list
// (start[ngroups] == total_tiles, each group's count from gemm_f64_tiles with
// the same tile shape).  vec: every group passes gemm_f64_vec_ok.
int gemm_f64_grouped(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, bool vec, GemmTile tile,
                     const GemmF64Args* groups, const int* start, int ngroups, int total_tiles, int max_ctas);
int gemm_f64_tiles(const GemmF64Args& p, GemmTile tile);
bool gemm_f64_vec_ok(bool a_kmajor, bool b_kmajor, const GemmF64Args& p);

// Tile shape (and split count, when can_split) that puts >= one CTA per SM.
GemmTile pick_tile(donof_ctx* ctx, int M, int N, int K, bool can_split, int* splits_out);

// Convenience: plain column-major GEMM with a split-K heuristic that fills the
// SMs; partial results go to the job/context scratch `part`.
int gemm_f64_auto(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N,
                  int K, const double* A, long long lda, const double* B, long long ldb,
                  double* C, long long ldc, double alpha, double beta, DevBuf* part);

// Like gemm_f64_auto with alpha = 1, beta = 0, but the split-K partial sums are
// left in `part` for the caller to reduce: *out = partials (ld M, stride M*N),
// *nparts = their count (1 when the product was not split).
int gemm_f64_partials(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K,
                      const double* A, long long lda, const double* B, long long ldb, DevBuf* part,
                      const double** out, int* nparts);

// The split of gemm_f64_partials for this shape (the autotuner's choice, timed
// now on these operands if the process has none yet): *splits partial products
// of *kchunk K-elements each.  A caller that splits the same way sums in the
// same order.
int gemm_f64_partials_splits(donof_ctx* ctx, cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K,
                             const double* A, long long lda, const double* B, long long ldb, DevBuf* part,
                             int* splits, int* kchunk);

// Fused FP64 tail of the Lagrangian (tail.cu): Y = sum of nparts partials
// (FP32 or FP64, part[g * pstride + m + nbf * b]), HC = H C5, H_mat = C^T HC,
// elag = [n o H_mat + C^T Y | 0] and E_elec (when E != nullptr).
int elag_tail_f64(donof_job* job, cudaStream_t st, const double* C, const double* H, const double* n, int nbf5,
                  const void* part, bool part_f32, int nparts, long long pstride, double* Hmat, double* elag,
                  double* E);

// Eigenvalues w and eigenvectors V (columns) of Symmetric(G) on the device by
// the parallel cyclic Jacobi method (eigh.cu); A: n x n scratch, scratch:
// eigh_scratch_bytes(n).  Synchronises the stream.
size_t eigh_scratch_bytes(int n);
int eigh_jacobi(donof_ctx* ctx, cudaStream_t st, const double* G, int n, double* A, double* V, double* w,
                void* scratch);

// b = I G^{-1/2} on the device from host G (naux x naux) and I (nbf x nbf x naux)
// (iaux.cu); part is scratch for the products.
int iaux_f64(donof_ctx* ctx, cudaStream_t st, const double* G_host, const double* I_host, int nbf, int naux,
             double* b, DevBuf* part);

// FP64-accurate T1 on the tensor cores from int8 digit slices (ozaki.cu):
// ozaki_build makes the slices of the job's b (once), t1_ozaki computes
// tmp[m + nbf*q + nbf*nbf5*l] = (B_l C5)[m, q]; transforms_f64 uses it whenever
// the job holds the slices.
bool ozaki_shape_ok(int nbf);
size_t ozaki_bytes(int nbf, int naux);
int ozaki_build(donof_job* job);
void ozaki_free(donof_job* job);
int t1_ozaki(donof_job* job, cudaStream_t st, const double* C, int nbf5, double* tmp);

// Tensor maps with 128-byte swizzle and zero fill (mixed.cu)
int make_tmap_bf16(donof_ctx* ctx, CUtensorMap* map, const void* base, int rank, const cuuint64_t* dims,
                   const cuuint64_t* strides_bytes, const cuuint32_t* box);
int make_tmap_u8(donof_ctx* ctx, CUtensorMap* map, const void* base, int rank, const cuuint64_t* dims,
                 const cuuint64_t* strides_bytes, const cuuint32_t* box);

// FP64 pipelines (lagrange.cu)
int transforms_f64(donof_job* job, cudaStream_t st, const double* C, int nbf5);
int lagrange2_f64(donof_job* job, cudaStream_t st, const double* C, const double* n,
                  const double* H, const double* cj12, const double* ck12, int nbf5, int nalpha,
                  int nbeta, double* elag, double* Hmat, double* E);
int jkh_mo_f64(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5,
               double* J, double* K, double* Hcore);

// Aux-index slices (lagrange.cu): Y of the job's slice of b (nbf x nbf5, FP64),
// and the Lagrangian from the Y summed over every slice.
int lagrange2_partial_f64(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* cj12,
                          const double* ck12, int nbf5, int nalpha, int nbeta, double* Y);
int lagrange2_finish_f64(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* H,
                         int nbf5, const double* Y, double* elag, double* Hmat, double* E);

// H_core from HC = H C5 (lagrange.cu).
int hcore_f64(donof_job* job, cudaStream_t st, const double* C, const double* HC, int nbf5, double* Hcore);

// Mixed-precision pipelines (mixed.cu)
int transforms_mixed(donof_job* job, cudaStream_t st, const double* C, int nbf5);
int lagrange2_mixed(donof_job* job, cudaStream_t st, const double* C, const double* n,
                    const double* H, const double* cj12, const double* ck12, int nbf5,
                    int nalpha, int nbeta, double* elag, double* Hmat, double* E);
int jkh_mo_mixed(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5,
                 double* J, double* K, double* Hcore);

// Grouped form of the fused mixed kernel (mixed.cu) for a batch: each job's
// Y partials (FP32, one nbf x nbf5 block per CTA of its range) from its bf16
// split of b and its Cs / FP32 coefficients; jobs must fit the fused kernel.
struct MixedGroupJob {
    donof_job* job;
    int nbf5, nalpha, nbeta, ctas;
    void* cs;                        // bf16 Cs (mixed_ldk(nbf) x 128)
    const float *n32, *cj32, *ck32;  // prep_coef outputs
    float* ypart;                    // ctas x nbf x nbf5
};
struct MixedSplitJob {               // device table entry of split_c_grouped
    const double* C;
    void* cs;
    int nbf, nbf5, ldk, pad;
};
bool mixed_fused_fits(int nbf, int nbf5);
int mixed_ldk(int nbf);
int launch_mixed_grouped(donof_ctx* ctx, cudaStream_t st, const MixedGroupJob* jobs, int njobs);
int split_c_grouped(donof_ctx* ctx, cudaStream_t st, const MixedSplitJob* d_jobs, int njobs, int max_ldk);
int prep_coef(donof_ctx* ctx, cudaStream_t st, const double* n, const double* cj12, const double* ck12, int nbf5,
              float* n32, float* cj32, float* ck32);

// General-shape mixed pipeline (mixed_general.cu), used when the fused kernel's
// shape limits (nbf <= 256, nbf5 <= 64) do not hold.
bool mixed_general_needed(int nbf, int nbf5);
int transforms_mixed_general(donof_job* job, cudaStream_t st, const double* C, int nbf5);
int lagrange2_mixed_general(donof_job* job, cudaStream_t st, const double* C, const double* n, const double* H,
                            const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta, double* elag,
                            double* Hmat, double* E);
int jkh_mo_mixed_general(donof_job* job, cudaStream_t st, const double* C, const double* H, int nbf5, double* J,
                         double* K, double* Hcore);
int mixed_t1_general(donof_job* job, cudaStream_t st, const double* C, int nbf5, float* tmp_out);

// Rotation C_new = C exp(Y(y)) (rotate.cu)
int rotate_f64(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
               const double* C, double* Cnew);
// Same, every launch gated by *done (skipped when nonzero; done may be null).
int rotate_f64_gated(donof_ctx* ctx, cudaStream_t st, const double* y, int nbf, int nbf5,
                     const double* C, double* Cnew, const int* done, DevBuf* part);
size_t rotate_scratch_bytes(int nbf);

// Grouped cooperative kernels for a batch of jobs (batch.cu): one launch runs
// the rotation (or the Lagrangian tail) of every job, job j on the CTAs
// [cta0, cta0 + ctas) with its own barrier state in a GROUP_STATE_BYTES slot of
// `states` (zeroed by the launcher).  Ranges are disjoint except that jobs with
// ctas == 1 may share a CTA; grid <= sm_count (co-resident).  A job whose
// *skip is nonzero is left out.
constexpr int GROUP_STATE_BYTES = 64;
struct RotJob {
    const double* y;
    const double* C;
    double* Cnew;
    double* work;  // rotate_work_doubles(nbf)
    void* state;
    const int* skip;
    int nbf, nbf5, cta0, ctas;
};
size_t rotate_work_doubles(int nbf);
int rotate_grouped(donof_ctx* ctx, cudaStream_t st, const RotJob* jobs, int njobs, void* states, int grid);
struct TailJob {
    const double *C, *H, *n;
    const void* part;  // Y partials: part[g * pstride + m + nbf * b], g < nparts
    long long pstride;
    double *Hmat, *elag, *E;
    double* work;  // 3 * nbf * nbf5 doubles
    void* state;
    const int* skip;
    int nbf, nbf5, part_f32, nparts, cta0, ctas;
};
int tail_grouped(donof_ctx* ctx, cudaStream_t st, const TailJob* jobs, int njobs, void* states, int grid);

// One job through DoNOF.energy's orbital / occupation alternation (energy.cu),
// driven step by step: setup; while !done(): begin() (the occupations of the
// current gamma to dev_n/dev_cj/dev_ck), the orbital optimisation of dev_C at
// them, after_orbopt(E, iterations); then finish().  donof_energy runs it with
// the single-job optimiser, donof_batch_energy with the grouped one.
class EnergyJob {
public:
    EnergyJob();
    ~EnergyJob();
    EnergyJob(const EnergyJob&) = delete;
    EnergyJob& operator=(const EnergyJob&) = delete;
    int setup(donof_job* job, donof_energy_params* prm, const double* H, const double* C, const double* gamma,
              double* history);
    int begin();
    // after the orbital optimisation: occ_fetch (device), occ_solve (host only,
    // safe to run for several jobs on several threads), end_iteration (device)
    int after_orbopt(double E_orb, int nit_orb);
    int occ_fetch();
    int occ_solve();
    int end_iteration(double E_orb, int nit_orb);
    int finish(double* C_out, double* gamma_out, double* n_out, double* elag_out, donof_energy_result* res);
    bool done() const;
    const double* dev_n() const;
    const double* dev_cj() const;
    const double* dev_ck() const;
    const double* dev_H() const;
    double* dev_C() const;

private:
    struct Impl;
    Impl* p;
};

// donof_energy with a cancellation flag, read before every outer iteration
// (cancel may be null): a set flag ends the loop with DONOF_ERR_STATE and the
// error text "cancelled" (energy.cu).
int energy_run(donof_job* job, donof_energy_params* prm, const double* H, double* C_inout, double* gamma_inout,
               double* n_out, double* elag_out, double* history, donof_energy_result* res,
               const std::atomic<int>* cancel);

// Orbital-gradient helpers (optim.cu): g = pack(4 elag - 4 elag^T); when
// maxabs != nullptr also atomically max-reduces |g| into it (must be zeroed).
int pack_grad(donof_ctx* ctx, cudaStream_t st, const double* elag, int nbf, int nbf5, double* g,
              unsigned long long* maxabs_bits);
inline long long nvar_of(int nbf, int nbf5) {
    return (long long)nbf5 * nbf - (long long)nbf5 * (nbf5 + 1) / 2;
}

}  // namespace donof
