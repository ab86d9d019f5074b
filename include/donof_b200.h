/*
 * libdonofb200 -- C ABI of the B200 (sm_100a) RI hot path for GNOF natural
 * orbital functional energies.
 *
 * The entry points replace the methods that DoNOF.jl's GPU package extension
 * (ext/DoNOFGPUExt.jl) adds for CuArray arguments; a Julia extension binds
 * them with ccall (one call per reference method, same argument meaning).
 *
 * Conventions
 *   - Every matrix is FP64, column-major (Julia layout), 0-based indices in the
 *     descriptions below:  C[m + nbf*p], b[m + nbf*n + nbf*nbf*l],
 *     H[m + nbf*n], n[p], cj12/ck12[p + nbf5*q], elag[a + nbf*b] (nbf x nbf),
 *     H_mat[i + nbf*j] (nbf x nbf5), J_MO/K_MO[p + nbf5*q], H_core[p].
 *   - Entry points without a suffix take HOST pointers, copy inputs to the
 *     device, run on the context stream and return when the outputs are back
 *     in host memory (the reference's per-call CuArray(...) / Array(...)).
 *   - Entry points with the _dev suffix take DEVICE pointers, only enqueue
 *     work on the context stream and return immediately.
 *   - Every call returns a status code (DONOF_OK = 0); donof_last_error()
 *     gives the text of the last failure on that context.
 *   - One context per host thread; a context owns one CUDA stream.
 */
#ifndef DONOF_B200_H
#define DONOF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* status codes */
#define DONOF_OK 0
#define DONOF_ERR_ARG 1       /* invalid argument (size, null pointer, mode) */
#define DONOF_ERR_CUDA 2      /* CUDA runtime error */
#define DONOF_ERR_OOM 3       /* device allocation failed */
#define DONOF_ERR_STATE 4     /* object in the wrong state for this call */
#define DONOF_ERR_NOT_CONVERGED 5
#define DONOF_ERR_TIMEOUT 6   /* a kernel gave up on a bounded wait; its outputs are not valid */

/* precision of the b tensor held by a job and of the bulk contractions */
#define DONOF_PREC_FP64 0   /* all contractions in FP64 (plain form) */
#define DONOF_PREC_MIXED 1  /* tensor-core 3 x bf16 split bulk contractions, FP32 accumulation */

/* orbital optimisers (src/minimization.jl:242-630) */
#define DONOF_ORB_ADAM 0
#define DONOF_ORB_ADABELIEF 1
#define DONOF_ORB_YOGI 2
#define DONOF_ORB_DEMON 3

typedef struct donof_ctx donof_ctx;
typedef struct donof_job donof_job;

/* --- context ------------------------------------------------------------ */
int donof_create(int device, donof_ctx** ctx);
int donof_destroy(donof_ctx* ctx);
/* use an existing cudaStream_t (passed as void*) instead of the own stream */
int donof_set_stream(donof_ctx* ctx, void* stream);
void* donof_get_stream(donof_ctx* ctx);
/* Most CTAs the context's persistent and cooperative kernels may use (0, the
 * default: one per SM).  A server running several jobs at once gives each
 * context a share of the SMs so that their kernels run side by side.         */
int donof_set_cta_limit(donof_ctx* ctx, int max_ctas);
int donof_synchronize(donof_ctx* ctx);
const char* donof_last_error(const donof_ctx* ctx);
const char* donof_status_string(int status);
int donof_version(void);

/* --- the b tensor ---------------------------------------------------------
 * donof_b_upload replaces eris_to_gpu (ext/DoNOFGPUExt.jl:36-50, called at
 * src/integrals.jl:59-62): copies the host RI tensor b[m,n,l] (nbf x nbf x
 * naux, FP64) to the device once per job.  precision = DONOF_PREC_MIXED also
 * keeps a bf16 hi/lo split copy for the mixed-precision form (the FP64 copy
 * stays, for refinement steps).
 * donof_b_attach wraps an existing device buffer without copying (the job
 * does not own it and it must outlive the job).
 * Both scan b once on the device and reject a tensor holding a NaN or an
 * infinity with DONOF_ERR_ARG (no job is created).                          */
int donof_b_upload(donof_ctx* ctx, const double* b_host, int nbf, int naux, int precision,
                   donof_job** job);
/* donof_iaux replaces Iaux / Iaux_gpu (src/integrals.jl:68-91,
 * ext/DoNOFGPUExt.jl:9-33) followed by eris_to_gpu: from the two-centre
 * integrals G (naux x naux, host, the upper triangle is read as
 * Symmetric(G)) and the three-centre integrals I (nbf x nbf x naux, host) it
 * builds b = I G^{-1/2} on the device (negative eigenvalues of G give zero
 * inverse square roots) and returns a job that owns it, as donof_b_upload. */
int donof_iaux(donof_ctx* ctx, const double* G, const double* I3c, int nbf, int naux, int precision,
               donof_job** job);
int donof_b_attach(donof_ctx* ctx, const double* b_dev, int nbf, int naux, int precision,
                   donof_job** job);
int donof_job_free(donof_job* job);
/* Precision used by the calls without an explicit one (DONOF_PREC_MIXED needs
 * a job created with DONOF_PREC_MIXED; switching to FP64 is always allowed,
 * e.g. for the closing refinement iterations of a mixed-precision run).      */
int donof_job_set_precision(donof_job* job, int precision);
/* device bytes held by the job (b copies + scratch) */
size_t donof_job_device_bytes(const donof_job* job);

/* --- compute_Lagrange2, RI method -------------------------------------------
 * Replaces compute_Lagrange2(C,n,H,b::CuArray{T,3},cj12,ck12,nalpha,nbeta)
 * (ext/DoNOFGPUExt.jl:150-245); CPU definition src/utils.jl:1-59.
 * Outputs elag (nbf x nbf; columns >= nbf5 are zero) and H_mat = C^T H C5
 * (nbf x nbf5).  The job's precision selects the plain FP64 or the mixed form.
 * E_elec, if not NULL, receives computeE_elec(H_mat, n, elag)
 * (src/utils.jl:216-227).                                                  */
int donof_lagrange2(donof_job* job, const double* C, const double* n, const double* H,
                    const double* cj12, const double* ck12, int nbf5, int nalpha, int nbeta,
                    double* elag, double* H_mat, double* E_elec);
int donof_lagrange2_dev(donof_job* job, const double* C, const double* n, const double* H,
                        const double* cj12, const double* ck12, int nbf5, int nalpha,
                        int nbeta, double* elag, double* H_mat, double* E_elec);
/* Same as donof_lagrange2_dev with an explicit precision (overrides the job's;
 * DONOF_PREC_MIXED needs a job uploaded with DONOF_PREC_MIXED).            */
int donof_lagrange2_prec_dev(donof_job* job, int precision, const double* C, const double* n,
                             const double* H, const double* cj12, const double* ck12,
                             int nbf5, int nalpha, int nbeta, double* elag, double* H_mat,
                             double* E_elec);

/* Allocation-free compute_Lagrange2 (plain FP64 form, device pointers).
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * hosts whose device memory belongs to another runtime's pool, services that
 * must not grow their device footprint while running, or code that may not
 * block on the synchronising allocator.  Every intermediate lives in one
 * 32 MiB device array inside the library, held by every GPU that loads it
 * until the process exits; sizes whose intermediates do not fit
 * ((nbf*nbf5 + 2*nbf5*nbf5) * naux doubles plus small terms) are rejected
 * with DONOF_ERR_ARG.  The first call on a device looks that array up (make
 * it before any stream capture); all calls share it, so calls that overlap on
 * the GPU race.  The job must not allocate either: attach b with
 * donof_b_attach and DONOF_PREC_FP64.                                        */
int donof_lagrange2_noalloc_dev(donof_job* job, const double* C, const double* n, const double* H,
                                const double* cj12, const double* ck12, int nbf5, int nalpha,
                                int nbeta, double* elag, double* H_mat, double* E_elec);

/* --- the aux index split across GPUs -----------------------------------------
 * compute_Lagrange2 (src/utils.jl:1-59) with b[:, :, l] split into contiguous
 * slices of the aux index, one per GPU (each job holds its slice: nbf x nbf x
 * naux_r).  Every elag term of the reference is a sum over l; in the
 * restructured form elag[:, :nbf5] = n o H_mat + C^T Y with
 * Y = sum_l tmp_l W_l, so each GPU computes the Y of its slice
 * (donof_lagrange2_partial_dev, Y nbf x nbf5 FP64, device), the ranks sum
 * their Y with one all-reduce (nbf * nbf5 doubles, e.g. NCCL), and
 * donof_lagrange2_finish_dev gives elag, H_mat and E_elec from the summed Y.
 * J_MO and K_MO of JKH_MO are sums over l the same way (all-reduce the
 * outputs of donof_jkh_mo_dev of each slice; H_core is the same on every
 * rank).  Plain FP64 form.                                                 */
int donof_lagrange2_partial_dev(donof_job* job, const double* C, const double* n, const double* cj12,
                                const double* ck12, int nbf5, int nalpha, int nbeta, double* Y);
int donof_lagrange2_finish_dev(donof_job* job, const double* C, const double* n, const double* H, int nbf5,
                               const double* Y, double* elag, double* H_mat, double* E_elec);

/* --- JKH_MO, RI method ----------------------------------------------------
 * Replaces computeJKH_MO / JKH_MO(C,H,b::CuArray{T,3},nbf,nbf5,nbfaux)
 * (ext/DoNOFGPUExt.jl:52-94); CPU definition src/integrals.jl:131-172.
 * J_MO[p,q] = sum_l b_pp^l b_qq^l, K_MO[p,q] = sum_l (b_pq^l)^2,
 * H_core[p] = C_p^T H C_p, with b_pq^l = sum_mn C[m,p] b[m,n,l] C[n,q].     */
int donof_jkh_mo(donof_job* job, const double* C, const double* H, int nbf5, double* J_MO,
                 double* K_MO, double* H_core);
int donof_jkh_mo_dev(donof_job* job, const double* C, const double* H, int nbf5, double* J_MO,
                     double* K_MO, double* H_core);
int donof_jkh_mo_prec_dev(donof_job* job, int precision, const double* C, const double* H,
                          int nbf5, double* J_MO, double* K_MO, double* H_core);

/* --- three-index transform ---------------------------------------------------
 * b_pq^l = sum_mn C[m,p] b[m,n,l] C[n,q] for p, q < nbf5: the b_mnl -> b_pnl ->
 * b_pql transform of JKH_MO / compute_eris_full (src/integrals.jl:159-160,
 * 287-288; ext/DoNOFGPUExt.jl:71-72).  b_pq (device, may be NULL) receives
 * b_pq[p + nbf5*q + nbf5*nbf5*l].                                            */
int donof_transform_dev(donof_job* job, int precision, const double* C, int nbf5, double* b_pq);

/* --- FP64 form on the tensor cores ----------------------------------------
 * enable != 0 makes the int8 digit slices of the job's b (7 slices of 7 bits
 * per row, scaled by a power of two; 7/8 of b's FP64 size) and from then on
 * runs the FP64 form's first contraction tmp_l = b_l C5 (src/utils.jl:19,
 * src/integrals.jl:150) as exact int8 x int8 -> int32 tensor-core products
 * recombined in FP64 (Ozaki scheme): within ~1e-13 of the largest |tmp| of
 * an FP64 GEMM, inside the form's 1e-10 parity.  enable = 0 frees the slices
 * (the DMMA GEMM runs again).  Needs nbf <= 16384.  donof_job_fp64_tc tells
 * whether the slices are present.                                            */
int donof_job_set_fp64_tc(donof_job* job, int enable);
int donof_job_fp64_tc(const donof_job* job);
/* FP64 form's first contraction alone: tmp[m + nbf*q + nbf*nbf5*l] =
 * sum_n b[m,n,l] C[n,q] (device, FP64), by whichever engine the job uses.   */
int donof_t1_dev(donof_job* job, const double* C, int nbf5, double* tmp);

/* --- rotate_orbital ------------------------------------------------------
 * Replaces rotate_orbital(y,C,p) (ext/DoNOFGPUExt.jl:355-382, which runs in
 * FP32); CPU definition src/utils.jl:499-521, followed here in FP64:
 * y (nvar = nbf5*nbf - nbf5*(nbf5+1)/2) is unpacked row-wise over i < nbf5,
 * j > i into the antisymmetric Y, and C_new = C exp(Y).                      */
int donof_rotate(donof_ctx* ctx, const double* y, int nbf, int nbf5, const double* C,
                 double* C_new);
int donof_rotate_dev(donof_ctx* ctx, const double* y, int nbf, int nbf5, const double* C,
                     double* C_new);

/* --- calcorbg --------------------------------------------------------------
 * Orbital gradient at y (src/pnof.jl:1389-1407): C' = rotate_orbital(y, C),
 * elag = compute_Lagrange2(C', ...), grad = 4 elag - 4 elag^T packed over
 * i < nbf5, j > i.  y may be NULL for y = 0 (the call at src/energy.jl:188). */
int donof_orbgrad(donof_job* job, const double* y, const double* C, const double* n,
                  const double* H, const double* cj12, const double* ck12, int nbf5, int nalpha,
                  int nbeta, double* grad);
/* The host side of one iteration of the reference's optimiser loop
 * (src/minimization.jl:390-412), for a caller that drives the loop itself
 * through donof_rotate + donof_lagrange2: g = 4 elag - 4 elag^T packed over
 * i < nbf5, j > i (nvar values), then the update of iteration it (1-based) of
 * method (DONOF_ORB_*; Demon's beta1 decays over maxloop) with step alpha into
 * the caller's state m, v, vmax and the rotation y (nvar doubles each, zero
 * before iteration 1); *gmax = max|g| (may be NULL).  Host arrays, no device
 * work.                                                                     */
int donof_orb_step_host(int method, int it, int maxloop, double alpha, const double* elag, int nbf, int nbf5,
                        double* g, double* m, double* v, double* vmax, double* y, double* gmax);

/* --- orbital optimiser -----------------------------------------------------
 * One call of orbopt_adam / orbopt_adabelief / orbopt_yogi / orbopt_demon
 * (src/minimization.jl:242-630) with the whole loop resident on the device:
 * gradient packing, the AMSGrad-style update, rotation, Lagrangian, energy
 * and best-(E, C) tracking.  C is read from and written back to C_inout.
 * *alpha and *maxloop are read and updated like p.alpha / p.maxloop (step
 * back-off when no iteration improved E).                                  */
int donof_orbopt(donof_job* job, int method, const double* n, const double* cj12,
                 const double* ck12, const double* H, int nbf5, int nalpha, int nbeta,
                 double* alpha, int* maxloop, double threshgorb, double* C_inout, double* E,
                 int* nit, int* success);
/* Same with n, cj12, ck12, H and C_inout in device memory (C_inout is updated
 * in place on the context stream; the call returns after the loop ends).     */
int donof_orbopt_dev(donof_job* job, int method, const double* n, const double* cj12,
                     const double* ck12, const double* H, int nbf5, int nalpha, int nbeta,
                     double* alpha, int* maxloop, double threshgorb, double* C_inout, double* E,
                     int* nit, int* success);

/* --- grouped orbital optimiser over a batch of jobs --------------------------
 * The orbital optimiser above (orbopt_adam / _adabelief / _yogi / _demon,
 * src/minimization.jl:242-630, plain FP64 form) run for several molecules at
 * once: each gradient step of all jobs is one grouped launch per stage (the
 * three-index transforms and the Lagrangian GEMM as grouped persistent tensor-
 * core kernels over a work list spanning every job, the rotation and the
 * Lagrangian tail as grouped cooperative kernels), and the whole loop is one
 * captured CUDA graph that repeats the step until every job has met its own
 * stopping rule.  DoNOF.jl optimises one molecule per call; each job here
 * gives bit-for-bit what donof_orbopt_dev gives it alone (every product sums
 * in the same order; the Lagrangian GEMM takes the autotuner's split for the
 * job's shape, as the single-job path does).
 * donof_batch_create fixes the jobs (each with its FP64 RI tensor uploaded by
 * donof_b_upload / donof_b_attach on the same device) and their sizes, and
 * allocates the batch's device scratch (donof_batch_device_bytes).  The first
 * call times the tile shapes of the grouped GEMMs on the batch's operands (the
 * batch's autotuner) and captures the loop graph; make it outside any stream
 * capture.  Calls of one batch must not overlap.                             */
typedef struct donof_batch donof_batch;
typedef struct {
    donof_job* job;   /* RI tensor b of this instance (nbf, naux from the job) */
    int nbf5, nalpha, nbeta;
} donof_batch_shape;
/* Per-job inputs and outputs, all arrays in DEVICE memory (layouts as above). */
typedef struct {
    const double* n;      /* nbf5 occupations */
    const double* cj12;   /* nbf5 x nbf5 */
    const double* ck12;   /* nbf5 x nbf5 */
    const double* H;      /* nbf x nbf core Hamiltonian */
    double* C;            /* nbf x nbf: start orbitals in, optimised orbitals out (orbopt) */
    double alpha;         /* in/out, as *alpha of donof_orbopt */
    int maxloop;          /* in/out, as *maxloop of donof_orbopt */
    double threshgorb;    /* in */
    double E;             /* out: E_elec */
    int nit, success;     /* out */
} donof_batch_item;
int donof_batch_create(donof_ctx* ctx, int count, const donof_batch_shape* shapes, donof_batch** batch);
/* Form of the batch's Lagrangian (donof_batch_lagrange2 / _orbopt / _energy):
 * DONOF_PREC_FP64 (default) or DONOF_PREC_MIXED -- the fused tcgen05 kernel
 * of the mixed form for every job in one grouped launch (each job on its own
 * CTA range, b read from its bf16 split: the jobs must be uploaded with
 * DONOF_PREC_MIXED and have nbf <= 256, nbf5 <= 64), then the grouped FP64
 * tail.  The rotation, optimiser and occupation steps stay FP64.  Mixed
 * results agree with the FP64 ones to the mixed form's tolerance; they are not
 * bit-for-bit a job's mixed result alone (the Y partials are summed over the
 * job's CTA range, which depends on the batch).  donof_batch_serve runs FP64
 * batches only.                                                               */
int donof_batch_set_precision(donof_batch* batch, int precision);
int donof_batch_destroy(donof_batch* batch);
size_t donof_batch_device_bytes(const donof_batch* batch);
/* Optimiser loop of every job (items[j] for shapes[j]); returns when all ended.
 * An item with maxloop = 0 leaves its job out of the call (untouched).       */
int donof_batch_orbopt(donof_batch* batch, int method, donof_batch_item* items);
/* compute_Lagrange2 (src/utils.jl:1-59) of every job at items[j].C in one
 * grouped evaluation: elag[j] (nbf x nbf) and H_mat[j] (nbf x nbf5) device
 * arrays (or NULL), E[j] = E_elec on the host (E may be NULL).               */
int donof_batch_lagrange2(donof_batch* batch, const donof_batch_item* items, double* const* elag,
                          double* const* H_mat, double* E);


/* --- occupation layer and occupation optimiser (host, FP64) ------------------
 * Native host code, no GPU: DoNOF.jl runs this part on the host too.
 * Sizes and switches of the GNOF occupation layer (names of src/param.jl):
 * nbf5, no1, nbeta, nalpha, ncwo, ista (0-5), HighSpin, occ_method
 * (0 = Softmax, 1 = Trigonometric) and h_cut.  nv = ncwo * (nbeta - no1).   */
typedef struct {
    int nbf5, no1, nbeta, nalpha, ncwo, ista, high_spin, occ_method;
    double h_cut;
} donof_occ_params;
/* Occupations n (nbf5) of ocupacion_softmax / _trigonometric (src/pnof.jl:
 * 1024-1163) at gamma (nv), and, if dn_dgamma != NULL, dn/dgamma (nbf5 x nv,
 * column-major).                                                            */
int donof_occupations(const donof_occ_params* p, const double* gamma, double* n, double* dn_dgamma);
/* GNOF coupling coefficients cj12, ck12 (nbf5 x nbf5, column-major, zero
 * diagonal) of PNOFi_selector / CJCKD8 (src/pnof.jl:1-53, 488-601) at n.     */
int donof_coupling(const donof_occ_params* p, const double* n, double* cj12, double* ck12);
/* Occupation energy at gamma from cached J_MO, K_MO (nbf5 x nbf5, column-
 * major) and H_core (nbf5): calce / calcocce (src/pnof.jl:1273-1322) with the
 * occupations of ocupacion_softmax / _trigonometric (:1047-1163) and the GNOF
 * couplings of CJCKD8 (:488-601); with grad != NULL also its gamma-gradient
 * (nv), calcoccg (:1324-1377, der_CJCKD8 :603-793).                          */
int donof_occ_energy(const donof_occ_params* p, const double* gamma, const double* J_MO,
                     const double* K_MO, const double* H_core, double* E, double* grad);
/* Replaces the minimisation of occoptr (src/minimization.jl:100-139, Optim.jl
 * ConjugateGradient with g_abstol): Hager-Zhang conjugate gradient with a
 * strong-Wolfe line search over gamma (in/out, nv), stopped when
 * max|grad| <= g_abstol or after max_iter iterations.  Returns the energy,
 * the iteration count and whether the gradient test was met.               */
int donof_occ_cg(const donof_occ_params* p, const double* J_MO, const double* K_MO,
                 const double* H_core, double* gamma, double g_abstol, int max_iter, double* E,
                 int* nit, int* converged);

/* occoptr's minimisation (as donof_occ_cg) on the GPU: one CTA runs the same
 * conjugate gradient and line search over J_MO, K_MO (nbf5 x nbf5), H_core
 * (nbf5) and gamma (nv, in/out), all in DEVICE memory, and writes result (device,
 * 3 + nv doubles): the energy, the iteration count, 1 if the gradient test was
 * met, then the gradient at the returned gamma.  Enqueued on the context
 * stream; allocates nothing.  Sums run in another order than on the host, so
 * the two solvers agree to rounding.                                          */
int donof_occ_cg_dev(donof_ctx* ctx, const donof_occ_params* p, const double* J_MO, const double* K_MO,
                     const double* H_core, double* gamma, double g_abstol, int max_iter, double* result);

/* --- the energy loop ------------------------------------------------------------
 * Switches and thresholds of DoNOF.energy's alternation (names of
 * src/param.jl): the occupation layer, the orbital optimiser (DONOF_ORB_*),
 * maxit outer iterations, maxloop and alpha (read and updated like p.maxloop and
 * p.alpha), threshgorb / threshgocc (convergence) and threshen (g_abstol of
 * occoptr); order_subspaces = 1 applies the final sort of src/guess.jl:58-106
 * (ipnof > 4); freeze_occ = 1 keeps gamma fixed; stop_rel_de > 0 ends the
 * loop once an outer iteration changes E by at most stop_rel_de |E| (the
 * mixed-precision phase stops there, where its energies' rounding would
 * steer the optimiser, and FP64 iterations take over); occ_device = 1 runs
 * occoptr's conjugate gradient on the GPU (one CTA, J_MO / K_MO stay on the
 * device) instead of the host.                                              */
typedef struct {
    donof_occ_params occ;
    int orb_method;
    int maxit;
    int maxloop;
    double alpha;
    double threshgorb, threshgocc, threshen;
    int order_subspaces;
    int freeze_occ;
    double stop_rel_de;  /* > 0: also stop (not converged) once |E - E_prev| <= stop_rel_de |E| */
    int occ_device;      /* 1: occoptr's minimisation on the GPU (as donof_occ_cg_dev), 0: on the host */
} donof_energy_params;
typedef struct {
    double E_elec;                /* E of the last orbital optimisation */
    int iterations, converged, tot_it_orb, tot_it_occ;
    double max_grad_orb, norm_grad_occ;
} donof_energy_result;
/* The orbital / occupation alternation of DoNOF.energy (src/energy.jl:140-224)
 * in one call, in the job's precision: orbopt on the device, occoptr (J_MO,
 * K_MO, H_core on the device, conjugate gradient over gamma on the host),
 * order_occupations_softmax, and the convergence test on max|g_orb| and
 * |g_occ|.  Host arrays: H and C_inout (nbf x nbf), gamma_inout (nv); n_out
 * (nbf5), elag_out (nbf x nbf) and history (6 per iteration: E, E_diff,
 * max|g_orb|, |g_occ|, orbital and occupation iterations) may be NULL.     */
int donof_energy(donof_job* job, donof_energy_params* params, const double* H, double* C_inout,
                 double* gamma_inout, double* n_out, double* elag_out, double* history,
                 donof_energy_result* result);
/* donof_energy (above) for every job of a batch (donof_batch_create): per outer iteration one
 * grouped orbital optimisation of the jobs still running, then each job's
 * occoptr, ordering and convergence test.  params[j], H[j], C_inout[j],
 * gamma_inout[j] and n_out[j] (or n_out NULL) as for donof_energy, host
 * arrays; every job uses the same orb_method and the FP64 form.  Each job
 * gives bit-for-bit what donof_energy gives it alone.                       */
int donof_batch_energy(donof_batch* batch, donof_energy_params* params, const double* const* H,
                       double* const* C_inout, double* const* gamma_inout, double* const* n_out,
                       donof_energy_result* results);

/* --- continuous batching at the step level ---------------------------------
 * donof_batch_serve runs donof_batch_energy's alternation over a stream of
 * requests: the batch's jobs are slots; a request whose job has a slot's shape
 * (nbf, naux of its RI tensor; nbf5, nalpha, nbeta of its parameters) takes
 * that slot when it frees, so that every outer iteration advances all running
 * requests as grouped launches (one per stage of a gradient step) and a request
 * that converges returns at once while the others go on.  Requests are pushed
 * into a queue (any host thread, also while donof_batch_serve runs) and taken in
 * arrival order, the oldest request that fits a free slot first;
 * donof_batch_serve returns once the queue is closed and every request that a
 * slot can take has finished (a request that fits no slot finishes with
 * DONOF_ERR_ARG).  Each request gives bit-for-bit what donof_energy gives it
 * alone.  Every request of one queue uses the same orb_method.  The request's
 * host arrays must stay valid until it is done (donof_batch_queue_poll).     */
typedef struct donof_batch_queue donof_batch_queue;
typedef struct {
    donof_job* job;                 /* FP64 RI tensor of this request (same device as the batch) */
    donof_energy_params params;     /* copied at push; alpha, maxloop as for donof_energy */
    const double* H;                /* host nbf x nbf */
    double* C_inout;                /* host nbf x nbf */
    double* gamma_inout;            /* host nv */
    double* n_out;                  /* host nbf5, or NULL */
} donof_batch_request;
int donof_batch_queue_create(donof_batch_queue** queue);
int donof_batch_queue_push(donof_batch_queue* queue, const donof_batch_request* request,
                           unsigned long long* ticket);
int donof_batch_queue_close(donof_batch_queue* queue);
/* done = 1 once the request finished; then *status is its outcome and *result
 * its energy result (wait != 0: block until done).                           */
int donof_batch_queue_poll(donof_batch_queue* queue, unsigned long long ticket, int wait, int* done,
                           int* status, donof_energy_result* result);
int donof_batch_queue_destroy(donof_batch_queue* queue);
int donof_batch_serve(donof_batch* batch, donof_batch_queue* queue);

/* --- serving ------------------------------------------------------------------
 * Continuous batching of energy jobs on one GPU behind a thread-safe queue:
 * jobs are admitted while their device footprint fits the budget (0: 85 % of
 * the free memory) and one of max_inflight workers is free (first fit in
 * arrival order, the head passed over at most 4 times); each worker runs its
 * job on its own context and stream, so the jobs in flight overlap.
 * precision: DONOF_PREC_FP64, DONOF_PREC_MIXED (the mixed form, then closing
 * FP64 iterations to the thresholds) or DONOF_PREC_AUTO (mixed where
 * nbf * nbf5 * naux >= DONOF_AUTO_MIXED_MIN_WORK, FP64 elsewhere).  A request's
 * host arrays (H, b, C, gamma; gamma NULL: the reference's initial guess) and
 * the output arrays (C_out nbf x nbf, n_out nbf5 or NULL) must stay valid until
 * the job is collected by donof_server_poll / donof_server_wait.             */
#define DONOF_PREC_AUTO 2
#define DONOF_AUTO_MIXED_MIN_WORK 2.0e7
typedef struct donof_server donof_server;
typedef struct {
    const double* H;
    const double* b;
    const double* C;
    const double* gamma;
    int nbf, naux;
    donof_energy_params params;
    int precision;
    double E_nuc;
} donof_request;
typedef struct {
    int status;                   /* DONOF_OK or the job's error (DONOF_ERR_STATE: cancelled) */
    double E_elec, E_tot;
    int iterations, converged;
    int precision;                /* the form that ran */
    double queue_s, latency_s;    /* submit -> start, submit -> done */
    char error[256];
} donof_result;
int donof_server_create(int device, size_t budget_bytes, int max_inflight, donof_server** server);
int donof_server_submit(donof_server* server, const donof_request* request, double* C_out, double* n_out,
                        unsigned long long* ticket);
/* done = 1 (and the result filled, the ticket released) once the job has ended */
int donof_server_poll(donof_server* server, unsigned long long ticket, donof_result* result, int* done);
int donof_server_wait(donof_server* server, unsigned long long ticket, donof_result* result);
/* Cancels a job: one still queued ends at once, one in flight at its next
 * outer iteration; either is then collected with status DONOF_ERR_STATE and
 * the error text "cancelled".  A job already done keeps its result.          */
int donof_server_cancel(donof_server* server, unsigned long long ticket);
/* Cancels the jobs not started, waits for those in flight and for callers
 * blocked in donof_server_wait (they return the job's result, or a cancelled
 * one), then frees the server and every job not collected.  No call on the
 * server may start once donof_server_destroy has begun.                      */
int donof_server_destroy(donof_server* server);

/* --- diagnostics -------------------------------------------------------------
 * Number of CUDA kernels this library has launched in the process so far.    */
unsigned long long donof_launch_count(void);
/* With profiling enabled, each call brackets its dominant kernel (the first
 * three-index transform of the FP64 form, the fused tensor-core kernel of the
 * mixed form) with CUDA events on the context stream; donof_profile_last_ms
 * waits for and returns the duration of the most recent one.                 */
int donof_profile_enable(donof_ctx* ctx, int enable);
int donof_profile_last_ms(donof_ctx* ctx, float* ms);
/* Number of GEMM shapes whose configuration the autotuner has chosen in this
 * process (each is timed once, at its first call outside stream capture).   */
int donof_autotune_entries(void);
/* Failure detection.  Every wait inside the library's kernels is bounded (an
 * mbarrier of the tensor-core pipelines, the grid barrier of a cooperative
 * kernel): a wait that runs out makes the kernel stop without touching its
 * outputs further and record the failure in its context's failure words
 * (page-locked host memory mapped into the device), with no fault and no hang.
 * The calls that synchronise (the host-buffer entry points, the optimiser and
 * energy loops, the batch calls) then return DONOF_ERR_TIMEOUT; the _dev entry
 * points only enqueue work, so their caller reads the words here.
 * donof_error_flags synchronises the context stream and returns the recorded
 * failures as a bit mask (1: mbarrier wait of a mixed-form kernel, 2: grid
 * barrier of a cooperative kernel, 4: a finiteness scan met NaN or infinity)
 * and clears them.  donof_job_error_flag does the same for the job's context
 * and reports 1 if any bit was set.                                           */
int donof_error_flags(donof_ctx* ctx, int* flags);
int donof_job_error_flag(donof_job* job, int* flag);
/* Cycle budget of every bounded wait in the context's kernels launched from now
 * on (0, the default: about one to two seconds of clock).  A tiny budget makes
 * the waits run out, so that a test can drive the failure path above; a
 * captured optimiser graph keeps the budget it was captured with.            */
int donof_set_wait_limit(donof_ctx* ctx, long long cycles);
/* First contraction of the mixed form alone, for checking it:
 * tmp[m + nbf*q + nbf*nbf5*l] = sum_n b[m,n,l] C[n,q] (FP32, device).        */
int donof_mixed_tmp_dev(donof_job* job, const double* C, int nbf5, float* tmp);

/* ---- Integral front end (replaces GaussianBasis.jl/libcint as called by
 * compute_integrals, src/integrals.jl:1-49: overlap, kinetic, nuclear,
 * ERI_2e2c, ERI_2e3c, ERI_2e4c).  McMurchie-Davidson over contracted shells
 * with l <= 5.  A basis is a list of shells: angular momentum l[s], centre
 * (bohr) centre[3s..3s+2], nprim[s] primitives whose exponents and contraction
 * coefficients follow in exps/coefs (as printed in a basis-set file; the
 * library normalises primitives like x^l and each contraction to unit
 * self-overlap).  spherical: real solid harmonics (p as x, y, z; l >= 2 as
 * m = -l..l), else Cartesian components (xx..x, xx..y, ..., zz..z).  Every
 * output is column-major and FP64.                                          */
typedef struct donof_basis donof_basis;
int donof_basis_create(int nshell, const int* l, const double* centre, const int* nprim, const double* exps,
                       const double* coefs, int spherical, donof_basis** basis);
int donof_basis_nbf(const donof_basis* basis);
int donof_basis_free(donof_basis* basis);
/* S, T and V (nbf x nbf; T or V may be null; V sums -Z_k/|r - R_k| over the
 * natom nuclei of charge Z[k] at xyz[3k..3k+2] bohr).  Replaces overlap,
 * kinetic, nuclear (src/integrals.jl:4-9).                                   */
int donof_int1e(const donof_basis* basis, int natom, const double* Z, const double* xyz, double* S, double* T,
                double* V);
/* G[P,Q] = (P|Q) over the auxiliary basis (naux x naux): ERI_2e2c
 * (src/integrals.jl:47).                                                     */
int donof_int2c2e(const donof_basis* aux, double* G);
/* I[m + nbf (n + nbf P)] = (mn|P) (nbf x nbf x naux): ERI_2e3c
 * (src/integrals.jl:49), host threads; donof_int3c2e_dev computes the same on
 * the context's device into device memory (orbital shells l <= 3, auxiliary
 * l <= 4).                                                                   */
int donof_int3c2e(const donof_basis* orb, const donof_basis* aux, double* I);
int donof_int3c2e_dev(donof_ctx* ctx, const donof_basis* orb, const donof_basis* aux, double* I_dev);
/* I[m + nbf (n + nbf (l + nbf s))] = (mn|ls) (nbf^4): ERI_2e4c
 * (src/integrals.jl:16), for small bases.                                    */
int donof_int4c2e(const donof_basis* basis, double* I);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* DONOF_B200_H */
