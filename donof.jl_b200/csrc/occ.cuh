// Internal C++ interface of the native occupation layer (occupation.cu), for
// host drivers inside the library (the energy loop of energy.cu).
#pragma once

#include <vector>

#include "common.cuh"
#include "occ_math.cuh"

namespace donof {
namespace occ {

// Sizes and index tables of the GNOF occupation layer (names of src/param.jl).
struct Occ {
    int N, no1, ndoc, nsoc, nbeta, nalpha, ncwo, nv, ista, high_spin, method;
    double h_cut;
    std::vector<int> S, P, G;  // strong (ndoc); weak P[g*ncwo + w]; gamma index G[g*ncwo + w]
    std::vector<int> KG;       // the ncwo gamma entries of pair g: KG[g*ncwo + c] (dn is zero elsewhere)
    std::vector<int> grp;      // pair of each orbital (-1 outside the pairs)
};

// false on inconsistent sizes or switches
bool setup(const donof_occ_params* q, Occ& o);
// the tables of o as a view (valid while o lives)
OccView view(const Occ& o);
// n (N) and dn (N x nv, dn[i * nv + k]) of ocupacion_softmax / _trigonometric
void occupations(const Occ& o, const double* gamma, double* n, double* dn);
// GNOF cj12, ck12 (N x N, column-major) of CJCKD8
void coupling(const Occ& o, const double* n, double* cj, double* ck);
// occupation energy (calce) and, with grad != nullptr, its gamma-gradient (calcoccg)
double energy_grad(const Occ& o, const double* gamma, const double* J, const double* K, const double* Hc,
                   double* grad);
// occoptr's minimisation on the device (occ_device.cu): one CTA runs the same
// CG over J, K, Hc and gamma in device memory (gamma in/out); result[0] = E,
// [1] = iterations, [2] = converged, [3, 3 + nv) = the gradient at gamma.
bool occ_cg_fits(const Occ& o);
int occ_cg_launch(donof_ctx* ctx, cudaStream_t st, const Occ& o, const double* J, const double* K, const double* Hc,
                  double* gamma, double g_abstol, int max_iter, double* result);
// occoptr's minimisation over gamma (Hager-Zhang CG, strong-Wolfe line search)
int cg(const Occ& o, const double* J_MO, const double* K_MO, const double* H_core, double* gamma,
       double g_abstol, int max_iter, double* E, int* nit, int* converged);

}  // namespace occ
}  // namespace donof
