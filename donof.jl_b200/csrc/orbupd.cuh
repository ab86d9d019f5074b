// One step of the AMSGrad-style update shared by orbopt_adam / orbopt_adabelief
// / orbopt_yogi / orbopt_demon (src/minimization.jl:307-316, 406-411, 503-508,
// 598-603): the coefficients of iteration i and the per-element update, used
// by the single-job graph loop (optim.cu) and the grouped one (batch.cu).
#pragma once

#include <math.h>

#include "../../include/donof_b200.h"

namespace donof {
namespace orbupd {

struct Coef {
    int method;
    double beta1, beta2, bc1, bc2, alpha;  // bc = 1 - beta^i
};

__host__ __device__ __forceinline__ Coef coef(int method, int i, int maxloop, double alpha) {
    Coef c;
    c.method = method;
    c.beta1 = (method == DONOF_ORB_DEMON) ? 0.6 : 0.5;
    c.beta2 = (method == DONOF_ORB_DEMON) ? 0.999 : 0.9;
    if (method == DONOF_ORB_DEMON) {
        const double binit = c.beta1;
        const double rate = (i - 1.0) / (maxloop - 1.0);
        c.beta1 = binit * (1.0 - rate) / ((1.0 - binit) + binit * (1.0 - rate));
    }
    c.bc1 = 1.0 - pow(c.beta1, (double)i);
    c.bc2 = 1.0 - pow(c.beta2, (double)i);
    c.alpha = alpha;
    return c;
}

__host__ __device__ __forceinline__ void step(const Coef& c, long long k, const double* __restrict__ g, double* __restrict__ m,
                                     double* __restrict__ v, double* __restrict__ vmax, double* __restrict__ y) {
    const double gk = g[k];
    const double mk = c.beta1 * m[k] + (1.0 - c.beta1) * gk;
    double vk;
    if (c.method == DONOF_ORB_ADABELIEF) {
        const double dd = gk - mk;
        vk = c.beta2 * v[k] + (1.0 - c.beta2) * (dd * dd);
    } else if (c.method == DONOF_ORB_YOGI) {
        const double g2 = gk * gk;
        const double dv = v[k] - g2;
        const double sg = (dv > 0.0) ? 1.0 : ((dv < 0.0) ? -1.0 : 0.0);
        vk = v[k] - (1.0 - c.beta2) * sg * g2;
    } else {
        vk = c.beta2 * v[k] + (1.0 - c.beta2) * (gk * gk);
    }
    const double vm = fmax(vmax[k], vk / c.bc2);
    m[k] = mk;
    v[k] = vk;
    vmax[k] = vm;
    y[k] = -c.alpha * (mk / c.bc1) / sqrt(vm + 1e-16);
}

}  // namespace orbupd
}  // namespace donof
