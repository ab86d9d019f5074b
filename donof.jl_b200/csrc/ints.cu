// Gaussian-basis integrals for the RI front end (src/integrals.jl:1-49, which
// the reference computes through GaussianBasis.jl / libcint): overlap,
// kinetic, nuclear attraction, two-centre (P|Q), three-centre (mn|P) and, for
// small bases, four-centre (mn|ls) electron-repulsion integrals over
// contracted Cartesian or real-spherical shells, by the McMurchie-Davidson
// scheme of ints.cuh.  The host path runs the shell pairs on host threads; the
// three-centre integrals, the front end's largest product (nbf^2 naux), also
// run as a B200 kernel (donof_int3c2e_dev) from the same __host__ __device__
// code.
//
// Conventions: primitives normalised like x^l (the libcint convention for
// Cartesian shells), contractions renormalised to unit self-overlap;
// Cartesian components ordered xx..x, xx..y, ..., zz..z; spherical shells
// p as (x, y, z) and l >= 2 as m = -l..l, real solid harmonics scaled to unit
// norm.  Matrices are column-major; I[m + nbf (n + nbf P)].
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "common.cuh"
#include "ints.cuh"

struct donof_basis {
    int nshell = 0, nbf = 0, spherical = 1, lmax = 0, maxprim = 0;
    std::vector<int> l, nprim, prim0, ao0;
    std::vector<double> ctr;     // 3 per shell (bohr)
    std::vector<double> ex, co;  // exponents; coefficients with primitive and contraction normalisation
    // device copy for the three-centre kernel (made on first use)
    void* dev = nullptr;
    int dev_device = -1;
};

namespace donof {
namespace {

double dfact(int n) {  // n!! for n >= -1
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

int cart_index(int l, int lx, int ly) {
    int k = 0;
    for (int a = l; a >= 0; --a)
        for (int b = l - a; b >= 0; --b) {
            if (a == lx && b == ly) return k;
            ++k;
        }
    return -1;
}

int nfunc(int l, bool spherical) { return spherical ? 2 * l + 1 : ints::ncart(l); }

// Cartesian -> real-spherical coefficients for every l <= LMAX: column s of
// table[l] (ncart(l) values) is the solid harmonic S_{l,m} (Schlegel and Frisch,
// Int. J. Quantum Chem. 54, 83 (1995): the sum over t, u, v of
// (-1)^{t+v-v_m} 4^{-t} C(l,t) C(l-t,|m|+t) C(t,u) C(|m|,2v)
// x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|}), scaled so that with Cartesian
// components normalised like x^l it has unit norm.
struct SphTable {
    std::vector<double> c[ints::LMAX + 1];
    SphTable() {
        for (int l = 0; l <= ints::LMAX; ++l) {
            const int nc = ints::ncart(l), ns = 2 * l + 1;
            c[l].assign((size_t)nc * ns, 0.0);
            for (int s = 0; s < ns; ++s) {
                int m;
                if (l == 1) m = (s == 0) ? 1 : (s == 1 ? -1 : 0);  // p as x, y, z
                else m = s - l;
                const int am = m < 0 ? -m : m, wm = m < 0 ? 1 : 0;
                double* col = c[l].data() + (size_t)s * nc;
                for (int t = 0; t <= (l - am) / 2; ++t)
                    for (int u = 0; u <= t; ++u)
                        for (int w = wm; w <= am; w += 2) {
                            const int px = 2 * t + am - 2 * u - w, py = 2 * u + w, pz = l - 2 * t - am;
                            if (px < 0 || pz < 0) continue;
                            const double sign = (((t + (w - wm) / 2) & 1) != 0) ? -1.0 : 1.0;
                            const double v = sign * pow(0.25, t) * binom(l, t) * binom(l - t, am + t) * binom(t, u) *
                                             binom(am, w);
                            col[cart_index(l, px, py)] += v;
                        }
                // norm with the component overlaps Omega(c1, c2) = prod_d (n_d - 1)!! / (2l - 1)!!
                double nrm = 0.0;
                for (int a = 0; a < nc; ++a)
                    for (int b = 0; b < nc; ++b) {
                        int ax, ay, az, bx, by, bz;
                        ints::cart_xyz(l, a, &ax, &ay, &az);
                        ints::cart_xyz(l, b, &bx, &by, &bz);
                        const int nx = ax + bx, ny = ay + by, nz = az + bz;
                        if ((nx | ny | nz) & 1) continue;
                        nrm += col[a] * col[b] * dfact(nx - 1) * dfact(ny - 1) * dfact(nz - 1) / dfact(2 * l - 1);
                    }
                const double f = 1.0 / sqrt(nrm);
                for (int a = 0; a < nc; ++a) col[a] *= f;
            }
        }
    }
};

const SphTable& sph_table() {
    static const SphTable t;
    return t;
}

// Apply the shells' Cartesian -> spherical maps along every index of a block
// stored with the first index slowest (dims ncart(l_k)); out gets dims nfunc.
void block_to_sph(int nidx, const int* ls, bool spherical, const double* in, double* out, std::vector<double>& tmp) {
    int dims[4];
    size_t total = 1;
    for (int k = 0; k < nidx; ++k) {
        dims[k] = ints::ncart(ls[k]);
        total *= dims[k];
    }
    if (!spherical) {
        memcpy(out, in, total * sizeof(double));
        return;
    }
    tmp.assign(in, in + total);
    std::vector<double> nxt;
    for (int k = 0; k < nidx; ++k) {
        const int nc = dims[k], ns = 2 * ls[k] + 1;
        size_t outer = 1, inner = 1;
        for (int q = 0; q < k; ++q) outer *= dims[q];
        for (int q = k + 1; q < nidx; ++q) inner *= dims[q];
        nxt.assign(outer * ns * inner, 0.0);
        const double* T = sph_table().c[ls[k]].data();
        for (size_t o = 0; o < outer; ++o)
            for (int s = 0; s < ns; ++s)
                for (int c = 0; c < nc; ++c) {
                    const double f = T[(size_t)s * nc + c];
                    if (f == 0.0) continue;
                    const double* src = tmp.data() + (o * nc + c) * inner;
                    double* dst = nxt.data() + (o * ns + s) * inner;
                    for (size_t i = 0; i < inner; ++i) dst[i] += f * src[i];
                }
        dims[k] = ns;
        tmp.swap(nxt);
    }
    memcpy(out, tmp.data(), tmp.size() * sizeof(double));
}

// Run body(w) for w = 0..count-1 on the host's threads.
template <class Body>
void parallel_for(long long count, Body body) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if ((long long)nt > count) nt = (unsigned)(count > 0 ? count : 1);
    std::atomic<long long> next{0};
    auto worker = [&]() {
        for (long long w; (w = next.fetch_add(1)) < count;) body(w);
    };
    std::vector<std::thread> th;
    for (unsigned i = 1; i < nt; ++i) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
}

// ---- the three-centre integrals on the device
constexpr int DEV_LORB = 3;  // orbital shells up to f
constexpr int DEV_LAUX = 4;  // auxiliary shells up to g
constexpr int SPH_DOUBLES = 1 + 9 + 30 + 70 + 135;  // ncart(l) (2l + 1), l <= 4

struct DevBasis {
    int nshell, nbf, spherical, pad;
    const int *l, *nprim, *prim0, *ao0;
    const int* order;  // shells sorted by (l, primitive count): neighbouring threads take alike shells
    const double *ctr, *ex, *co;
};

__constant__ double c_sph[SPH_DOUBLES];

__host__ __device__ inline int sph_off(int l) { return l == 0 ? 0 : (l == 1 ? 1 : (l == 2 ? 10 : (l == 3 ? 40 : 110))); }

// One thread per (orbital shell pair, auxiliary shell): the Cartesian block
// over all primitive triples, then the spherical (or Cartesian) values
// written to I[m + nbf (n + nbf P)] and I[n + nbf (m + nbf P)].  LO and LX
// bound the orbital and auxiliary l (they size the per-thread arrays).
template <int LO, int LX>
__global__ void __launch_bounds__(128) int3c2e_kernel(const DevBasis orb, const DevBasis aux, long long npair,
                                                      double* __restrict__ I) {
    constexpr int DEV_BLOCK = ints::ncart(LO) * ints::ncart(LO) * ints::ncart(LX);
    constexpr int DEV_SCRATCH = ints::coulomb_scratch(LO, LO, LX, 0);
    const long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (w >= npair * aux.nshell) return;
    const long long pw = w / aux.nshell;
    const int k = aux.order[w % aux.nshell];
    int i = (int)((sqrt(8.0 * (double)pw + 1.0) - 1.0) / 2.0);
    while ((long long)i * (i + 1) / 2 > pw) --i;
    while ((long long)(i + 1) * (i + 2) / 2 <= pw) ++i;
    const int j = (int)(pw - (long long)i * (i + 1) / 2);
    const int la = orb.l[i], lb = orb.l[j], lk = aux.l[k];
    const int na = ints::ncart(la), nb = ints::ncart(lb), nk = ints::ncart(lk);
    double blk[DEV_BLOCK];
    double scr[DEV_SCRATCH];
    for (int x = 0; x < na * nb * nk; ++x) blk[x] = 0.0;
    const double* A = orb.ctr + 3 * i;
    const double* B = orb.ctr + 3 * j;
    const double* C = aux.ctr + 3 * k;
    for (int pa = 0; pa < orb.nprim[i]; ++pa)
        for (int pb = 0; pb < orb.nprim[j]; ++pb)
            for (int pc = 0; pc < aux.nprim[k]; ++pc) {
                const int ka = orb.prim0[i] + pa, kb = orb.prim0[j] + pb, kc = aux.prim0[k] + pc;
                ints::coulomb_prim(la, lb, orb.ex[ka], orb.ex[kb], A, B, lk, 0, aux.ex[kc], 0.0, C, C,
                                   orb.co[ka] * orb.co[kb] * aux.co[kc], blk, scr);
            }
    const int fa = orb.spherical ? 2 * la + 1 : na, fb = orb.spherical ? 2 * lb + 1 : nb;
    const int fk = aux.spherical ? 2 * lk + 1 : nk;
    const long long nbf = orb.nbf;
    for (int x = 0; x < fa; ++x)
        for (int y = 0; y < fb; ++y)
            for (int s = 0; s < fk; ++s) {
                double v = 0.0;
                for (int ca = 0; ca < na; ++ca) {
                    const double ta = orb.spherical ? c_sph[sph_off(la) + x * na + ca] : (ca == x ? 1.0 : 0.0);
                    if (ta == 0.0) continue;
                    for (int cb = 0; cb < nb; ++cb) {
                        const double tb = orb.spherical ? c_sph[sph_off(lb) + y * nb + cb] : (cb == y ? 1.0 : 0.0);
                        if (tb == 0.0) continue;
                        for (int ck = 0; ck < nk; ++ck) {
                            const double tk = aux.spherical ? c_sph[sph_off(lk) + s * nk + ck] : (ck == s ? 1.0 : 0.0);
                            v += ta * tb * tk * blk[(ca * nb + cb) * nk + ck];
                        }
                    }
                }
                const long long m = orb.ao0[i] + x, n = orb.ao0[j] + y, P = aux.ao0[k] + s;
                I[m + nbf * (n + nbf * P)] = v;
                I[n + nbf * (m + nbf * P)] = v;
            }
}

// The basis' arrays in device memory (one allocation, made once per basis).
int upload_basis(donof_ctx* ctx, donof_basis* b, DevBasis* d) {
    const size_t ni = (size_t)b->nshell, np = b->ex.size();
    const size_t bytes = 5 * ni * sizeof(int) + (3 * ni + 2 * np) * sizeof(double) + 64;
    if (!b->dev || b->dev_device != ctx->device) {
        if (b->dev) cudaFree(b->dev);
        b->dev = nullptr;
        DONOF_CUDA(ctx, cudaMalloc(&b->dev, bytes));
        b->dev_device = ctx->device;
        std::vector<char> h(bytes, 0);
        char* q = h.data();
        auto put = [&](const void* src, size_t n) {
            memcpy(q, src, n);
            q += (n + 7) / 8 * 8;
        };
        put(b->ctr.data(), 3 * ni * sizeof(double));
        put(b->ex.data(), np * sizeof(double));
        put(b->co.data(), np * sizeof(double));
        put(b->l.data(), ni * sizeof(int));
        put(b->nprim.data(), ni * sizeof(int));
        put(b->prim0.data(), ni * sizeof(int));
        put(b->ao0.data(), ni * sizeof(int));
        std::vector<int> order(ni);
        for (size_t s = 0; s < ni; ++s) order[s] = (int)s;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return b->l[x] != b->l[y] ? b->l[x] < b->l[y] : b->nprim[x] < b->nprim[y];
        });
        put(order.data(), ni * sizeof(int));
        DONOF_CUDA(ctx, cudaMemcpy(b->dev, h.data(), bytes, cudaMemcpyHostToDevice));
    }
    char* q = static_cast<char*>(b->dev);
    auto take = [&](size_t n) {
        char* r = q;
        q += (n + 7) / 8 * 8;
        return r;
    };
    d->nshell = b->nshell;
    d->nbf = b->nbf;
    d->spherical = b->spherical;
    d->ctr = reinterpret_cast<const double*>(take(3 * ni * sizeof(double)));
    d->ex = reinterpret_cast<const double*>(take(np * sizeof(double)));
    d->co = reinterpret_cast<const double*>(take(np * sizeof(double)));
    d->l = reinterpret_cast<const int*>(take(ni * sizeof(int)));
    d->nprim = reinterpret_cast<const int*>(take(ni * sizeof(int)));
    d->prim0 = reinterpret_cast<const int*>(take(ni * sizeof(int)));
    d->ao0 = reinterpret_cast<const int*>(take(ni * sizeof(int)));
    d->order = reinterpret_cast<const int*>(take(ni * sizeof(int)));
    return DONOF_OK;
}

}  // namespace
}  // namespace donof

using donof::set_error;

extern "C" {

int donof_basis_create(int nshell, const int* l, const double* centre, const int* nprim, const double* exps,
                       const double* coefs, int spherical, donof_basis** out) {
    if (!out || nshell < 1 || !l || !centre || !nprim || !exps || !coefs) {
        set_error(nullptr, "donof_basis_create: null pointer or no shells");
        return DONOF_ERR_ARG;
    }
    *out = nullptr;
    auto* b = new donof_basis();
    b->nshell = nshell;
    b->spherical = spherical ? 1 : 0;
    int p0 = 0, ao = 0;
    for (int s = 0; s < nshell; ++s) {
        if (l[s] < 0 || l[s] > donof::ints::LMAX || nprim[s] < 1) {
            set_error(nullptr, "donof_basis_create: shell %d has l = %d (0..%d) and %d primitives", s, l[s],
                      donof::ints::LMAX, nprim[s]);
            delete b;
            return DONOF_ERR_ARG;
        }
        const int L = l[s];
        b->l.push_back(L);
        b->nprim.push_back(nprim[s]);
        b->prim0.push_back(p0);
        b->ao0.push_back(ao);
        for (int k = 0; k < 3; ++k) b->ctr.push_back(centre[3 * s + k]);
        // primitives normalised like x^l, then the contraction to unit self-overlap
        std::vector<double> c(nprim[s]);
        for (int k = 0; k < nprim[s]; ++k) {
            const double a = exps[p0 + k];
            if (!(a > 0.0)) {
                set_error(nullptr, "donof_basis_create: shell %d has a non-positive exponent", s);
                delete b;
                return DONOF_ERR_ARG;
            }
            c[k] = coefs[p0 + k] *
                   sqrt(pow(2.0 * a / M_PI, 1.5) * pow(4.0 * a, L) / donof::dfact(2 * L - 1));
        }
        double self = 0.0;
        for (int i = 0; i < nprim[s]; ++i)
            for (int j = 0; j < nprim[s]; ++j) {
                const double p = exps[p0 + i] + exps[p0 + j];
                self += c[i] * c[j] * pow(M_PI / p, 1.5) * donof::dfact(2 * L - 1) / pow(2.0 * p, L);
            }
        if (!(self > 0.0)) {
            set_error(nullptr, "donof_basis_create: shell %d has zero norm", s);
            delete b;
            return DONOF_ERR_ARG;
        }
        const double f = 1.0 / sqrt(self);
        for (int k = 0; k < nprim[s]; ++k) {
            b->ex.push_back(exps[p0 + k]);
            b->co.push_back(c[k] * f);
        }
        p0 += nprim[s];
        ao += donof::nfunc(L, b->spherical != 0);
        b->lmax = std::max(b->lmax, L);
        b->maxprim = std::max(b->maxprim, nprim[s]);
    }
    b->nbf = ao;
    *out = b;
    return DONOF_OK;
}

int donof_basis_nbf(const donof_basis* b) { return b ? b->nbf : -1; }

int donof_basis_free(donof_basis* b) {
    if (!b) return DONOF_ERR_ARG;
    if (b->dev) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (b->dev_device >= 0) cudaSetDevice(b->dev_device);
        cudaFree(b->dev);
        if (cur >= 0) cudaSetDevice(cur);
    }
    delete b;
    return DONOF_OK;
}

int donof_int1e(const donof_basis* b, int natom, const double* Z, const double* xyz, double* S, double* T,
                double* V) {
    using namespace donof;
    if (!b || !S || (V && natom > 0 && (!Z || !xyz)) || natom < 0) {
        set_error(nullptr, "donof_int1e: null pointer");
        return DONOF_ERR_ARG;
    }
    const int ns = b->nshell, nbf = b->nbf;
    const bool sph = b->spherical != 0;
    const long long npair = (long long)ns * (ns + 1) / 2;
    parallel_for(npair, [&](long long w) {
        int i = (int)((sqrt(8.0 * w + 1.0) - 1.0) / 2.0);
        while ((long long)i * (i + 1) / 2 > w) --i;
        while ((long long)(i + 1) * (i + 2) / 2 <= w) ++i;
        const int j = (int)(w - (long long)i * (i + 1) / 2);
        const int la = b->l[i], lb = b->l[j], na = ints::ncart(la), nb = ints::ncart(lb);
        std::vector<double> s(na * nb, 0.0), t(na * nb, 0.0), v(na * nb, 0.0);
        std::vector<double> scr(ints::one_e_scratch(la, lb));
        for (int pa = 0; pa < b->nprim[i]; ++pa)
            for (int pb = 0; pb < b->nprim[j]; ++pb) {
                const int ka = b->prim0[i] + pa, kb = b->prim0[j] + pb;
                ints::one_e_prim(la, lb, b->ex[ka], b->ex[kb], &b->ctr[3 * i], &b->ctr[3 * j], natom, Z, xyz,
                                 b->co[ka] * b->co[kb], s.data(), T ? t.data() : nullptr,
                                 V ? v.data() : nullptr, scr.data());
            }
        const int ls[2] = {la, lb};
        const int fa = nfunc(la, sph), fb = nfunc(lb, sph);
        std::vector<double> o(fa * fb), tmp;
        double* mats[3] = {S, T, V};
        std::vector<double>* blocks[3] = {&s, &t, &v};
        for (int k = 0; k < 3; ++k) {
            if (!mats[k]) continue;
            block_to_sph(2, ls, sph, blocks[k]->data(), o.data(), tmp);
            for (int x = 0; x < fa; ++x)
                for (int y = 0; y < fb; ++y) {
                    const long long r = b->ao0[i] + x, c = b->ao0[j] + y;
                    mats[k][r + (long long)nbf * c] = o[x * fb + y];
                    mats[k][c + (long long)nbf * r] = o[x * fb + y];
                }
        }
    });
    return DONOF_OK;
}

int donof_int2c2e(const donof_basis* aux, double* G) {
    using namespace donof;
    if (!aux || !G) {
        set_error(nullptr, "donof_int2c2e: null pointer");
        return DONOF_ERR_ARG;
    }
    const int ns = aux->nshell, n = aux->nbf;
    const bool sph = aux->spherical != 0;
    const long long npair = (long long)ns * (ns + 1) / 2;
    parallel_for(npair, [&](long long w) {
        int i = (int)((sqrt(8.0 * w + 1.0) - 1.0) / 2.0);
        while ((long long)i * (i + 1) / 2 > w) --i;
        while ((long long)(i + 1) * (i + 2) / 2 <= w) ++i;
        const int j = (int)(w - (long long)i * (i + 1) / 2);
        const int la = aux->l[i], lc = aux->l[j];
        std::vector<double> blk(ints::ncart(la) * ints::ncart(lc), 0.0);
        std::vector<double> scr(ints::coulomb_scratch(la, 0, lc, 0));
        const double* A = &aux->ctr[3 * i];
        const double* C = &aux->ctr[3 * j];
        for (int pa = 0; pa < aux->nprim[i]; ++pa)
            for (int pc = 0; pc < aux->nprim[j]; ++pc) {
                const int ka = aux->prim0[i] + pa, kc = aux->prim0[j] + pc;
                ints::coulomb_prim(la, 0, aux->ex[ka], 0.0, A, A, lc, 0, aux->ex[kc], 0.0, C, C,
                                   aux->co[ka] * aux->co[kc], blk.data(), scr.data());
            }
        const int ls[2] = {la, lc};
        const int fa = nfunc(la, sph), fc = nfunc(lc, sph);
        std::vector<double> o(fa * fc), tmp;
        block_to_sph(2, ls, sph, blk.data(), o.data(), tmp);
        for (int x = 0; x < fa; ++x)
            for (int y = 0; y < fc; ++y) {
                const long long r = aux->ao0[i] + x, c = aux->ao0[j] + y;
                G[r + (long long)n * c] = o[x * fc + y];
                G[c + (long long)n * r] = o[x * fc + y];
            }
    });
    return DONOF_OK;
}

int donof_int3c2e(const donof_basis* orb, const donof_basis* aux, double* I) {
    using namespace donof;
    if (!orb || !aux || !I) {
        set_error(nullptr, "donof_int3c2e: null pointer");
        return DONOF_ERR_ARG;
    }
    const int ns = orb->nshell, nx = aux->nshell, nbf = orb->nbf;
    const bool sph = orb->spherical != 0, sphx = aux->spherical != 0;
    const long long npair = (long long)ns * (ns + 1) / 2;
    parallel_for(npair * nx, [&](long long w) {
        const long long pw = w / nx;
        const int k = (int)(w % nx);
        int i = (int)((sqrt(8.0 * pw + 1.0) - 1.0) / 2.0);
        while ((long long)i * (i + 1) / 2 > pw) --i;
        while ((long long)(i + 1) * (i + 2) / 2 <= pw) ++i;
        const int j = (int)(pw - (long long)i * (i + 1) / 2);
        const int la = orb->l[i], lb = orb->l[j], lk = aux->l[k];
        std::vector<double> blk(ints::ncart(la) * ints::ncart(lb) * ints::ncart(lk), 0.0);
        std::vector<double> scr(ints::coulomb_scratch(la, lb, lk, 0));
        const double* A = &orb->ctr[3 * i];
        const double* B = &orb->ctr[3 * j];
        const double* C = &aux->ctr[3 * k];
        for (int pa = 0; pa < orb->nprim[i]; ++pa)
            for (int pb = 0; pb < orb->nprim[j]; ++pb)
                for (int pc = 0; pc < aux->nprim[k]; ++pc) {
                    const int ka = orb->prim0[i] + pa, kb = orb->prim0[j] + pb, kc = aux->prim0[k] + pc;
                    ints::coulomb_prim(la, lb, orb->ex[ka], orb->ex[kb], A, B, lk, 0, aux->ex[kc], 0.0, C, C,
                                       orb->co[ka] * orb->co[kb] * aux->co[kc], blk.data(), scr.data());
                }
        // the orbital indices in the orbital basis' form, the auxiliary one in its own
        std::vector<double> o, tmp;
        const int ls2[2] = {la, lb};
        const int fa = nfunc(la, sph), fb = nfunc(lb, sph), fk = nfunc(lk, sphx), nck = ints::ncart(lk);
        std::vector<double> ab((size_t)fa * fb * nck);
        {
            // orbital pair: transform the (a, b) block for each Cartesian aux component
            std::vector<double> one(ints::ncart(la) * ints::ncart(lb)), onesph(fa * fb);
            for (int c = 0; c < nck; ++c) {
                for (int x = 0; x < ints::ncart(la) * ints::ncart(lb); ++x) one[x] = blk[(size_t)x * nck + c];
                block_to_sph(2, ls2, sph, one.data(), onesph.data(), tmp);
                for (int x = 0; x < fa * fb; ++x) ab[(size_t)x * nck + c] = onesph[x];
            }
        }
        o.assign((size_t)fa * fb * fk, 0.0);
        if (sphx) {
            const double* T = sph_table().c[lk].data();
            for (int x = 0; x < fa * fb; ++x)
                for (int s = 0; s < fk; ++s) {
                    double v = 0.0;
                    for (int c = 0; c < nck; ++c) v += T[(size_t)s * nck + c] * ab[(size_t)x * nck + c];
                    o[(size_t)x * fk + s] = v;
                }
        } else {
            o = ab;
        }
        for (int x = 0; x < fa; ++x)
            for (int y = 0; y < fb; ++y)
                for (int s = 0; s < fk; ++s) {
                    const long long m = orb->ao0[i] + x, n = orb->ao0[j] + y, P = aux->ao0[k] + s;
                    const double v = o[((size_t)x * fb + y) * fk + s];
                    I[m + (long long)nbf * (n + (long long)nbf * P)] = v;
                    I[n + (long long)nbf * (m + (long long)nbf * P)] = v;
                }
    });
    return DONOF_OK;
}

int donof_int4c2e(const donof_basis* b, double* I) {
    using namespace donof;
    if (!b || !I) {
        set_error(nullptr, "donof_int4c2e: null pointer");
        return DONOF_ERR_ARG;
    }
    const int ns = b->nshell;
    const long long nbf = b->nbf;
    const bool sph = b->spherical != 0;
    const long long npair = (long long)ns * (ns + 1) / 2;
    auto unpair = [](long long w, int* i, int* j) {
        int a = (int)((sqrt(8.0 * w + 1.0) - 1.0) / 2.0);
        while ((long long)a * (a + 1) / 2 > w) --a;
        while ((long long)(a + 1) * (a + 2) / 2 <= w) ++a;
        *i = a;
        *j = (int)(w - (long long)a * (a + 1) / 2);
    };
    parallel_for(npair * npair, [&](long long w) {
        const long long p1 = w / npair, p2 = w % npair;
        if (p2 > p1) return;
        int i, j, k, l;
        unpair(p1, &i, &j);
        unpair(p2, &k, &l);
        const int li = b->l[i], lj = b->l[j], lk = b->l[k], ll = b->l[l];
        std::vector<double> blk((size_t)ints::ncart(li) * ints::ncart(lj) * ints::ncart(lk) * ints::ncart(ll), 0.0);
        std::vector<double> scr(ints::coulomb_scratch(li, lj, lk, ll));
        for (int pa = 0; pa < b->nprim[i]; ++pa)
            for (int pb = 0; pb < b->nprim[j]; ++pb)
                for (int pc = 0; pc < b->nprim[k]; ++pc)
                    for (int pd = 0; pd < b->nprim[l]; ++pd) {
                        const int ka = b->prim0[i] + pa, kb = b->prim0[j] + pb;
                        const int kc = b->prim0[k] + pc, kd = b->prim0[l] + pd;
                        ints::coulomb_prim(li, lj, b->ex[ka], b->ex[kb], &b->ctr[3 * i], &b->ctr[3 * j], lk, ll,
                                           b->ex[kc], b->ex[kd], &b->ctr[3 * k], &b->ctr[3 * l],
                                           b->co[ka] * b->co[kb] * b->co[kc] * b->co[kd], blk.data(), scr.data());
                    }
        const int ls[4] = {li, lj, lk, ll};
        const int f[4] = {nfunc(li, sph), nfunc(lj, sph), nfunc(lk, sph), nfunc(ll, sph)};
        std::vector<double> o((size_t)f[0] * f[1] * f[2] * f[3]), tmp;
        block_to_sph(4, ls, sph, blk.data(), o.data(), tmp);
        for (int a = 0; a < f[0]; ++a)
            for (int c = 0; c < f[1]; ++c)
                for (int e = 0; e < f[2]; ++e)
                    for (int g = 0; g < f[3]; ++g) {
                        const long long m = b->ao0[i] + a, n = b->ao0[j] + c, r = b->ao0[k] + e, s = b->ao0[l] + g;
                        const double v = o[(((size_t)a * f[1] + c) * f[2] + e) * f[3] + g];
                        const long long idx[8][4] = {{m, n, r, s}, {n, m, r, s}, {m, n, s, r}, {n, m, s, r},
                                                     {r, s, m, n}, {s, r, m, n}, {r, s, n, m}, {s, r, n, m}};
                        for (auto& q : idx) I[q[0] + nbf * (q[1] + nbf * (q[2] + nbf * q[3]))] = v;
                    }
    });
    return DONOF_OK;
}

int donof_int3c2e_dev(donof_ctx* ctx, const donof_basis* orb, const donof_basis* aux, double* I_dev) {
    using namespace donof;
    if (!ctx || !orb || !aux || !I_dev) {
        set_error(ctx, "donof_int3c2e_dev: null pointer");
        return DONOF_ERR_ARG;
    }
    if (orb->lmax > DEV_LORB || aux->lmax > DEV_LAUX) {
        set_error(ctx, "donof_int3c2e_dev: the device kernel takes orbital shells up to l = %d and auxiliary "
                       "shells up to l = %d (basis has %d and %d); use donof_int3c2e",
                  DEV_LORB, DEV_LAUX, orb->lmax, aux->lmax);
        return DONOF_ERR_ARG;
    }
    DONOF_CUDA(ctx, cudaSetDevice(ctx->device));
    {
        static std::atomic<unsigned long long> sph_mask{0};
        const unsigned long long bit = 1ull << (ctx->device & 63);
        if (!(sph_mask.load() & bit)) {
            double h[SPH_DOUBLES];
            for (int l = 0; l <= DEV_LAUX; ++l) {
                const std::vector<double>& t = sph_table().c[l];
                memcpy(h + sph_off(l), t.data(), t.size() * sizeof(double));
            }
            DONOF_CUDA(ctx, cudaMemcpyToSymbol(c_sph, h, sizeof(h)));
            sph_mask.fetch_or(bit);
        }
    }
    DevBasis dorb{}, daux{};
    DONOF_CHECK(upload_basis(ctx, const_cast<donof_basis*>(orb), &dorb));
    DONOF_CHECK(upload_basis(ctx, const_cast<donof_basis*>(aux), &daux));
    const long long npair = (long long)orb->nshell * (orb->nshell + 1) / 2;
    const long long work = npair * aux->nshell;
    const long long blocks = (work + 127) / 128;
    // the smallest per-thread arrays that hold the bases' shells
    if (orb->lmax <= 2 && aux->lmax <= 3)
        int3c2e_kernel<2, 3><<<(unsigned)blocks, 128, 0, ctx->stream>>>(dorb, daux, npair, I_dev);
    else if (orb->lmax <= 2)
        int3c2e_kernel<2, 4><<<(unsigned)blocks, 128, 0, ctx->stream>>>(dorb, daux, npair, I_dev);
    else
        int3c2e_kernel<3, 4><<<(unsigned)blocks, 128, 0, ctx->stream>>>(dorb, daux, npair, I_dev);
    count_launch();
    DONOF_CUDA(ctx, cudaGetLastError());
    return DONOF_OK;
}

}  // extern "C"
