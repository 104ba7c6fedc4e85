// dftbaby_b200: FP64 CUDA kernels for analytic ground- and excited-state
// gradients (DFTBaby's ExcGradients.py path) on B200 (sm_100a).
//
// The reference forms gradS, gradH0 and the gamma gradients as dense
// (3 Nat, Norb, Norb) tensors and contracts them plane by plane.  Here every
// gradient term is first reduced, with GEMMs on the host side, to adjoint
// matrices X (Norb x Norb) and Y (Nat x Nat) such that the term equals
// <gradS_n, X> or <gradGamma_n, Y>; the kernels below then evaluate the
// spline derivatives for each orbital pair on the fly and contract them with
// X without ever writing the 3 Nat Norb^2 tensors.  dftb_gradients_h0_and_s
// still produces the dense tensors for callers of the reference interface.

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "dftbaby_b200.h"

namespace {

thread_local char g_last_error_grad[256] = "";

int check_launch(const char *where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_last_error_grad, sizeof(g_last_error_grad), "%s: %s", where, cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    return DFTB_OK;
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

#include "sk_device.cuh"

// ----------------------------------------------------------------------------
// Knot interval of FITPACK's linear search (splder.f / splev.f): the smallest
// l in [k+1, n-k-1] (1-based) with arg < t(l+1), or n-k-1.  The knots of the
// tables are (nearly) uniform, so the search starts from the uniform guess
// and walks to the same l the linear search finds.
// ----------------------------------------------------------------------------
__device__ __forceinline__ int knot_interval(const double *__restrict__ t, int n, double arg) {
    const int k1 = 4, nk1 = n - k1;
    const double dt = t[k1 + 1] - t[k1];
    int l = dt > 0.0 ? (int)((arg - t[0]) / dt) + 1 : k1;
    l = l < k1 ? k1 : (l > nk1 ? nk1 : l);
    while (l > k1 && arg < t[l - 1]) --l;
    while (l < nk1 && arg >= t[l]) ++l;
    return l;
}

// Value (nu = 0) or first derivative (nu = 1) of a cubic spline at arg with
// knot interval l: fpbspl of degree 3 - nu and, for nu = 1, the derivative
// coefficients w(i) = 3 (c(i+1) - c(i)) / (t(i+4) - t(i+1)) (splder.f).
__device__ double spline_eval(const double *__restrict__ t, const double *__restrict__ c, int l, double arg, int nu) {
    const int k = 3 - nu;
    double h[4], hh[3];
    h[0] = 1.0;
    for (int j = 1; j <= k; ++j) {
        for (int i = 1; i <= j; ++i) hh[i - 1] = h[i - 1];
        h[0] = 0.0;
        for (int i = 1; i <= j; ++i) {
            const int li = l + i, lj = li - j;
            const double f = hh[i - 1] / (t[li - 1] - t[lj - 1]);
            h[i - 1] = h[i - 1] + f * (t[li - 1] - arg);
            h[i] = f * (arg - t[lj - 1]);
        }
    }
    double sp = 0.0;
    int ll = l - 4;
    for (int j = 0; j <= k; ++j) {
        ++ll;
        double w;
        if (nu == 0) {
            w = c[ll - 1];
        } else {
            const double fac = t[ll + 3] - t[ll];  // t(ll+4) - t(ll+1) in the 1-based indices of splder.f
            w = fac > 0.0 ? 3.0 * (c[ll] - c[ll - 1]) / fac : c[ll - 1];
        }
        sp += w * h[j];
    }
    return sp;
}

// splev_deriv_uniform (splines.f90:96-115): FITPACK splder, argument clamped to
// [t(k+1), t(n-k)].
__device__ double splder1(const double *__restrict__ t, int n, const double *__restrict__ c, double x) {
    const double tb = t[3], te = t[n - 4];
    const double arg = x < tb ? tb : (x > te ? te : x);
    return spline_eval(t, c, knot_interval(t, n, arg), arg, 1);
}

__device__ __forceinline__ void sk_value_deriv(const SkTables &T, int ipair, int tab, double r, double &v,
                                               double &d) {
    if (tab >= T.nsk || T.filled[ipair * T.nsk + tab] != 1) {
        v = 0.0;
        d = 0.0;
        return;
    }
    const size_t b = ((size_t)ipair * T.nsk + tab) * T.npts;
    v = splev_uniform(T.knots + b, T.npts, T.coefs + b, r);
    d = splder1(T.knots + b, T.npts, T.coefs + b, r);
}

// Gradient of sk_rule with respect to the vector r e from centre 1 to centre 2
// (slako_transformations_grad_lmax2.f90, l <= 1): chain rule through
// d e_a/d r_k = (delta_ak - e_a e_k)/r and d r/d r_k = e_k.
__device__ void sk_rule_grad(const SkTables &T, int ipair, double r, const double e[3], int l1, int m1, int l2,
                             int m2, double g[3]) {
    if (l1 == 0 && l2 == 0) {
        double v, d;
        sk_value_deriv(T, ipair, 0, r, v, d);
        for (int k = 0; k < 3; ++k) g[k] = d * e[k];
        return;
    }
    if (l1 + l2 == 1) {
        const int b = axis_of_m(l1 == 0 ? m2 : m1);
        double v, d;
        sk_value_deriv(T, ipair, l1 == 0 ? 2 : 4, r, v, d);
        for (int k = 0; k < 3; ++k) g[k] = v * ((b == k ? 1.0 : 0.0) - e[b] * e[k]) / r + e[b] * d * e[k];
        return;
    }
    const int a = axis_of_m(m1), b = axis_of_m(m2);
    double v5, d5, v6, d6;
    sk_value_deriv(T, ipair, 5, r, v5, d5);
    sk_value_deriv(T, ipair, 6, r, v6, d6);
    const double radial = (a == b ? d5 : 0.0) + e[a] * e[b] * (d6 - d5);
    for (int k = 0; k < 3; ++k) {
        const double ang = (a == k ? e[b] : 0.0) + (b == k ? e[a] : 0.0) - 2.0 * e[a] * e[b] * e[k];
        g[k] = (v6 - v5) * ang / r + radial * e[k];
    }
}

// Derivatives of S_mu,nu and H0_mu,nu, taken in the reference's orientation of
// the ordered pair (mu, nu), with respect to the position of the atom of nu
// (slako.f90:466-560).  The caller guarantees different atoms and l <= 1.
__device__ void pair_sk_gradient(int nat, const OrbTables &O, const double *r, const double *x, const double *y,
                                 const double *z, const SkTables &TS, const SkTables &TH, int mu, int nu,
                                 double gs[3], double gh[3]) {
    const int i = O.ind[mu], j = O.ind[nu];
    const int typi = O.typ[mu], typj = O.typ[nu];
    const int l1 = O.ls[mu], m1 = O.ms[mu], l2 = O.ls[nu], m2 = O.ms[nu];
    const int tmin = min(typi, typj), tmax = max(typi, typj);
    const int ipair = tmax * (tmax + 1) / 2 + tmin;
    double rij, e[3];
    pair_dir(nat, r, x, y, z, i, j, rij, e);
    if (typi <= typj) {
        sk_rule_grad(TS, ipair, rij, e, l1, m1, l2, m2, gs);
        sk_rule_grad(TH, ipair, rij, e, l1, m1, l2, m2, gh);
    } else {
        const double me[3] = {-e[0], -e[1], -e[2]};
        sk_rule_grad(TS, ipair, rij, me, l2, m2, l1, m1, gs);
        sk_rule_grad(TH, ipair, rij, me, l2, m2, l1, m1, gh);
        for (int c = 0; c < 3; ++c) {
            gs[c] = -gs[c];
            gh[c] = -gh[c];
        }
    }
}

// First orbital of atom j in the sorted, contiguous orbital -> atom table.
__device__ __forceinline__ int first_orbital(const int *ind, int norb, int j) {
    int lo = 0, hi = norb;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ind[mid] < j) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < NT / 32; ++q) s += red[q];
    return s;
}

constexpr int kGradThreads = 256;

// One CTA per atom j: out[3j+c] = sum over orbitals nu of j and mu of other,
// proximate atoms of dS_mu,nu/dR_j,c XS[mu][nu] + dH0_mu,nu/dR_j,c XH[mu][nu].
// With XS = X + X^T this is <gradS_{3j+c}, X> of the reference's tensor.
__global__ void __launch_bounds__(kGradThreads) sk_grad_contract_kernel(
    int norb, int nat, OrbTables O, const double *r, const double *x, const double *y, const double *z,
    const int *mprox, SkTables TS, SkTables TH, const double *XS, const double *XH, double *out) {
    __shared__ double red[kGradThreads / 32];
    const int j = blockIdx.x;
    const int f0 = first_orbital(O.ind, norb, j), f1 = first_orbital(O.ind, norb, j + 1);
    const int nj = f1 - f0;
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long p = threadIdx.x; p < (long long)nj * norb; p += kGradThreads) {
        const int nu = f0 + (int)(p / norb), mu = (int)(p % norb);
        const int i = O.ind[mu];
        if (i == j || mprox[(size_t)i * nat + j] == 0) continue;
        if (O.ls[mu] > 1 || O.ls[nu] > 1) continue;
        double gs[3], gh[3];
        pair_sk_gradient(nat, O, r, x, y, z, TS, TH, mu, nu, gs, gh);
        const size_t o = (size_t)mu * norb + nu;
        const double xs = XS ? XS[o] : 0.0, xh = XH ? XH[o] : 0.0;
        for (int c = 0; c < 3; ++c) acc[c] += gs[c] * xs + gh[c] * xh;
    }
    for (int c = 0; c < 3; ++c) {
        const double s = block_sum<kGradThreads>(acc[c], red);
        if (threadIdx.x == 0) out[3 * j + c] = s;
    }
}

// Dense gradS / gradH0 (3 nat, norb, norb) as slako.gradients_h0ands returns
// them: one thread per ordered pair (mu, nu); each element is written by
// exactly one thread (the planes start zeroed).
__global__ void sk_grad_dense_kernel(int norb, int nat, OrbTables O, const double *r, const double *x,
                                     const double *y, const double *z, const int *mprox, SkTables TS, SkTables TH,
                                     double *gradS, double *gradH0) {
    const int mu = blockIdx.x * blockDim.x + threadIdx.x;
    const int nu = blockIdx.y;
    if (mu >= norb || nu >= norb || mu == nu) return;
    const int i = O.ind[mu], j = O.ind[nu];
    if (i == j || mprox[(size_t)i * nat + j] == 0) return;
    if (O.ls[mu] > 1 || O.ls[nu] > 1) return;
    double gs[3], gh[3];
    pair_sk_gradient(nat, O, r, x, y, z, TS, TH, mu, nu, gs, gh);
    const size_t plane = (size_t)norb * norb;
    for (int c = 0; c < 3; ++c) {
        const size_t pl = (size_t)(3 * j + c) * plane;
        gradS[pl + (size_t)mu * norb + nu] = gs[c];
        gradS[pl + (size_t)nu * norb + mu] = gs[c];
        gradH0[pl + (size_t)mu * norb + nu] = gh[c];
        gradH0[pl + (size_t)nu * norb + mu] = gh[c];
    }
}

// ----------------------------------------------------------------------------
// Atom-pair terms: gamma and gamma^lr derivatives contracted with atom-pair
// adjoints, and the repulsive potential.
// ----------------------------------------------------------------------------
struct VrepTables {
    const double *knots, *coefs;  // (npair, nknots)
    const double *dmax;           // (npair)
    int nknots;
};

// FITPACK splev / splder with extrapolation (scipy's ext=0), zero from dmax on
// (RepulsivePotential.getVrep, RepulsivePotential.py:87-100).
__device__ double vrep_eval(const VrepTables &V, int ipair, double R, int nu) {
    if (R >= V.dmax[ipair]) return 0.0;
    const double *t = V.knots + (size_t)ipair * V.nknots, *c = V.coefs + (size_t)ipair * V.nknots;
    return spline_eval(t, c, knot_interval(t, V.nknots, R), R, nu);
}

// d/dR erf(C R)/R (GammaGaussian.g_deriv, GammaApproximation.py:141-148).
__device__ __forceinline__ double gauss_gamma_deriv(double C, double R) {
    if (fabs(R) < 1.0e-5) return 0.0;
    const double cR = C * R;
    return 2.0 * C / sqrt(M_PI) * exp(-cR * cR) / R - erf(cR) / (R * R);
}

// One CTA per atom i:
//   out[3i+c] = sum_{j != i} [ g1(R_ij) Yg[i][j] + g1lr(R_ij) Ylr[i][j] + Vrep'(R_ij) ] e_ij,c
// with e_ij = (R_i - R_j)/R_ij.  With Y = A + A^T this is <gradGamma_{3i+c}, A> of the
// reference's g1_AT / g1_AO tensors for atom-block sums A.
__global__ void __launch_bounds__(kGradThreads) pair_grad_kernel(int nat, const double *pos, const int *atype,
                                                                  const double *sigma, double r_lr,
                                                                  const double *Yg, const double *Ylr,
                                                                  VrepTables V, int use_vrep, double *out) {
    __shared__ double red[kGradThreads / 32];
    const int i = blockIdx.x;
    double acc[3] = {0.0, 0.0, 0.0};
    const double si = sigma[i];
    for (int j = threadIdx.x; j < nat; j += kGradThreads) {
        if (j == i) continue;
        const double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1],
                     dz = pos[3 * i + 2] - pos[3 * j + 2];
        const double R = sqrt(dx * dx + dy * dy + dz * dz);
        const double s2 = si * si + sigma[j] * sigma[j];
        double w = 0.0;
        if (Yg) w += gauss_gamma_deriv(1.0 / sqrt(2.0 * s2), R) * Yg[(size_t)i * nat + j];
        if (Ylr) w += gauss_gamma_deriv(1.0 / sqrt(2.0 * (s2 + 0.5 * r_lr * r_lr)), R) * Ylr[(size_t)i * nat + j];
        if (use_vrep) {
            const int ta = atype[i], tb = atype[j];
            const int tmin = min(ta, tb), tmax = max(ta, tb);
            w += vrep_eval(V, tmax * (tmax + 1) / 2 + tmin, R, 1);
        }
        acc[0] += w * dx / R;
        acc[1] += w * dy / R;
        acc[2] += w * dz / R;
    }
    for (int c = 0; c < 3; ++c) {
        const double s = block_sum<kGradThreads>(acc[c], red);
        if (threadIdx.x == 0) out[3 * i + c] = s;
    }
}

// Half the repulsive energy of every atom: e[i] = 1/2 sum_{j != i} Vrep(R_ij).
__global__ void __launch_bounds__(kGradThreads) vrep_energy_kernel(int nat, const double *pos, const int *atype,
                                                                    VrepTables V, double *e) {
    __shared__ double red[kGradThreads / 32];
    const int i = blockIdx.x;
    double acc = 0.0;
    for (int j = threadIdx.x; j < nat; j += kGradThreads) {
        if (j == i) continue;
        const double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1],
                     dz = pos[3 * i + 2] - pos[3 * j + 2];
        const double R = sqrt(dx * dx + dy * dy + dz * dz);
        const int ta = atype[i], tb = atype[j];
        const int tmin = min(ta, tb), tmax = max(ta, tb);
        acc += vrep_eval(V, tmax * (tmax + 1) / 2 + tmin, R, 0);
    }
    const double s = block_sum<kGradThreads>(acc, red);
    if (threadIdx.x == 0) e[i] = 0.5 * s;
}

int fail_grad(int code, const char *what) {
    snprintf(g_last_error_grad, sizeof(g_last_error_grad), "%s", what);
    return code;
}

}  // namespace

extern "C" {

const char *dftb_grad_last_error(void) { return g_last_error_grad; }

int dftb_gradients_h0_and_s(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                            const double *r, const double *x, const double *y, const double *z, const int *mprox,
                            int deg, const int *tab_filled, const double *S_knots, const double *S_coefs,
                            const double *H_knots, const double *H_coefs, int npair, int nsk, int npts,
                            double *gradS, double *gradH0, void *stream) {
    if (norb <= 0 || nat <= 0 || npair <= 0 || nsk <= 0 || npts < 8)
        return fail_grad(DFTB_ERR_BAD_SIZE, "gradients_h0_and_s: sizes");
    if (deg != 3) return fail_grad(DFTB_ERR_UNSUPPORTED, "gradients_h0_and_s: only cubic splines");
    if (norb > 65535) return fail_grad(DFTB_ERR_BAD_SIZE, "gradients_h0_and_s: norb above 65535");
    if (!ind || !typ || !ls || !ms || !r || !x || !y || !z || !mprox || !tab_filled || !S_knots || !S_coefs ||
        !H_knots || !H_coefs || !gradS || !gradH0)
        return fail_grad(DFTB_ERR_NULL, "gradients_h0_and_s: null");
    const size_t bytes = sizeof(double) * 3 * (size_t)nat * norb * norb;
    if (cudaMemsetAsync(gradS, 0, bytes, S(stream)) != cudaSuccess ||
        cudaMemsetAsync(gradH0, 0, bytes, S(stream)) != cudaSuccess)
        return check_launch("gradients_h0_and_s: memset");
    OrbTables O{ind, typ, ls, ms};
    SkTables TS{tab_filled, S_knots, S_coefs, nsk, npts};
    SkTables TH{tab_filled, H_knots, H_coefs, nsk, npts};
    dim3 grid(cdiv(norb, 128), norb);
    sk_grad_dense_kernel<<<grid, 128, 0, S(stream)>>>(norb, nat, O, r, x, y, z, mprox, TS, TH, gradS, gradH0);
    return check_launch("sk_grad_dense_kernel");
}

int dftb_sk_gradient_contract(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                              const double *r, const double *x, const double *y, const double *z, const int *mprox,
                              int deg, const int *tab_filled, const double *S_knots, const double *S_coefs,
                              const double *H_knots, const double *H_coefs, int npair, int nsk, int npts,
                              const double *XS, const double *XH, double *grad, void *stream) {
    if (norb <= 0 || nat <= 0 || npair <= 0 || nsk <= 0 || npts < 8)
        return fail_grad(DFTB_ERR_BAD_SIZE, "sk_gradient_contract: sizes");
    if (deg != 3) return fail_grad(DFTB_ERR_UNSUPPORTED, "sk_gradient_contract: only cubic splines");
    if (!ind || !typ || !ls || !ms || !r || !x || !y || !z || !mprox || !tab_filled || !S_knots || !S_coefs ||
        !H_knots || !H_coefs || !grad || (!XS && !XH))
        return fail_grad(DFTB_ERR_NULL, "sk_gradient_contract: null");
    OrbTables O{ind, typ, ls, ms};
    SkTables TS{tab_filled, S_knots, S_coefs, nsk, npts};
    SkTables TH{tab_filled, H_knots, H_coefs, nsk, npts};
    sk_grad_contract_kernel<<<nat, kGradThreads, 0, S(stream)>>>(norb, nat, O, r, x, y, z, mprox, TS, TH, XS, XH,
                                                                 grad);
    return check_launch("sk_grad_contract_kernel");
}

int dftb_pair_gradients(int nat, const double *pos, const int *atype, const double *sigma, double r_lr,
                        const double *Yg, const double *Ylr, const double *vrep_knots, const double *vrep_coefs,
                        const double *vrep_dmax, int nknots, double *grad, void *stream) {
    if (nat <= 0) return fail_grad(DFTB_ERR_BAD_SIZE, "pair_gradients: nat");
    const int use_vrep = vrep_knots != nullptr;
    if (use_vrep && (nknots < 8 || !vrep_coefs || !vrep_dmax))
        return fail_grad(DFTB_ERR_BAD_SIZE, "pair_gradients: repulsive-potential tables");
    if (!pos || !grad || ((Yg || Ylr) && !sigma) || (use_vrep && !atype))
        return fail_grad(DFTB_ERR_NULL, "pair_gradients: null");
    VrepTables V{vrep_knots, vrep_coefs, vrep_dmax, nknots};
    pair_grad_kernel<<<nat, kGradThreads, 0, S(stream)>>>(nat, pos, atype, sigma, r_lr, Yg, Ylr, V, use_vrep, grad);
    return check_launch("pair_grad_kernel");
}

int dftb_repulsive_energy(int nat, const double *pos, const int *atype, const double *vrep_knots,
                          const double *vrep_coefs, const double *vrep_dmax, int nknots, double *e_atom,
                          void *stream) {
    if (nat <= 0 || nknots < 8) return fail_grad(DFTB_ERR_BAD_SIZE, "repulsive_energy: sizes");
    if (!pos || !atype || !vrep_knots || !vrep_coefs || !vrep_dmax || !e_atom)
        return fail_grad(DFTB_ERR_NULL, "repulsive_energy: null");
    VrepTables V{vrep_knots, vrep_coefs, vrep_dmax, nknots};
    vrep_energy_kernel<<<nat, kGradThreads, 0, S(stream)>>>(nat, pos, atype, V, e_atom);
    return check_launch("vrep_energy_kernel");
}

}  // extern "C"
