// Device helpers shared by the CUDA sources: DFTBaby's spline evaluation and
// the Slater-Koster angular rules for s and p orbitals.  Included inside an
// anonymous namespace by each translation unit.
#pragma once

// ----------------------------------------------------------------------------
// B-spline evaluation with DFTBaby's uniform-knot interval rule
// (splines.f90:25-148).  The interval index l (1-based) is
// INT((x - t(1)) / (t(k+3) - t(k+2))) + 1, arguments at or beyond t(n-k) are
// clamped there, and l < k is raised to k+1.  Coefficient indices below 1,
// reachable only for x < 3 knot spacings (~0.12 bohr), contribute zero.
// ----------------------------------------------------------------------------
__device__ double splev_uniform(const double *__restrict__ t, int n, const double *__restrict__ c, double x) {
    const int k = 3, k1 = 4, nk1 = n - k1;
    const double tb = t[k1 - 1], te = t[nk1];
    double arg;
    int l;
    if (x <= tb) {
        arg = tb;
        l = k1;
    } else if (x >= te) {
        arg = te;
        l = nk1;
    } else {
        arg = x;
        const double dt = t[k1 + 1] - t[k1];
        l = (int)((x - t[0]) / dt) + 1;
    }
    if (l < k) l = k1;
    // de Boor-Cox recurrence for the k+1 non-zero B-splines (fpbspl)
    double h[4], hh[3];
    h[0] = 1.0;
#pragma unroll
    for (int j = 1; j <= k; ++j) {
#pragma unroll
        for (int i = 1; i <= j; ++i) hh[i - 1] = h[i - 1];
        h[0] = 0.0;
#pragma unroll
        for (int i = 1; i <= j; ++i) {
            const int li = l + i, lj = li - j;
            const double f = hh[i - 1] / (t[li - 1] - t[lj - 1]);
            h[i - 1] = h[i - 1] + f * (t[li - 1] - arg);
            h[i] = f * (arg - t[lj - 1]);
        }
    }
    double sp = 0.0;
    int ll = l - k1;
#pragma unroll
    for (int j = 0; j < k1; ++j) {
        ++ll;
        if (ll >= 1) sp += c[ll - 1] * h[j];
    }
    return sp;
}

// real spherical harmonic m -> Cartesian axis (m=-1: y, m=0: z, m=1: x)
__device__ __forceinline__ int axis_of_m(int m) { return m == -1 ? 1 : (m == 0 ? 2 : 0); }

struct SkTables {
    const int *filled;  // (npair, nsk)
    const double *knots, *coefs;  // (npair, nsk, npts)
    int nsk, npts;
};

__device__ __forceinline__ double sk_value(const SkTables &T, int ipair, int tab, double r) {
    if (tab >= T.nsk || T.filled[ipair * T.nsk + tab] != 1) return 0.0;
    const size_t b = ((size_t)ipair * T.nsk + tab) * T.npts;
    return splev_uniform(T.knots + b, T.npts, T.coefs + b, r);
}

// Slater-Koster rule for S/H0 between (l1,m1) on centre 1 and (l2,m2) on
// centre 2 with e pointing from 1 to 2 (slako_transformations_lmax2.f90, l<=1).
// Table indices: 0 ss-sigma, 2 sp-sigma, 4 ps-sigma, 5 pp-pi, 6 pp-sigma.
__device__ double sk_rule(const SkTables &T, int ipair, double r, const double e[3], int l1, int m1, int l2,
                          int m2) {
    if (l1 == 0 && l2 == 0) return sk_value(T, ipair, 0, r);
    if (l1 == 0 && l2 == 1) return e[axis_of_m(m2)] * sk_value(T, ipair, 2, r);
    if (l1 == 1 && l2 == 0) return e[axis_of_m(m1)] * sk_value(T, ipair, 4, r);
    const int a = axis_of_m(m1), b = axis_of_m(m2);
    const double vpi = sk_value(T, ipair, 5, r), vsig = sk_value(T, ipair, 6, r);
    return (a == b ? vpi : 0.0) + e[a] * e[b] * (vsig - vpi);
}

// Dipole rule <l1 m1| r_c |l2 m2> (slako_transformations_dipole_lmax2.f90,
// l<=1); D table indices 3 (s-s), 1,4 (s-p), 6,13 (p-s), 7,8,14 (p-p).
__device__ void sk_dipole_rule(const SkTables &T, int ipair, double r, const double e[3], int l1, int m1,
                               int l2, int m2, double out[3]) {
    if (l1 == 0 && l2 == 0) {
        const double d3 = sk_value(T, ipair, 3, r);
#pragma unroll
        for (int c = 0; c < 3; ++c) out[c] = e[c] * d3;
        return;
    }
    if (l1 + l2 == 1) {
        const int b = axis_of_m(l1 == 0 ? m2 : m1);
        const double dpi = sk_value(T, ipair, l1 == 0 ? 1 : 6, r);
        const double dsig = sk_value(T, ipair, l1 == 0 ? 4 : 13, r);
#pragma unroll
        for (int c = 0; c < 3; ++c) out[c] = (c == b ? dpi : 0.0) + e[c] * e[b] * (dsig - dpi);
        return;
    }
    const int a = axis_of_m(m1), b = axis_of_m(m2);
    const double d7 = sk_value(T, ipair, 7, r), d8 = sk_value(T, ipair, 8, r), d14 = sk_value(T, ipair, 14, r);
    const double cub = d14 - d7 - 2.0 * d8;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double v = e[a] * e[c] * e[b] * cub;
        if (a == c) v += e[b] * d7;
        if (c == b) v += e[a] * d8;
        if (a == b) v += e[c] * d8;
        out[c] = v;
    }
}

struct OrbTables {
    const int *ind, *typ, *ls, *ms;
};

// Geometry of the lower-triangle element (mu >= nu) as the reference reads it:
// r(j,i), x(j,i), ... = (R_j - R_i)/r with i = atom(mu), j = atom(nu).
__device__ __forceinline__ void pair_dir(int nat, const double *r, const double *x, const double *y,
                                         const double *z, int i, int j, double &rij, double e[3]) {
    const size_t o = (size_t)j * nat + i;
    rij = r[o];
    e[0] = x[o];
    e[1] = y[o];
    e[2] = z[o];
}

