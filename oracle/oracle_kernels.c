/*
 * CPU oracle: C/OpenMP restatement of DFTBaby's Fortran kernels on the
 * LR-TD-DFTB path.  TEST INFRASTRUCTURE ONLY -- used by tests/, the smoke
 * check and bench.py's CPU baseline; never by the product path.
 *
 * Restated from (file:line inside the DFTBaby project):
 *   splev_uniform / fpbspl  DFTB/extensions/splines.f90:25-92, 118-148
 *   directional_cosines     DFTB/extensions/slako.f90:31-70
 *   H0andS                  DFTB/extensions/slako.f90:77-231
 *   DipoleMatrix            DFTB/extensions/slako.f90:238-394
 *   SK rules (s,p subset)   DFTB/extensions/slako_transformations_lmax2.f90
 *                           DFTB/extensions/slako_transformations_dipole_lmax2.f90
 *   trans_charges           DFTB/extensions/tddftb.f90:12-112
 *   monopoles               DFTB/extensions/mulliken.f90:11-66
 *   splev_deriv_uniform     DFTB/extensions/splines.f90:96-115 with splder.f (FITPACK)
 *   gradients_H0andS        DFTB/extensions/slako.f90:402-569
 *   SK gradient rules       DFTB/extensions/slako_transformations_grad_lmax2.f90
 *   repulsive potential     scipy.interpolate.splev (FITPACK splev/splder, ext=0)
 *                           as called by RepulsivePotential.getVrep
 *                           (DFTB/RepulsivePotential/RepulsivePotential.py:87-100)
 *
 * Array layouts are C row-major.  Symmetric matrices (S, H0, P) are Norb x Norb.
 * The dipole matrix is returned as three planes D[c][mu][nu], c = x,y,z.
 * Transition charges are q[A][p][q] (A = atom index first), i.e. numpy arrays
 * of the reference's logical shape (Nat, n1, n2).
 *
 * The Slater-Koster angular rules are written in tensor form (see sk_rule and
 * sk_dipole_rule); tests/golden/sk_rules.npz pins them against the reference's
 * own per-case rule table.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- B-splines ------------------------------------------------------- */

/* De Boor-Cox recurrence for the k+1 non-zero B-splines at x, knot interval l
 * (1-based, as in the Fortran).  splines.f90:118-148 */
static void fpbspl(const double *t, int k, double x, int l, double *h)
{
    double hh[5];
    h[0] = 1.0;
    for (int j = 1; j <= k; ++j) {
        for (int i = 1; i <= j; ++i) hh[i - 1] = h[i - 1];
        h[0] = 0.0;
        for (int i = 1; i <= j; ++i) {
            int li = l + i, lj = li - j;
            double f = hh[i - 1] / (t[li - 1] - t[lj - 1]);
            h[i - 1] = h[i - 1] + f * (t[li - 1] - x);
            h[i] = f * (x - t[lj - 1]);
        }
    }
}

/* Bug-compatible evaluation of a spline with uniformly spaced interior knots.
 * splines.f90:25-92.  The interval index is l = INT((x - t(1))/dt) + 1 with
 * dt = t(k+3) - t(k+2); for not-a-knot knots from splrep this selects the
 * piece two knots to the left of the containing interval, and arguments at or
 * beyond t(n-k) are clamped there.  A coefficient index below 1 (reachable
 * only for x < 3*dt, i.e. nuclei closer than ~0.12 bohr) reads outside the
 * array in the reference; it contributes zero here. */
/* Test switch: when nonzero, oracle_splev_uniform evaluates the spline exactly
 * (FITPACK interval search, argument clamped like splder) instead of the
 * reference's shifted-interval shortcut, so that energies and their analytic
 * gradients (which use splder) become consistent to rounding. */
int oracle_exact_splines = 0;

double oracle_splev_uniform(const double *t, int n, const double *c, int k, double x)
{
    int k1 = k + 1, nk1 = n - k1;
    if (oracle_exact_splines) {
        double tb = t[k1 - 1], te = t[nk1];
        double arg = x < tb ? tb : (x > te ? te : x);
        int l = k1, l1 = l + 1;
        while (!(arg < t[l1 - 1] || l == nk1)) {
            l = l1;
            l1 = l + 1;
        }
        double h[6];
        fpbspl(t, k, arg, l, h);
        double sp = 0.0;
        for (int j = 1; j <= k1; ++j) sp += c[l - k1 + j - 1] * h[j - 1];
        return sp;
    }
    double tb = t[k1 - 1], te = t[nk1];
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
        double dt = t[k1 + 1] - t[k1];
        l = (int)((x - t[0]) / dt) + 1;
    }
    if (l < k) l = k1;
    double h[6];
    fpbspl(t, k, arg, l, h);
    double sp = 0.0;
    int ll = l - k1;
    for (int j = 1; j <= k1; ++j) {
        ++ll;
        if (ll >= 1) sp += c[ll - 1] * h[j - 1];
    }
    return sp;
}

/* First derivative of a spline, FITPACK splder with nu = 1 as called by
 * splev_deriv_uniform (splines.f90:96-115, splder.f).  The derivative is a
 * spline of degree k-1 on the same knots with coefficients
 * w(i) = k (c(i+1) - c(i)) / (t(i+k+1) - t(i+1)) (left at c(i) where that knot
 * span is not positive); the argument is clamped to [t(k+1), t(n-k)] and the
 * knot interval found by a linear search, unlike splev_uniform. */
double oracle_splder1(const double *t, int n, const double *c, int k, double x)
{
    int k1 = k + 1, nk1 = n - k1;
    double tb = t[k1 - 1], te = t[nk1];
    double arg = x < tb ? tb : (x > te ? te : x);
    int l = k1, l1 = l + 1;
    while (!(arg < t[l1 - 1] || l == nk1)) {
        l = l1;
        l1 = l + 1;
    }
    double h[6];
    fpbspl(t, k - 1, arg, l, h);
    double sp = 0.0;
    int ll = l - k1;
    for (int j = 1; j <= k; ++j) {
        ++ll;  /* 1-based index of the derivative coefficient */
        double fac = t[ll + k] - t[ll];
        double w = fac > 0.0 ? k * (c[ll] - c[ll - 1]) / fac : c[ll - 1];
        sp += w * h[j - 1];
    }
    return sp;
}

/* FITPACK splev / splder (nu = 0 or 1) with extrapolation (scipy's ext=0): the
 * knot interval is searched with t(l) <= x < t(l+1), k+1 <= l <= n-k-1, and x
 * is not clamped.  Used for the repulsive potentials. */
double oracle_splev_ext(const double *t, int n, const double *c, int k, double x, int nu)
{
    int k1 = k + 1, nk1 = n - k1;
    int l = k1, l1 = l + 1;
    while (!(x < t[l1 - 1] || l == nk1)) {
        l = l1;
        l1 = l + 1;
    }
    double h[6];
    double sp = 0.0;
    int ll = l - k1;
    if (nu == 0) {
        fpbspl(t, k, x, l, h);
        for (int j = 1; j <= k1; ++j) {
            ++ll;
            sp += c[ll - 1] * h[j - 1];
        }
    } else {
        fpbspl(t, k - 1, x, l, h);
        for (int j = 1; j <= k; ++j) {
            ++ll;
            double fac = t[ll + k] - t[ll];
            double w = fac > 0.0 ? k * (c[ll] - c[ll - 1]) / fac : c[ll - 1];
            sp += w * h[j - 1];
        }
    }
    return sp;
}

/* ---- Slater-Koster angular rules ------------------------------------- */

/* real spherical harmonic index m -> Cartesian axis (m=-1: y, 0: z, 1: x) */
static inline int axis_of_m(int m) { return m == -1 ? 1 : (m == 0 ? 2 : 0); }

/* S or H0 element between orbital (l1,m1) on centre 1 and (l2,m2) on centre 2,
 * e = unit vector from centre 1 to centre 2, V = SK integrals of the pair
 * (table index as in the reference: 0 ss-sigma, 2 sp-sigma, 4 ps-sigma,
 * 5 pp-pi, 6 pp-sigma).  Equivalent to slako_transformations_lmax2.f90 for l<=1. */
double oracle_sk_rule(int l1, int m1, int l2, int m2, const double *e, const double *V)
{
    if (l1 == 0 && l2 == 0) return V[0];
    if (l1 == 0 && l2 == 1) return e[axis_of_m(m2)] * V[2];
    if (l1 == 1 && l2 == 0) return e[axis_of_m(m1)] * V[4];
    int a = axis_of_m(m1), b = axis_of_m(m2);
    return (a == b ? V[5] : 0.0) + e[a] * e[b] * (V[6] - V[5]);
}

/* Gradient of oracle_sk_rule with respect to the vector r e from centre 1 to
 * centre 2 (the position of centre 2), given the SK integrals V and their
 * radial derivatives Vd at r.  Chain rule through the direction cosines,
 * d e_a / d r_k = (delta_ak - e_a e_k) / r, and the radius, d r / d r_k = e_k.
 * Equivalent to slako_transformations_grad_lmax2.f90 for l<=1. */
void oracle_sk_rule_grad(int l1, int m1, int l2, int m2, double r, const double *e, const double *V,
                         const double *Vd, double *g)
{
    for (int k = 0; k < 3; ++k) {
        double gk;
        if (l1 == 0 && l2 == 0) {
            gk = Vd[0] * e[k];
        } else if (l1 == 0 && l2 == 1) {
            int b = axis_of_m(m2);
            gk = V[2] * ((b == k ? 1.0 : 0.0) - e[b] * e[k]) / r + e[b] * Vd[2] * e[k];
        } else if (l1 == 1 && l2 == 0) {
            int a = axis_of_m(m1);
            gk = V[4] * ((a == k ? 1.0 : 0.0) - e[a] * e[k]) / r + e[a] * Vd[4] * e[k];
        } else {
            int a = axis_of_m(m1), b = axis_of_m(m2);
            double ang = (a == k ? e[b] : 0.0) + (b == k ? e[a] : 0.0) - 2.0 * e[a] * e[b] * e[k];
            gk = (V[6] - V[5]) * ang / r + ((a == b ? Vd[5] : 0.0) + e[a] * e[b] * (Vd[6] - Vd[5])) * e[k];
        }
        g[k] = gk;
    }
}

/* Dipole element <l1 m1| r_c |l2 m2> (c: 0=x,1=y,2=z) with dipole SK integrals
 * D (indices 1,3,4 for s-s/s-p; 6,13 for p-s; 7,8,14 for p-p).  Equivalent to
 * slako_transformations_dipole_lmax2.f90 for l<=1. */
double oracle_sk_dipole_rule(int l1, int m1, int c, int l2, int m2, const double *e, const double *D)
{
    if (l1 == 0 && l2 == 0) return e[c] * D[3];
    if (l1 == 0 && l2 == 1) {
        int b = axis_of_m(m2);
        return (c == b ? D[1] : 0.0) + e[c] * e[b] * (D[4] - D[1]);
    }
    if (l1 == 1 && l2 == 0) {
        int b = axis_of_m(m1);
        return (c == b ? D[6] : 0.0) + e[c] * e[b] * (D[13] - D[6]);
    }
    int a = axis_of_m(m1), b = axis_of_m(m2);
    double r = e[a] * e[c] * e[b] * (D[14] - D[7] - 2.0 * D[8]);
    if (a == c) r += e[b] * D[7];
    if (c == b) r += e[a] * D[8];
    if (a == b) r += e[c] * D[8];
    return r;
}

/* ---- geometry ---------------------------------------------------------- */

/* r(i,j) and unit vectors from atom j to atom i; z=1 on the diagonal.
 * slako.f90:31-70.  r,x,y,z are Nat x Nat row-major with [i][j]. */
void oracle_directional_cosines(int nat, const double *pos, double *r, double *x, double *y, double *z)
{
#pragma omp parallel for
    for (int j = 0; j < nat; ++j)
        for (int i = 0; i < nat; ++i) {
            double xc = pos[3 * i] - pos[3 * j];
            double yc = pos[3 * i + 1] - pos[3 * j + 1];
            double zc = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(xc * xc + yc * yc + zc * zc);
            size_t o = (size_t)i * nat + j;
            r[o] = rr;
            if (rr > 0.0) {
                x[o] = xc / rr;
                y[o] = yc / rr;
                z[o] = zc / rr;
            } else {
                x[o] = 0.0;
                y[o] = 0.0;
                z[o] = 1.0;
            }
        }
}

/* direction and distance from atom i (orbital mu) to atom j (orbital nu):
 * the reference reads r(j,i), x(j,i), ... = (pos_j - pos_i)/r */
static void pair_geometry(const double *pos, int i, int j, double *rij, double *e)
{
    double xc = pos[3 * j] - pos[3 * i];
    double yc = pos[3 * j + 1] - pos[3 * i + 1];
    double zc = pos[3 * j + 2] - pos[3 * i + 2];
    double rr = sqrt(xc * xc + yc * yc + zc * zc);
    *rij = rr;
    if (rr > 0.0) {
        e[0] = xc / rr;
        e[1] = yc / rr;
        e[2] = zc / rr;
    } else {
        e[0] = 0.0;
        e[1] = 0.0;
        e[2] = 1.0;
    }
}

/* ---- H0 and S ---------------------------------------------------------- */

/* slako.f90:77-231.  Orbital tables ind/typ/ls/ms have length norb, typ are
 * atom types 0..ntype-1, mprox is Nat x Nat (1 = interacting), tables are
 * [npair][nsk][npts].  S and H0 (norb x norb) are fully overwritten. */
void oracle_h0_and_s(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                     const double *pos, const int *mprox, const double *orben, int deg,
                     const int *tab_filled, const double *S_knots, const double *S_coefs,
                     const double *H_knots, const double *H_coefs, int npair, int nsk, int npts,
                     double *S, double *H0)
{
    (void)npair;
    memset(S, 0, sizeof(double) * (size_t)norb * norb);
    memset(H0, 0, sizeof(double) * (size_t)norb * norb);
#pragma omp parallel for schedule(dynamic, 1)
    for (int nu = 0; nu < norb; ++nu) {
        double Si[16], Hi[16];
        int j = ind[nu], typj = typ[nu], l2 = ls[nu], m2 = ms[nu];
        for (int mu = nu; mu < norb; ++mu) {
            int i = ind[mu], typi = typ[mu], l1 = ls[mu], m1 = ms[mu];
            if (mprox[(size_t)i * nat + j] == 0) continue;
            size_t o = (size_t)mu * norb + nu;
            if (mu == nu) {
                S[o] = 1.0;
                H0[o] = orben[mu];
                continue;
            }
            double rij, e[3];
            pair_geometry(pos, i, j, &rij, e);
            if (i != j) {
                int tmin = typi < typj ? typi : typj, tmax = typi < typj ? typj : typi;
                int ipair = tmax * (tmax + 1) / 2 + tmin;
                for (int tab = 0; tab < nsk; ++tab) {
                    if (tab_filled[ipair * nsk + tab] == 1) {
                        size_t b = ((size_t)ipair * nsk + tab) * npts;
                        Si[tab] = oracle_splev_uniform(S_knots + b, npts, S_coefs + b, deg, rij);
                        Hi[tab] = oracle_splev_uniform(H_knots + b, npts, H_coefs + b, deg, rij);
                    } else {
                        Si[tab] = 0.0;
                        Hi[tab] = 0.0;
                    }
                }
            }
            if (typi <= typj) {
                if (i == j) {
                    S[o] = 0.0;
                    H0[o] = 0.0;
                } else {
                    S[o] = oracle_sk_rule(l1, m1, l2, m2, e, Si);
                    H0[o] = oracle_sk_rule(l1, m1, l2, m2, e, Hi);
                }
            } else {
                double me[3] = {-e[0], -e[1], -e[2]};
                S[o] = oracle_sk_rule(l2, m2, l1, m1, me, Si);
                H0[o] = oracle_sk_rule(l2, m2, l1, m1, me, Hi);
            }
        }
    }
    for (int nu = 0; nu < norb; ++nu)
        for (int mu = 0; mu < nu; ++mu) {
            S[(size_t)mu * norb + nu] = S[(size_t)nu * norb + mu];
            H0[(size_t)mu * norb + nu] = H0[(size_t)nu * norb + mu];
        }
}

/* ---- overlap between two geometries ------------------------------------- */

/* slako.f90:576-687 (overlap12, called by ScalarCoupling._overlap_AB_f90, ScalarCoupling.py:105-137).
 * S(mu, nu) = <phi_mu(geometry 1) | phi_nu(geometry 2)> for every orbital pair: no proximity
 * cutoff and no on-site shortcut (an atom and its displaced copy are evaluated with the SK tables,
 * whose splev_uniform clamps r below the first knot).  The direction runs from the atom of mu in
 * geometry 1 to the atom of nu in geometry 2 (the reference reads r(j,i) of
 * directional_cosines(pos1, pos2), slako.f90:31-70), and each element is evaluated in its own
 * orientation.  pos1, pos2: (nat, 3); S: (norb, norb) row-major. */
void oracle_overlap12(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                      const double *pos1, const double *pos2, int deg, const int *tab_filled,
                      const double *S_knots, const double *S_coefs, int npair, int nsk, int npts, double *S)
{
    (void)npair;
    (void)nat;
#pragma omp parallel for schedule(dynamic, 1)
    for (int nu = 0; nu < norb; ++nu) {
        double Si[16];
        int j = ind[nu], typj = typ[nu], l2 = ls[nu], m2 = ms[nu];
        for (int mu = 0; mu < norb; ++mu) {
            int i = ind[mu], typi = typ[mu], l1 = ls[mu], m1 = ms[mu];
            double xc = pos2[3 * j] - pos1[3 * i], yc = pos2[3 * j + 1] - pos1[3 * i + 1],
                   zc = pos2[3 * j + 2] - pos1[3 * i + 2];
            double rij = sqrt(xc * xc + yc * yc + zc * zc), e[3];
            if (rij > 0.0) {
                e[0] = xc / rij;
                e[1] = yc / rij;
                e[2] = zc / rij;
            } else {
                e[0] = 0.0;
                e[1] = 0.0;
                e[2] = 1.0;
            }
            int tmin = typi < typj ? typi : typj, tmax = typi < typj ? typj : typi;
            int ipair = tmax * (tmax + 1) / 2 + tmin;
            for (int tab = 0; tab < nsk; ++tab) {
                if (tab_filled[ipair * nsk + tab] == 1) {
                    size_t b = ((size_t)ipair * nsk + tab) * npts;
                    Si[tab] = oracle_splev_uniform(S_knots + b, npts, S_coefs + b, deg, rij);
                } else {
                    Si[tab] = 0.0;
                }
            }
            size_t o = (size_t)mu * norb + nu;
            if (typi <= typj) {
                S[o] = oracle_sk_rule(l1, m1, l2, m2, e, Si);
            } else {
                double me[3] = {-e[0], -e[1], -e[2]};
                S[o] = oracle_sk_rule(l2, m2, l1, m1, me, Si);
            }
        }
    }
}

/* ---- gradients of H0 and S ------------------------------------------------ */

/* Derivative of the S and H0 elements of the ordered pair (mu, nu) (the reference's
 * orientation: direction from the atom of mu to the atom of nu) with respect to
 * the position of the atom of nu.  slako.f90:466-560. */
static void pair_gradient(int mu, int nu, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                          const double *pos, int deg, const int *tab_filled, const double *S_knots,
                          const double *S_coefs, const double *H_knots, const double *H_coefs, int nsk, int npts,
                          double *sg, double *hg)
{
    (void)nat;
    int i = ind[mu], typi = typ[mu], l1 = ls[mu], m1 = ms[mu];
    int j = ind[nu], typj = typ[nu], l2 = ls[nu], m2 = ms[nu];
    double rij, e[3], Si[16], Hi[16], Sd[16], Hd[16];
    pair_geometry(pos, i, j, &rij, e);
    int tmin = typi < typj ? typi : typj, tmax = typi < typj ? typj : typi;
    int ipair = tmax * (tmax + 1) / 2 + tmin;
    for (int tab = 0; tab < nsk; ++tab) {
        Si[tab] = Hi[tab] = Sd[tab] = Hd[tab] = 0.0;
        if (tab_filled[ipair * nsk + tab] == 1) {
            size_t b = ((size_t)ipair * nsk + tab) * npts;
            Si[tab] = oracle_splev_uniform(S_knots + b, npts, S_coefs + b, deg, rij);
            Hi[tab] = oracle_splev_uniform(H_knots + b, npts, H_coefs + b, deg, rij);
            Sd[tab] = oracle_splder1(S_knots + b, npts, S_coefs + b, deg, rij);
            Hd[tab] = oracle_splder1(H_knots + b, npts, H_coefs + b, deg, rij);
        }
    }
    if (typi <= typj) {
        oracle_sk_rule_grad(l1, m1, l2, m2, rij, e, Si, Sd, sg);
        oracle_sk_rule_grad(l1, m1, l2, m2, rij, e, Hi, Hd, hg);
    } else {
        /* centres swapped: the rule is a function of -e, i.e. of pos_i - pos_j */
        double me[3] = {-e[0], -e[1], -e[2]};
        oracle_sk_rule_grad(l2, m2, l1, m1, rij, me, Si, Sd, sg);
        oracle_sk_rule_grad(l2, m2, l1, m1, rij, me, Hi, Hd, hg);
        for (int c = 0; c < 3; ++c) {
            sg[c] = -sg[c];
            hg[c] = -hg[c];
        }
    }
}

/* Test switch: when nonzero, the element (mu, nu) with mu < nu is differentiated
 * in the orientation (nu, mu) that H0andS uses for its value (it fills the
 * mu >= nu triangle and mirrors it), making gradients and matrices consistent
 * even where a pair's s-p and p-s tables disagree.  The reference
 * differentiates every ordered pair in its own orientation (default, 0). */
int oracle_consistent_gradients = 0;

/* slako.f90:402-569.  gradS, gradH0 are [3*nat][norb][norb]; element
 * [3j+c][mu][nu] (and its mirror [3j+c][nu][mu]) receives the derivative of
 * S_mu,nu with respect to coordinate c of atom j = ind[nu], for every ordered
 * pair mu != nu on different, proximate atoms.  Spline values come from
 * splev_uniform, their radial derivatives from splder. */
void oracle_gradients_h0_and_s(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                               const double *pos, const int *mprox, int deg, const int *tab_filled,
                               const double *S_knots, const double *S_coefs, const double *H_knots,
                               const double *H_coefs, int npair, int nsk, int npts, double *gradS, double *gradH0)
{
    (void)npair;
    size_t plane = (size_t)norb * norb;
    memset(gradS, 0, sizeof(double) * 3 * nat * plane);
    memset(gradH0, 0, sizeof(double) * 3 * nat * plane);
    /* parallel over the atom j that owns the derivative: each thread writes only planes 3j..3j+2 */
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < nat; ++j) {
        for (int nu = 0; nu < norb; ++nu) {
            if (ind[nu] != j) continue;
            for (int mu = 0; mu < norb; ++mu) {
                int i = ind[mu];
                if (mprox[(size_t)i * nat + j] == 0 || mu == nu || i == j) continue;
                double sg[3], hg[3];
                if (oracle_consistent_gradients && mu < nu) {
                    pair_gradient(nu, mu, nat, ind, typ, ls, ms, pos, deg, tab_filled, S_knots, S_coefs, H_knots,
                                  H_coefs, nsk, npts, sg, hg);
                    for (int c = 0; c < 3; ++c) {
                        sg[c] = -sg[c];
                        hg[c] = -hg[c];
                    }
                } else {
                    pair_gradient(mu, nu, nat, ind, typ, ls, ms, pos, deg, tab_filled, S_knots, S_coefs, H_knots,
                                  H_coefs, nsk, npts, sg, hg);
                }
                for (int c = 0; c < 3; ++c) {
                    size_t pl = (size_t)(3 * j + c) * plane;
                    gradS[pl + (size_t)mu * norb + nu] += sg[c];
                    gradS[pl + (size_t)nu * norb + mu] += sg[c];
                    gradH0[pl + (size_t)mu * norb + nu] += hg[c];
                    gradH0[pl + (size_t)nu * norb + mu] += hg[c];
                }
            }
        }
    }
}

/* ---- dipole matrix ----------------------------------------------------- */

/* slako.f90:238-394.  D receives three planes [3][norb][norb]. */
void oracle_dipole_matrix(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                          const double *pos, const int *mprox, const double *S, int deg,
                          const int *tab_filled_D, const double *D_knots, const double *D_coefs,
                          int npair, int nskd, int npts, double *D)
{
    (void)npair;
    size_t plane = (size_t)norb * norb;
    memset(D, 0, sizeof(double) * 3 * plane);
#pragma omp parallel for schedule(dynamic, 1)
    for (int nu = 0; nu < norb; ++nu) {
        double Di[32];
        int j = ind[nu], typj = typ[nu], l2 = ls[nu], m2 = ms[nu];
        for (int mu = nu; mu < norb; ++mu) {
            int i = ind[mu], typi = typ[mu], l1 = ls[mu], m1 = ms[mu];
            if (mprox[(size_t)i * nat + j] == 0) continue;
            double rij, e[3];
            pair_geometry(pos, i, j, &rij, e);
            int tmin = typi < typj ? typi : typj, tmax = typi < typj ? typj : typi;
            int ipair = tmax * (tmax + 1) / 2 + tmin;
            for (int tab = 0; tab < nskd; ++tab) {
                if (tab_filled_D[ipair * nskd + tab] == 1) {
                    size_t b = ((size_t)ipair * nskd + tab) * npts;
                    Di[tab] = oracle_splev_uniform(D_knots + b, npts, D_coefs + b, deg, rij);
                } else {
                    Di[tab] = 0.0;
                }
            }
            size_t o = (size_t)mu * norb + nu;
            double s = S[o];
            /* mr = +1 (x), -1 (y), 0 (z) in the reference; planes are x,y,z */
            if (typi <= typj) {
                for (int c = 0; c < 3; ++c)
                    D[c * plane + o] = oracle_sk_dipole_rule(l1, m1, c, l2, m2, e, Di) + pos[3 * j + c] * s;
            } else {
                double me[3] = {-e[0], -e[1], -e[2]};
                for (int c = 0; c < 3; ++c)
                    D[c * plane + o] = oracle_sk_dipole_rule(l2, m2, c, l1, m1, me, Di) + pos[3 * i + c] * s;
            }
        }
    }
    for (int c = 0; c < 3; ++c)
        for (int nu = 0; nu < norb; ++nu)
            for (int mu = 0; mu < nu; ++mu)
                D[c * plane + (size_t)mu * norb + nu] = D[c * plane + (size_t)nu * norb + mu];
}

/* ---- transition charges ------------------------------------------------ */

/* q^{pq}_A = 1/2 sum_{mu in A} (C_mu,p (SC)_mu,q + C_mu,q (SC)_mu,p).
 * tddftb.f90:12-112.  orbs_occ is norb x nocc row-major (column i = MO i),
 * orbs_virt norb x nvirt, S norb x norb.  Outputs q_oo[Nat][nocc][nocc],
 * q_ov[Nat][nocc][nvirt], q_vv[Nat][nvirt][nvirt]; any may be NULL. */
void oracle_trans_charges(int norb, int nat, int nocc, int nvirt, const double *orbs_occ,
                          const double *orbs_virt, const double *S, const int *orbs_per_atom,
                          double *q_oo, double *q_ov, double *q_vv)
{
    double *sco = (double *)calloc((size_t)norb * nocc, sizeof(double));
    double *scv = (double *)calloc((size_t)norb * nvirt, sizeof(double));
#pragma omp parallel for
    for (int mu = 0; mu < norb; ++mu)
        for (int nu = 0; nu < norb; ++nu) {
            double s = S[(size_t)mu * norb + nu];
            for (int i = 0; i < nocc; ++i) sco[(size_t)mu * nocc + i] += s * orbs_occ[(size_t)nu * nocc + i];
            for (int a = 0; a < nvirt; ++a) scv[(size_t)mu * nvirt + a] += s * orbs_virt[(size_t)nu * nvirt + a];
        }
    int *first = (int *)malloc(sizeof(int) * (nat + 1));
    first[0] = 0;
    for (int A = 0; A < nat; ++A) first[A + 1] = first[A] + orbs_per_atom[A];
#define QBLOCK(OUT, C1, SC1, N1, C2, SC2, N2)                                                  \
    if (OUT) {                                                                                 \
        _Pragma("omp parallel for") for (int p = 0; p < N1; ++p) for (int q = 0; q < N2; ++q) \
            for (int A = 0; A < nat; ++A) {                                                    \
                double acc = 0.0;                                                              \
                for (int mu = first[A]; mu < first[A + 1]; ++mu)                               \
                    acc += C1[(size_t)mu * N1 + p] * SC2[(size_t)mu * N2 + q] +                \
                           C2[(size_t)mu * N2 + q] * SC1[(size_t)mu * N1 + p];                 \
                OUT[((size_t)A * N1 + p) * N2 + q] = 0.5 * acc;                                \
            }                                                                                  \
    }
    QBLOCK(q_oo, orbs_occ, sco, nocc, orbs_occ, sco, nocc)
    QBLOCK(q_ov, orbs_occ, sco, nocc, orbs_virt, scv, nvirt)
    QBLOCK(q_vv, orbs_virt, scv, nvirt, orbs_virt, scv, nvirt)
#undef QBLOCK
    free(first);
    free(sco);
    free(scv);
}

/* ---- Mulliken monopoles ------------------------------------------------ */

/* q_A = sum_{mu in A} sum_nu P S, dq_A = sum (P - P0) S.  mulliken.f90:11-66 */
void oracle_monopoles(int norb, int nat, const double *P, const double *P0, const double *S,
                      const int *orbs_per_atom, double *q, double *dq)
{
    int mu = 0;
    for (int A = 0; A < nat; ++A) {
        double qa = 0.0, dqa = 0.0;
        for (int k = 0; k < orbs_per_atom[A]; ++k, ++mu)
            for (int nu = 0; nu < norb; ++nu) {
                size_t o = (size_t)mu * norb + nu;
                qa += P[o] * S[o];
                dqa += (P[o] - P0[o]) * S[o];
            }
        q[A] = qa;
        dq[A] = dqa;
    }
}
