/*
 * dftbaby_b200 -- C ABI of the B200 (sm_100a) LR-TD-DFTB kernels.
 *
 * Conventions for every entry point:
 *   - array arguments are DEVICE pointers to row-major FP64 (int32 for index
 *     tables) memory owned by the caller; sizes are passed explicitly;
 *   - logical shapes follow the DFTBaby arrays they replace (e.g. q_ov has
 *     shape (Nat, nocc, nvirt), expansion vectors (nocc, nvirt, nvec));
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); work is
 *     enqueued asynchronously, nothing synchronises;
 *   - the return value is a status code (DFTB_OK or a negative DFTB_ERR_*);
 *     no entry point allocates device memory -- where scratch space is needed
 *     the caller passes a workspace whose size the *_workspace_size query
 *     returns.  The one exception is library state: dftb_apbv and
 *     dftb_trans_charges / dftb_trans_charges_diag (cuBLAS) and
 *     dftb_batched_eigh (cuSOLVER) create one handle per calling thread and
 *     device on first use, and those handles hold the libraries' own device
 *     memory until the process exits.  dftb_trans_charges_noalloc uses no
 *     library handle.
 *
 * Each function cites the DFTBaby interface it replaces (file:line inside the
 * DFTBaby project).
 */
#ifndef DFTBABY_B200_H
#define DFTBABY_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFTB_OK 0
#define DFTB_ERR_BAD_SIZE -1    /* a size argument is out of range            */
#define DFTB_ERR_NULL -2        /* a required pointer is NULL                 */
#define DFTB_ERR_CUDA -3        /* a CUDA launch or runtime call failed       */
#define DFTB_ERR_WORKSPACE -4   /* the workspace is smaller than required     */
#define DFTB_ERR_UNSUPPORTED -5 /* angular momentum or table layout not handled */
#define DFTB_ERR_NOT_CONVERGED -6 /* an iterative solve hit its iteration limit */

/* Library version and the CUDA error string of the last failing call on this
 * host thread (empty if none). */
const char *dftb_version(void);
const char *dftb_last_error(void);

/* Distances and directional cosines between all atoms.
 * Replaces slako.directional_cosines (DFTB/extensions/slako.f90:31-70):
 * r[i][j] = |R_i - R_j|, (x,y,z)[i][j] = (R_i - R_j)/r, and (0,0,1) when r = 0.
 * pos: (nat, 3). r, x, y, z: (nat, nat). */
int dftb_directional_cosines(int nat, const double *pos, double *r, double *x, double *y, double *z,
                             void *stream);

/* Slater-Koster overlap S and reference Hamiltonian H0.
 * Replaces slako.h0ands (DFTB/extensions/slako.f90:77-231), including the
 * B-spline evaluation of splines.f90:25-92 with its interval selection and its
 * clamp at the last knot.
 *   ind, typ, ls, ms : (norb) atom index, atom type, l, m of every orbital;
 *                      the orbitals of one atom are contiguous and atoms are
 *                      in increasing order;
 *   r, x, y, z       : (nat, nat) from dftb_directional_cosines;
 *   mprox            : (nat, nat) int, 1 where the atoms interact;
 *   orben            : (norb) on-site energies;
 *   tab_filled       : (npair, nsk) int; knots/coefs: (npair, nsk, npts);
 *   S, H0            : (norb, norb) outputs, every element written.
 * Only s and p orbitals (l <= 1) are implemented: elements that involve an
 * orbital with l > 1 are written as NaN.
 * Two geometries (slako.overlap12, slako.f90:576-687): call it on the union
 * of the atoms ordered [geometry 2, geometry 1] (atom indices of geometry 1
 * shifted by nat, r/x/y/z from dftb_directional_cosines of the union, mprox
 * all ones); rows norb.. and columns ..norb of S are overlap12's
 * <phi_mu(geometry 1)|phi_nu(geometry 2)>, evaluated in the same orientation. */
int dftb_h0_and_s(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                  const double *r, const double *x, const double *y, const double *z, const int *mprox,
                  const double *orben, int deg, const int *tab_filled, const double *S_knots,
                  const double *S_coefs, const double *H_knots, const double *H_coefs, int npair, int nsk,
                  int npts, double *S, double *H0, void *stream);

/* Dipole matrix D[c][mu][nu] = <mu| r_c |nu>, c = x, y, z (three planes).
 * Replaces slako.dipolematrix (DFTB/extensions/slako.f90:238-394); the
 * reference returns it as (norb, norb, 3) after rollaxis
 * (DFTB/SKMatrixElements.py:355-356).
 *   pos : (nat, 3); S: (norb, norb) from dftb_h0_and_s; D: (3, norb, norb). */
int dftb_dipole_matrix(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                       const double *r, const double *x, const double *y, const double *z, const double *pos,
                       const int *mprox, const double *S, int deg, const int *tab_filled_D,
                       const double *D_knots, const double *D_coefs, int npair, int nskd, int npts, double *D,
                       void *stream);

/* Gaussian gamma matrices.
 * Replaces GammaMatrix.gamma_atomwise with GammaGaussian / GammaGaussianLC
 * (DFTB/GammaApproximation.py:122-151, 210-243, 388-405):
 *   gamma[A][B]    = erf(R/sqrt(2(sA^2+sB^2)))/R,            gamma[A][A] = 1/(sqrt(pi) sA)
 *   gamma_lr[A][B] = erf(R/sqrt(2(sA^2+sB^2+Rlr^2/2)))/R,   gamma_lr[A][A] = 1/sqrt(pi(sA^2+Rlr^2/4))
 * sigma: (nat) Gaussian widths; r: (nat, nat).  gamma_lr may be NULL. */
int dftb_gamma_matrices(int nat, const double *r, const double *sigma, double r_lr, double *gamma,
                        double *gamma_lr, void *stream);

/* AO expansion G[mu][nu] = g[atom(mu)][atom(nu)] (gamma_AOwise's g0_AO,
 * DFTB/GammaApproximation.py:406-447, without the unused gradient array). */
int dftb_ao_expand(int norb, int nat, const int *ind, const double *g, double *G, void *stream);

/* SCC Hamiltonian H = H0 + 1/2 S o (e_mu + e_nu), e = gamma . dq per atom.
 * Replaces DFTB2._construct_h1 / _coulomb_hamiltonian and the sum
 * H = H0 + Hcoul (DFTB/DFTB2.py:668-717, 1023).
 * estat: (nat) output, the electrostatic potential gamma . dq. */
int dftb_scc_hamiltonian(int norb, int nat, const int *ind, const double *H0, const double *S,
                         const double *gamma, const double *dq, double *estat, double *H, void *stream);

/* Mulliken monopoles q_A = sum_{mu in A} sum_nu P S, dq_A = sum (P - P0) S.
 * Replaces mulliken.monopoles (DFTB/extensions/mulliken.f90:11-66).
 * P, P0, S: (norb, norb); orbs_per_atom: (nat); q, dq: (nat). */
int dftb_monopoles(int norb, int nat, const double *P, const double *P0, const double *S,
                   const int *orbs_per_atom, double *q, double *dq, void *stream);

/* Mulliken transition charges
 *   q^{pq}_A = 1/2 sum_{mu in A} (C_mu,p (S C)_mu,q + C_mu,q (S C)_mu,p)
 * for the occupied-occupied, occupied-virtual and virtual-virtual blocks.
 * Replaces tddftb.trans_charges (DFTB/extensions/tddftb.f90:12-112).
 *   orbs_occ: (norb, nocc), orbs_virt: (norb, nvirt), S: (norb, norb);
 *   q_oo: (nat, nocc, nocc), q_ov: (nat, nocc, nvirt), q_vv: (nat, nvirt, nvirt);
 *   any of the three outputs may be NULL to skip it;
 *   work: at least dftb_trans_charges_workspace_size() bytes.
 * The two S.C products run in cuBLAS (cublasDgemm, resolved at run time) when
 * libcublas can be loaded, otherwise in the library's own FP64 GEMM. */
size_t dftb_trans_charges_workspace_size(int norb, int nocc, int nvirt);
int dftb_trans_charges(int norb, int nat, int nocc, int nvirt, const double *orbs_occ, const double *orbs_virt,
                       const double *S, const int *orbs_per_atom, double *q_oo, double *q_ov, double *q_vv,
                       void *work, size_t work_bytes, void *stream);

/* Allocation-free variant of dftb_trans_charges (no counterpart in DFTBaby).
 * For callers that cannot allocate device memory where they need the charges:
 * hosts that reserve the GPU's memory up front in their own pool and forbid
 * further cudaMalloc, or bindings that only receive device pointers.  Same
 * arguments and results as dftb_trans_charges, without the workspace: the
 * scratch (S.C of both orbital blocks and per-atom orbital offsets) lives in a
 * fixed 8 MiB device array that each GPU loading the library holds until the
 * process exits.  Requests needing more than dftb_trans_charges_noalloc_max_bytes()
 * of scratch (dftb_trans_charges_workspace_size() > 8 MiB) return
 * DFTB_ERR_WORKSPACE and launch nothing, as do more than 65535 atoms.  The
 * first call on a device looks up the array's address for that device
 * (cudaGetSymbolAddress), so make it before any stream capture.  With CUDA's
 * lazy module loading (the default) the array is also committed on that device
 * only when this library's kernels are first used there, which may be this
 * first call: a host that reserves the GPU's memory for its own pool should
 * make one call (any size) before reserving it.  The cached address belongs
 * to the device's primary context and does not survive cudaDeviceReset.  All
 * calls on one device share the array: calls that may run concurrently on the
 * GPU race and must be serialised.  No device memory is allocated or freed. */
size_t dftb_trans_charges_noalloc_max_bytes(void);
int dftb_trans_charges_noalloc(int norb, int nat, int nocc, int nvirt, const double *orbs_occ,
                               const double *orbs_virt, const double *S, const int *orbs_per_atom, double *q_oo,
                               double *q_ov, double *q_vv, void *stream);

/* Diagonal transition charges q^{ii}_A and q^{aa}_A (the inputs of the
 * Lambda-2 diagnostic, DFTB/LR_TDDFTB.py:538-560), without the full blocks.
 *   q_ii: (nat, nocc), q_aa: (nat, nvirt); work as for dftb_trans_charges. */
int dftb_trans_charges_diag(int norb, int nat, int nocc, int nvirt, const double *orbs_occ,
                            const double *orbs_virt, const double *S, const int *orbs_per_atom, double *q_ii,
                            double *q_aa, void *work, size_t work_bytes, void *stream);

/* Hermitian TD-DFTB product for the singlet problem without long-range
 * correction, applied to nvec vectors at once:
 *   u = omega^2 o v + 4 sqrt(omega) o (q^T gamma q (sqrt(omega) o v))
 * Replaces Rv() inside Solver.HermitianDavidson (DFTB/Solver.py:431-444).
 *   gamma: (nat, nat); q_ov: (nat, nocc, nvirt); omega: (nocc, nvirt);
 *   vs, us: (nocc, nvirt, nvec); work: dftb_hermitian_rv_workspace_size(). */
size_t dftb_hermitian_rv_workspace_size(int nat, int nvec);
int dftb_hermitian_rv(int nat, int nocc, int nvirt, int nvec, const double *gamma, const double *q_ov,
                      const double *omega, const double *vs, double *us, void *work, size_t work_bytes,
                      void *stream);

/* (A+B).v and (A-B).v for nvec vectors, singlets, in the transition-charge
 * form of the reference:
 *   (A+B)v = omega v + 4 q_ov^T g q_ov v - K1 v - K2 v,   (A-B)v = omega v + K2 v - K1 v,
 *   K1 v = sum q_oo g_lr q_vv v   ((ij|ab) exchange),  K2 v = sum q_ov g_lr q_ov v  ((ib|ja) exchange);
 * with lc = 0 the exchange terms are skipped.
 * Replaces tddftb.apbv / tddftb.ambv (DFTB/extensions/tddftb.f90:114-287) and
 * Solver._ApBv / _AmBv (DFTB/Solver.py:583-635).
 *   g, g_lr: (nat, nat); q_oo, q_ov, q_vv as for dftb_trans_charges;
 *   omega: (nocc, nvirt); vs, us: (nocc, nvirt, nvec);
 *   work: dftb_apbv_workspace_size() bytes with lc = 1, and
 *   dftb_hermitian_rv_workspace_size() bytes with lc = 0.
 * The two q_ov contractions of the Coulomb term run in cuBLAS (cublasDgemm,
 * one handle per calling thread and device, bound to `stream`) when
 * libcublas.so.12 can be loaded at run time, otherwise in the library's own
 * FP64 GEMM; vs and us must not overlap. */
size_t dftb_apbv_workspace_size(int nat, int nocc, int nvirt, int nvec);
int dftb_apbv(int nat, int nocc, int nvirt, int nvec, int lc, const double *g, const double *g_lr,
              const double *q_oo, const double *q_ov, const double *q_vv, const double *omega, const double *vs,
              double *us, void *work, size_t work_bytes, void *stream);
int dftb_ambv(int nat, int nocc, int nvirt, int nvec, int lc, const double *g, const double *g_lr,
              const double *q_oo, const double *q_ov, const double *q_vv, const double *omega, const double *vs,
              double *us, void *work, size_t work_bytes, void *stream);

/* Davidson correction vectors: for c in [0, nnew),
 *   Q[:, c] = W[:, src[c]] / (w[state[c]] - omega),  where |w - omega| < 1e-6
 *   is replaced by 1e-6 * omega.
 * Replaces the preconditioning loops of Solver.HermitianDavidson and
 * Solver.nonHermitianDavidson (DFTB/Solver.py:530-539, 852-882).
 *   W: (nov, ldw) residual columns, omega: (nov), w: eigenvalue per state,
 *   src, state: (nnew) int32 column / state indices, Q: (nov, ldq). */
int dftb_davidson_precondition(int nov, int nnew, const double *W, int ldw, const int *src, const int *state,
                               const double *w, const double *omega, double *Q, int ldq, void *stream);

/* Residual update W[:, c] = AV[:, c] - lam[c] * X[:, c] for c < ncol and the
 * column norms |W[:, c]| (Solver.py:505-509, 823-832).
 *   AV, X, W: (nov, ld*) column blocks; lam: (ncol); norms: (ncol) output. */
int dftb_davidson_residual(int nov, int ncol, const double *AV, int ldav, const double *X, int ldx,
                           const double *lam, double *W, int ldw, double *norms, void *stream);

/* Split-precision BF16 product on the tcgen05 tensor cores (no counterpart in
 * DFTBaby; it carries the mixed-precision form of the long-range exchange
 * contractions of Solver._ApBv/_AmBv, DFTB/Solver.py:583-635):
 *   C(m, n) = alpha * sum_{s < nseg} sum_k A_s(m, k) B_s(n, k),  FP32 accumulation,
 * A_s: (M, K) and B_s: (N, K) K-major BF16, leading dimensions multiples of 8
 * elements, bases 16-byte aligned (A and B are host arrays of nseg device
 * pointers, nseg <= 3).  With X = X_hi + X_lo the three segments
 * (A_hi,B_hi), (A_hi,B_lo), (A_lo,B_hi) give ~2^-16 relative accuracy.
 * Epilogue: optional elementwise factor G (FP32, ldg), FP32 output C (ldc),
 * BF16 hi/lo outputs row-major (Ohi/Olo, ldo) and/or transposed (Thi/Tlo, ldt).
 * err: device int set non-zero if an internal wait timed out. */
int dftb_bf16x3_gemm(int M, int N, int K, int nseg, const void *const *A, int lda, const void *const *B, int ldb,
                     float alpha, const float *G, int ldg, float *C, int ldc, void *Ohi, void *Olo, int ldo,
                     void *Thi, void *Tlo, int ldt, int *err, void *stream);
/* Same product with two execution options: shared_split = 1 takes nseg = 2
 * pointers (A_hi, A_lo) and (B_hi, B_lo), loads the four tiles once per
 * K-block and accumulates hi.hi + hi.lo + lo.hi; ksplit > 1 splits the K range
 * over ksplit CTAs per output tile that add into C with atomics (C zeroed by the
 * caller; G and the BF16 outputs are then not allowed). */
int dftb_bf16x3_gemm_ex(int M, int N, int K, int nseg, int shared_split, int ksplit, const void *const *A, int lda,
                        const void *const *B, int ldb, float alpha, const float *G, int ldg, float *C, int ldc,
                        void *Ohi, void *Olo, int ldo, void *Thi, void *Tlo, int ldt, int *err, void *stream);
/* X (rows x cols, FP32 or FP64, optionally transposed and scaled) -> BF16
 * hi/lo pair with leading dimension ld; columns beyond the matrix are zeroed. */
int dftb_split_bf16(int rows, int cols, const float *X, int ldx, int transpose, void *hi, void *lo, int ld,
                    void *stream);
int dftb_split_bf16_f64(int rows, int cols, const double *X, int ldx, int transpose, double scale, void *hi,
                        void *lo, int ld, void *stream);
const char *dftb_tc_last_error(void);

/* FP64 product C = alpha * op(A) . op(B) + beta * C (row-major, op = transpose
 * when trans != 0) emulated on the int8 tensor cores (no counterpart in
 * DFTBaby; it carries the FP64 contractions of the SCC, DFTB2.py:1086-1266,
 * and of the FP64 exchange products, Solver.py:583-635).  Ozaki scheme II:
 * rows of op(A) and columns of op(B) are scaled by powers of two and rounded
 * to integers of b bits, b the largest with k 2^(2b) < P/2 (at most 53; P the
 * product of the first nmod of 16 coprime moduli <= 256), the integer product
 * is formed exactly from nmod int8 GEMMs of residues (int32 accumulation) and
 * recovered by the Chinese remainder theorem.  Each entry enters with b bits
 * relative to the largest magnitude of its row (column); nmod = 16 gives
 * b = 53 for every k <= 131071.  A row or column holding Inf or NaN gives NaN
 * in its row (column) of C.  work: dftb_ozaki_workspace_size bytes, 256-byte
 * aligned; err: device int set non-zero if an internal wait timed out.
 * Returns DFTB_ERR_BAD_SIZE for k > 131071 or nmod outside 8..16. */
size_t dftb_ozaki_workspace_size(int m, int n, int k, int nmod);
int dftb_ozaki_dgemm(int transa, int transb, int m, int n, int k, double alpha, const double *A, int lda,
                     const double *B, int ldb, double beta, double *C, int ldc, int nmod, void *work,
                     size_t work_bytes, int *err, void *stream);
/* The same product in two stages, for operands used in several products.
 * An operand is a K-major matrix Y (rows_total x k) in residue form (per-row
 * exponents and nmod int8 residue planes; dftb_ozaki_operand_size bytes,
 * 256-byte aligned).  dftb_ozaki_prepare fills rows [row0, row0 + rows) of
 * it from Y(r, c) = trans ? X[c][r] : X[r][c] (X row-major, ldx); the call
 * that fills the last rows also zeroes the padding rows, so an operand built
 * from several row blocks (a stacked matrix) is complete once every block is
 * prepared.  dftb_ozaki_product then forms
 *   C(i, j) = alpha * G(i, j) * sum_c A(i, c) B(j, c) + beta * C(i, j)
 * for i < m, j < n from two operands of the same k and nmod (G optional,
 * row-major ldg; work: dftb_ozaki_product_workspace_size bytes). */
size_t dftb_ozaki_operand_size(int rows, int k, int nmod);
int dftb_ozaki_prepare(int trans, int rows, int k, const double *X, int ldx, int nmod, void *operand, int rows_total,
                       int row0, void *stream);
size_t dftb_ozaki_product_workspace_size(int m, int n, int nmod);
int dftb_ozaki_product(int m, int n, int k, int nmod, const void *A, int rows_a, const void *B, int rows_b,
                       double alpha, const double *G, int ldg, double beta, double *C, int ldc, void *work,
                       size_t work_bytes, int *err, void *stream);
const char *dftb_ozaki_last_error(void);

/* Layout changes of (nov x m) column blocks of the Davidson solve (no
 * counterpart in DFTBaby, whose vectors are numpy arrays).
 * Y (cols x rows, leading dimension ldy) = X^T of a row-major FP64 X (rows x
 * cols, leading dimension ldx); cols <= 2097120. */
int dftb_transpose_f64(int rows, int cols, const double *X, int ldx, double *Y, int ldy, void *stream);
/* K1, K2 (nocc*nvirt x m, FP64, row-major) from the FP32 output Kall (m x
 * 2 nvirt x nocc) of the last launch of the tensor-core exchange, whose rows
 * 2a and 2a + 1 hold K1^T and K2^T of product column c:
 *   K_y[(i nvirt + a) m + c] = Kall[c][2a + y][i];  nvirt <= 65535. */
int dftb_exchange_unpack(int m, int nvirt, int nocc, const float *Kall, double *K1, double *K2, void *stream);

/* General FP64 product C = alpha * op(A) . op(B) + beta * C on row-major
 * matrices (op = transpose when trans != 0), the contraction engine behind the
 * entry points above, exported for the host-side solver. */
int dftb_dgemm(int transa, int transb, int m, int n, int k, double alpha, const double *A, int lda,
               const double *B, int ldb, double beta, double *C, int ldc, void *stream);

/* ---- analytic gradients (DFTB/ExcGradients.py) ------------------------------ */

/* Dense gradients of S and H0.
 * Replaces slako.gradients_h0ands (DFTB/extensions/slako.f90:402-569, called
 * from ExcGradients._gradients_H0andS_f90, ExcGradients.py:151-177) with its
 * spline values from splev_uniform and radial derivatives from FITPACK splder
 * (splines.f90:96-115).  Arguments as dftb_h0_and_s (without orben);
 * gradS, gradH0: (3 nat, norb, norb), element [3j+c][mu][nu] (and its mirror
 * [3j+c][nu][mu]) = derivative of S_mu,nu with respect to coordinate c of the
 * atom j of nu, in the orientation of the ordered pair (mu, nu); zero
 * elsewhere.  norb <= 65535. */
int dftb_gradients_h0_and_s(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                            const double *r, const double *x, const double *y, const double *z, const int *mprox,
                            int deg, const int *tab_filled, const double *S_knots, const double *S_coefs,
                            const double *H_knots, const double *H_coefs, int npair, int nsk, int npts,
                            double *gradS, double *gradH0, void *stream);

/* Contraction of the same derivatives with adjoint matrices, without forming
 * the dense tensors:
 *   grad[3j+c] = sum_{nu on j} sum_{mu on other atoms} dS_mu,nu/dR_j,c XS[mu][nu]
 *                                                    + dH0_mu,nu/dR_j,c XH[mu][nu].
 * With XS = X + X^T this equals sum_{mu,nu} gradS[3j+c][mu][nu] X[mu][nu], the
 * np.tensordot(gradS, X, axes=([1,2],[0,1])) of ExcGradients.py:501-506, 704-705.
 * XS or XH may be NULL (term skipped).  grad: (3 nat), overwritten. */
int dftb_sk_gradient_contract(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                              const double *r, const double *x, const double *y, const double *z, const int *mprox,
                              int deg, const int *tab_filled, const double *S_knots, const double *S_coefs,
                              const double *H_knots, const double *H_coefs, int npair, int nsk, int npts,
                              const double *XS, const double *XH, double *grad, void *stream);

/* Atom-pair gradient terms:
 *   grad[3i+c] = sum_{j != i} [ g1(R_ij) Yg[i][j] + g1lr(R_ij) Ylr[i][j] + Vrep'(R_ij) ] (R_i - R_j)_c / R_ij
 * with g1, g1lr the radial derivatives of the Gaussian gamma and long-range
 * gamma (GammaGaussian.g_deriv, GammaGaussianLC.g_deriv,
 * GammaApproximation.py:141-148, 234-238; sigma per atom, r_lr the long-range
 * radius) and Vrep' the derivative of the repulsive potential of the pair
 * (gradient_Vrep, ExcGradients.py:181-211).  With Y = A + A^T for atom-block
 * sums A this is the contraction of GammaMatrix.gamma_AOwise's g1_AO / g1_AT
 * (GammaApproximation.py:406-447) with A.  Yg, Ylr: (nat, nat) or NULL;
 * vrep_knots / vrep_coefs: (npair, nknots) cubic FITPACK splines, pair index
 * tmax*(tmax+1)/2 + tmin of the atom types atype (nat), vrep_dmax (npair) the
 * last grid point (Vrep = 0 from there on), or vrep_knots = NULL to skip the
 * repulsive term.  grad: (3 nat), overwritten. */
int dftb_pair_gradients(int nat, const double *pos, const int *atype, const double *sigma, double r_lr,
                        const double *Yg, const double *Ylr, const double *vrep_knots, const double *vrep_coefs,
                        const double *vrep_dmax, int nknots, double *grad, void *stream);

/* Repulsive energy per atom, e_atom[i] = 1/2 sum_{j != i} Vrep(R_ij); the sum
 * over atoms is DFTB2.getRepulsiveEnergy (DFTB2.py:2339-2359).  Tables as in
 * dftb_pair_gradients. */
int dftb_repulsive_energy(int nat, const double *pos, const int *atype, const double *vrep_knots,
                          const double *vrep_coefs, const double *vrep_dmax, int nknots, double *e_atom,
                          void *stream);

/* Error string of the last failing gradient entry point on this host thread. */
const char *dftb_grad_last_error(void);

/* ---- learned Davidson guess: MLP element-wise kernels ------------------------
 * No counterpart in DFTBaby: the small network that scores excitation pairs
 * for the initial Davidson vectors and corrects the diagonal preconditioner.
 * Its matrix products run through dftb_bf16x3_gemm_ex (one BF16 segment, FP32
 * accumulation); these kernels do the work in between.  Activations and
 * weight copies are BF16 (passed as void *), everything else FP32; row-major. */

/* H = relu(Z + b) for ns samples x nh units; H (ldh) and, unless HT is NULL,
 * H^T (nh x ns, ldht). */
int dftb_mlp_bias_relu(int ns, int nh, const float *Z, int ldz, const float *b, void *H, int ldh, void *HT, int ldht,
                       void *stream);
/* dZ = G o (H > 0): dZ (optional, ldz) and dZ^T (nh x ns, lddzt); db += column sums of dZ. */
int dftb_mlp_relu_backward(int ns, int nh, const float *G, int ldg, const void *H, int ldh, void *dZ, int lddz,
                           void *dZT, int lddzt, float *db, void *stream);
/* Y = Z[:, :no] + b (ns x no, FP32).  With targets T (ns x no), sample weights m (ns)
 * and output weights wout (no): loss += sum wout m (Y - T)^2 * inv_norm (FP64 scalar),
 * dY = 2 wout m (Y - T) inv_norm into dYp (ns x lddy) and rows 0..no-1 of dYT
 * (lddyt), db += column sums of dY.  T = NULL: inference only.  no <= 8. */
int dftb_mlp_output(int ns, int no, const float *Z, int ldz, const float *b, const float *T, const float *m,
                    const float *wout, float inv_norm, float *Y, void *dYp, int lddy, void *dYT, int lddyt, float *db,
                    double *loss, void *stream);
/* One Adam step (bias-corrected for step >= 1, decoupled weight decay) on FP32
 * master weights W (rows x cols) with moments m1, m2; refreshes the BF16 copies
 * Wb (row-major) and WbT (transposed) where given. */
int dftb_mlp_adam(int rows, int cols, float *W, const float *G, float *m1, float *m2, float lr, float beta1,
                  float beta2, float eps, int step, float weight_decay, void *Wb, int ldwb, void *WbT, int ldwbt,
                  void *stream);
const char *dftb_mlp_last_error(void);

/* ---- batched symmetric eigensolver --------------------------------------------
 * No counterpart in DFTBaby, which calls LAPACK one matrix at a time
 * (DFTB2.py:1086, Solver.py:486, 772).  Eigenvalues (ascending) and eigenvectors of
 * batch symmetric n x n FP64 matrices stored contiguously in A (only the lower
 * triangle of each row-major block is read, as torch.linalg.eigh reads it); A is overwritten by the eigenvectors in column-major order (eigenvector j
 * is row j of each row-major n x n block), W receives batch x n eigenvalues, info
 * batch status words.  Runs cuSOLVER's cusolverDnXsyevBatched, resolved at run
 * time: DFTB_ERR_UNSUPPORTED when the loaded cuSOLVER lacks it or refuses the size.
 * work: dftb_batched_eigh_workspace_size() bytes of device memory. */
int dftb_batched_eigh_workspace_size(int n, int batch, size_t *bytes);
int dftb_batched_eigh(int n, int batch, double *A, double *W, void *work, size_t work_bytes, int *info, void *stream);
const char *dftb_eigh_last_error(void);

/* ---- the fused device solve ------------------------------------------------------
 * Replaces the Davidson branch of LR_TDDFTB._solve_lr_equations (DFTB/LR_TDDFTB.py:403-527)
 * for the problem without long-range correction, Solver.HermitianDavidson
 * (DFTB/Solver.py:404-578): R T = Omega^2 T with R = omega^2 + 4 sqrt(omega) q_ov^T gamma q_ov sqrt(omega).
 * An opaque handle owns the expansion space, its products, the projected matrix and the previous
 * solution (the warm start of the next solve, Solver.py:461-478), in device memory the caller
 * provides once: dftb_solver_workspace_size() bytes, or 0 when the sizes are out of range or cuBLAS /
 * cuSOLVER (resolved at run time) are missing.  The handle also holds one cuBLAS and one cuSOLVER
 * handle; dftb_solver_destroy releases them (not the workspace).  One handle per host thread: calls
 * on the same handle must not overlap.
 *   max_iter bounds the Davidson iterations of every solve (the space holds nstates (max_iter + 1)
 *   vectors at most, and at most 46340);
 *   gamma (nat, nat), q_ov (nat, nocc, nvirt), omega (nocc, nvirt): as for dftb_hermitian_rv;
 *   conv: the residual-norm threshold of every state (DFTBaby's diag_conv); maxiter <= max_iter;
 *   warm_start != 0 starts from the previous solve's X+Y (ignored before the first solve or after
 *   dftb_solver_reset);
 *   outputs (device): Omega (nstates), C, XmY, XpY (nstates, nocc, nvirt), each but Omega may be NULL;
 *   iterations (host, may be NULL): Davidson iterations taken.
 * Returns DFTB_ERR_NOT_CONVERGED (DFTBaby's ExcitedStatesNotConverged) when maxiter is reached.
 * The call synchronises the stream once per iteration to read the residual norms. */
typedef struct dftb_solver dftb_solver;
size_t dftb_solver_workspace_size(int nat, int nocc, int nvirt, int nstates, int max_iter);
int dftb_solver_create(int nat, int nocc, int nvirt, int nstates, int max_iter, void *work, size_t work_bytes,
                       dftb_solver **out);
int dftb_solver_solve_hermitian(dftb_solver *s, const double *gamma, const double *q_ov, const double *omega,
                                double conv, int maxiter, int warm_start, double *Omega, double *C, double *XmY,
                                double *XpY, int *iterations, void *stream);
int dftb_solver_reset(dftb_solver *s);
int dftb_solver_destroy(dftb_solver *s);
const char *dftb_solver_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DFTBABY_B200_H */
