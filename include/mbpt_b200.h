/*
 * libmbpt_b200 -- C ABI of the B200 (sm_100a) space-time ISDF RPA/GW route.
 *
 * Conventions
 *   - Every array argument named *_dev is a DEVICE pointer owned by the
 *     caller; *_host arguments are small host arrays read during the call.
 *   - Matrices are row-major FP64 unless stated; complex arrays are
 *     interleaved (re, im) FP64.
 *   - Calls are stream-ordered on `stream` (a cudaStream_t, NULL = legacy
 *     default stream) and take their scratch from the caller's `workspace`
 *     of `ws_bytes` bytes, sized by the matching *_workspace_bytes query.
 *     The FP64 products and the Cholesky/LU factorisations go through
 *     cuBLAS/cuSOLVER handles created on first use (per host thread);
 *     mbpt_dyson (and mbpt_rpa_energy through it) synchronises `stream`
 *     once to read the factorisations' info words.
 *   - The return value is an mbpt_status. Errors found on the device (a
 *     bounded wait that ran out) are written to the int at `err_dev`
 *     (zeroed by the caller before the call, read after it); NULL skips.
 *   - mode MBPT_MODE_FP64 runs every product in FP64 (cuBLAS DGEMM, the plain
 *     GPU path); MBPT_MODE_MIXED runs the N^3 products on the tcgen05 tensor
 *     cores as split (3-term) products with FP32 accumulation: BF16 pairs for
 *     the Coulomb-side products, TF32 pairs for G_occ / G_virt and for the
 *     inverse of the Dyson step. The tau <-> omega transforms, the
 *     Cholesky/log-det, the quadrature sums and the QP root search are FP64
 *     in both modes. MBPT_MODE_FP64_INT8 is FP64-accurate like
 *     MBPT_MODE_FP64, with the forward sweeps' products and the Cholesky
 *     updates of the Dyson step emulated on the int8 tensor cores (the Ozaki
 *     scheme, 8 seven-bit digits per operand: mbpt_dgemm_ozaki); accepted
 *     wherever MBPT_MODE_FP64 is.
 *   - The reverse sweeps (mbpt_chi0_backward, mbpt_sigma_backward,
 *     mbpt_dyson_backward) take the same two FP64 modes: native DGEMMs or
 *     the emulated product, which also forms the symmetric products' upper
 *     tiles only and the G branches' adjoints straight from its epilogue.
 *     The FP64 products of the rows beside the route that take no mode
 *     (mbpt_three_index_slices and its backward, mbpt_cd_integral_backward,
 *     the MO collocation of mbpt_sigma_ao) run on the emulated product;
 *     MBPT_FP64_GEMM=cublas in the environment keeps cuBLAS DGEMMs there.
 *   - The emulation's error is ~5e-15 of the operands' scale per product,
 *     about FP64 rounding, but it changes erratically with the inputs where
 *     rounding changes smoothly: a tau <-> omega transform whose weights
 *     cancel at 1e8 (the 16-point grids) amplifies it ~100x more, so FP64
 *     is the mode for such grids.
 *
 * Symbols: X (M x norb) collocation of the MO basis on the interpolation
 * points, columns [0, nocc) occupied; D (M x naux) Coulomb factor, Z = D D^T;
 * eps (norb) orbital energies; mu the chemical potential inside the gap.
 */
#ifndef MBPT_B200_H
#define MBPT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum mbpt_status {
  MBPT_OK = 0,
  MBPT_ERR_SHAPE = 1,       /* inconsistent or unsupported sizes */
  MBPT_ERR_NOT_SPD = 2,     /* 1 - chi0 not positive definite at some frequency */
  MBPT_ERR_NONFINITE = 3,   /* a non-finite value where a finite one is needed */
  MBPT_ERR_NO_ROOT = 4,     /* a QP equation without a root (per-state flag) */
  MBPT_ERR_TIMEOUT = 5,     /* a bounded device-side wait ran out */
  MBPT_ERR_CUDA = 6,        /* a CUDA runtime / library call failed */
  MBPT_ERR_WORKSPACE = 7,   /* workspace smaller than the query returned */
  MBPT_ERR_UNSUPPORTED = 8  /* device or option not supported */
};

enum mbpt_mode { MBPT_MODE_FP64 = 0, MBPT_MODE_MIXED = 1, MBPT_MODE_FP64_INT8 = 2 };

int mbpt_abi_version(void);
const char *mbpt_status_string(int status);
/* 1 when `device` is an sm_100 part this library was built for, else 0 */
int mbpt_device_supported(int device);

/* Instrumentation (no counterpart in MBPTcode, which has no device code):
 * the number of this library's kernels launched by the process so far, and
 * CUDA-event timing of the tensor-core engine's launches. mbpt_gemm_timing
 * with enable = 1 starts recording on the launching streams (enable = 2: all
 * but category 7, whose many small launches the event pairs would slow down);
 * a call with
 * non-NULL total_ms/launches (8 entries, indexed by epilogue kind: 0 split
 * store, 1 FP32 store, 2 Hadamard, 3 self-energy Hadamards, 4 row
 * contraction, 5 FP32 accumulate, 6 TF32-pair store; 7 collects the TF32
 * products of mbpt_dyson's inverse whatever their epilogue) waits for the
 * recorded launches, returns
 * their summed milliseconds and counts, and resets them. */
long long mbpt_launch_count(void);
int mbpt_gemm_timing(int enable, double *total_ms, long long *launches);

/* Self-test of failure detection (no counterpart in MBPTcode): one thread
 * waits, with the tensor-core engine's barrier-wait routine, on a
 * shared-memory mbarrier that it completes first (arrive = 1) or that nothing
 * completes (arrive = 0). The wait gives up after limit_us microseconds
 * (1 ... 1e6) and writes MBPT_ERR_TIMEOUT to *err_dev; the kernel then returns
 * normally, so the context stays usable. The engine's own waits give up the
 * same way after 4 s. */
int mbpt_wait_selftest(int arrive, int limit_us, int *err_dev, void *stream);

/* ---- chi0 sweep ---------------------------------------------------------
 * Replaces LinearResponse/space_time.py:607-651 chi0_imaginary_frequency
 * (with :478-530 polarizability_projected_tau per tau point and :533-560
 * polarizability_projected_sweep when proj_dev is given):
 *   proj(tau_k)  = -2 D^T [G_occ(tau_k) o G_virt(tau_k)] D
 *   chi0(i w_f)  = sum_k cosft_wt[f, k] proj(tau_k)
 * G_occ(tau) = X_o diag(e^{(eps_i - mu) tau}) X_o^T,
 * G_virt(tau) = X_v diag(e^{-(eps_a - mu) tau}) X_v^T.
 * chi0_dev: (nfreq, naux, naux) output; proj_dev: optional (ntau, naux, naux)
 * FP64 copy of proj(tau) (NULL: not kept).
 * tau_host (ntau), cosft_wt_host (nfreq x ntau). */
size_t mbpt_chi0_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux,
                                 int ntau, int mode);
int mbpt_chi0_sweep(const double *X_dev, int64_t M, int64_t norb, int64_t nocc,
                    const double *eps_dev, double mu, const double *D_dev, int64_t naux,
                    const double *tau_host, int ntau, const double *cosft_wt_host, int nfreq,
                    int mode, double *chi0_dev, double *proj_dev, void *workspace,
                    size_t ws_bytes, int *err_dev, void *stream);

/* ---- Dyson step and dielectric log-determinant ---------------------------
 * Replaces LinearResponse/space_time.py:956-968 dyson_screening (per
 * frequency, correlation=True) and :1073-1097 dielectric_log_determinant,
 * by a Cholesky factorisation of 1 - chi0 at each frequency (FP64). From
 * four frequencies on, one batched factorisation of all of them, whose
 * trailing updates run on the int8 tensor cores (the Ozaki scheme,
 * FP64-accurate) in MBPT_MODE_MIXED and as native FP64 DGEMMs in
 * MBPT_MODE_FP64 (the environment variable MBPT_DYSON_OZAKI=1 or =0 forces
 * either).
 * chi0_dev (nfreq, naux, naux): in chi0; out W - I = [1 - chi0]^-1 - 1 when
 * want_w, else the Cholesky factors.
 * logdet_dev, trace_dev (nfreq): log det(1 - chi0) and tr chi0.
 * info_host (nfreq): 0, or i > 0 when 1 - chi0 is not positive definite (its
 * log|det| and inverse then come from an LU factorisation and sign_host[f]
 * is the determinant's sign); the call then returns MBPT_ERR_NOT_SPD after
 * finishing every frequency. info_host/sign_host may be NULL.
 * mode: the factorisation and log-determinant are FP64 either way; the inverse
 * W = L^-T L^-1 is formed from the FP64 factor by cuBLAS level-3 products
 * (MBPT_MODE_FP64) or, with MBPT_MODE_MIXED, by TF32x3 tensor-core products
 * (the triangular inverse's off-diagonal blocks and L^-T L^-1): a few 2^-22
 * absolute on W - I, whose entries are bounded by 1. */
size_t mbpt_dyson_workspace_bytes(int64_t naux, int nfreq, int mode);
int mbpt_dyson(double *chi0_dev, int64_t naux, int nfreq, int want_w, int mode,
               double *logdet_dev, double *trace_dev, int *info_host, int *sign_host,
               void *workspace, size_t ws_bytes, int *err_dev, void *stream);
/* The same step without a host wait (no synchronisation of the caller's
 * stream): every frequency's inverse is issued from its Cholesky factor and
 * its info word lands in info_dev (nfreq ints on the device). A nonzero word
 * marks a frequency where 1 - chi0 is not positive definite: its W - I and
 * log-determinant are then not valid, and the caller repeats the step (and
 * what it fed) with mbpt_dyson, which takes such a frequency through LU. The
 * workspace is mbpt_dyson_workspace_bytes'. */
int mbpt_dyson_deferred(double *chi0_dev, int64_t naux, int nfreq, int want_w, int mode,
                        double *logdet_dev, double *trace_dev, int *info_dev, void *workspace,
                        size_t ws_bytes, int *err_dev, void *stream);

/* ---- dRPA correlation energy ----------------------------------------------
 * Replaces LinearResponse/space_time.py:1100-1183
 * rpa_correlation_energy_space_time (gas phase, serial):
 *   E_c = (1/2pi) sum_f omega_weights[f] [log det(1 - chi0_f) + tr chi0_f].
 * e_c_dev: one FP64 output. proj_dev optional as in mbpt_chi0_sweep.
 * logdet/trace of each frequency are left in the workspace head. */
size_t mbpt_rpa_energy_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux,
                                       int ntau, int nfreq, int mode);
int mbpt_rpa_energy(const double *X_dev, int64_t M, int64_t norb, int64_t nocc,
                    const double *eps_dev, double mu, const double *D_dev, int64_t naux,
                    const double *tau_host, int ntau, const double *cosft_wt_host,
                    const double *omega_weights_host, int nfreq, int mode, double *e_c_dev,
                    double *proj_dev, int *info_host, void *workspace, size_t ws_bytes,
                    int *err_dev, void *stream);

/* E_c = (1/2pi) sum_f w_f [logdet_f + trace_f], summed in frequency order
 * (LinearResponse/space_time.py:1158-1182), from mbpt_dyson's outputs;
 * omega_weights_dev (nfreq), e_c_dev one FP64 output. */
int mbpt_energy_sum(const double *logdet_dev, const double *trace_dev,
                    const double *omega_weights_dev, int nfreq, double *e_c_dev, void *stream);

/* ---- tau <-> omega transform (FP64) --------------------------------------
 * Replaces GW/imaginary_time.py:181-195 _transform_screened and the
 * frequency fold of LinearResponse/space_time.py:854-905 / the adjoint's
 * gradients/rpa/space_time_adjoint.py:440-454:
 *   out[j] = sum_k w[j, k] in[k],   in (K, n, n), out (J, n, n), w_dev (J x K). */
int mbpt_transform(const double *in_dev, int K, int64_t n, const double *w_dev, int J,
                   double *out_dev, void *stream);
/* The same transform added onto out: out[j] += sum_k w[j, k] in[k]. One
 * frequency block's share of W(tau) in the blocked screening of
 * GW/imaginary_time.py:230-348 (`screened_interaction_tau_blocked`,
 * freq_block), which holds chi0 for a block of frequencies only. */
int mbpt_transform_acc(const double *in_dev, int K, int64_t n, const double *w_dev, int J,
                       double *out_dev, void *stream);

/* ---- self-energy branch sums --------------------------------------------
 * Replaces GW/imaginary_time.py:403-533 self_energy_matrix_imaginary_time
 * followed by :581-587 sigma_ao_to_mo_diagonal (X_ao = X, mo_coeff = I),
 * in the diagonal form of :39-92 SigmaPairs.add: for each tau_k
 *   Zt = D Wt(tau_k) D^T,
 *   branch[0,k,s] = +sum_PQ X[P,p] (G_occ(tau_k) o Zt)_PQ X[Q,p]
 *   branch[1,k,s] = -sum_PQ X[P,p] (G_virt(tau_k) o Zt)_PQ X[Q,p],
 * p = states[s]. Wt_dev (ntau, naux, naux), or NULL for W = I at every tau
 * (Zt = D D^T, the bare Coulomb factor: with tau = 0 the lesser branch is
 * then -Sigma_x,pp, the exchange diagonal); states_dev (nstates) int64;
 * branch_dev (2, ntau, nstates) output. */
size_t mbpt_sigma_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux,
                                  int ntau, int nstates, int mode);
int mbpt_sigma_branch_sums(const double *X_dev, int64_t M, int64_t norb, int64_t nocc,
                           const double *eps_dev, double mu, const double *D_dev,
                           int64_t naux, const double *Wt_dev, const double *tau_host,
                           int ntau, const int64_t *states_dev, int nstates, int mode,
                           double *branch_dev, void *workspace, size_t ws_bytes, int *err_dev,
                           void *stream);

/* Sigma_c(i w_p) = -1/2 [C (S^> + S^<) + i S (S^> - S^<)]
 * (GW/imaginary_time.py:525-532), C_dev/S_dev (npade x ntau);
 * sigma_dev (nstates, npade) complex interleaved. */
int mbpt_sigma_frequency(const double *branch_dev, int ntau, int nstates, const double *C_dev,
                         const double *S_dev, int npade, double *sigma_dev, void *stream);

/* ---- Pade continuation and QP roots --------------------------------------
 * Replaces GW/qp_solve.py:575-695 finish_qp (its per-state loop),
 * :529-558 solve_qp_from_imaginary_axis, analytic_continuation.py:64-89
 * PadeFit and Solvers/qp_equation.py:1353-1393
 * solve_qp_equation_pole_strength, for all states at once:
 *   root of w = eps_anchor[p] + xc[s] + Re Sigma_c(w), largest Z.
 * sigma_dev (nstates, npade) complex on the positive branch;
 * pade_freq_host (npade); eps_anchor_dev (norb); xc_dev (nstates) or NULL
 * (zero static term); warm_dev (nstates) predicted roots or NULL.
 * flags bits: 1 quasiparticle (Z > 1/2), 2 no root (root NaN),
 * 4 Z outside (0, 1], 8 Pade ordering failed, 16 warm start accepted,
 * 32 bracket list overflow. evals: Sigma evaluations per state. */
int mbpt_qp_solve(const double *sigma_dev, const double *pade_freq_host, int npade,
                  const double *eps_anchor_dev, const double *xc_dev,
                  const int64_t *states_dev, int nstates, int64_t nocc, double mu, int greedy,
                  const double *warm_dev, double *roots_dev, double *z_dev, int *flags_dev,
                  int *evals_dev, void *workspace, size_t ws_bytes, void *stream);

/* Re Sigma_c at real frequencies from the same continuation
 * (analytic_continuation.py:25-31 pade_eval on each state's PadeFit):
 * out_dev[s, q] = Re Sigma_c(query_dev[s, q]) for the nstates x nq query
 * frequencies (Hartree); NaN for a state whose greedy ordering failed.
 * Used for the features of the learned QP warm start (Sigma_c at eps +- 0.1). */
int mbpt_pade_eval(const double *sigma_dev, const double *pade_freq_host, int npade,
                   const int64_t *states_dev, int nstates, int64_t nocc, double mu, int greedy,
                   const double *query_dev, int nq, double *out_dev, void *workspace,
                   size_t ws_bytes, void *stream);

/* ---- reverse sweep of the polarizability ---------------------------------
 * Replaces gradients/rpa/space_time_adjoint.py:136-218
 * polarizability_backward: for an adjoint proj_bar (ntau, naux, naux) of
 * proj(tau), accumulates eps_bar (norb), X_bar (M x norb), D_bar (M x naux),
 * recomputing G_occ(tau), G_virt(tau) per tau point (nothing is stored
 * across tau). The outputs are overwritten. */
size_t mbpt_chi0_backward_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux,
                                          int mode);
int mbpt_chi0_backward(const double *proj_bar_dev, const double *X_dev, int64_t M,
                       int64_t norb, int64_t nocc, const double *eps_dev, double mu,
                       const double *D_dev, int64_t naux, const double *tau_host, int ntau,
                       int mode, double *eps_bar_dev, double *X_bar_dev, double *D_bar_dev,
                       void *workspace, size_t ws_bytes, int *err_dev, void *stream);

/* chi0_bar(f) = (w_f / 2pi) [I - (1 - chi0_f)^-T] from W - I (the Dyson
 * output): gradients/rpa/space_time_adjoint.py:528-539 (gas phase).
 * Overwrites w_minus_i_dev (nfreq, naux, naux) in place; omega_weights_dev
 * (nfreq). */
int mbpt_energy_adjoint_seed(double *w_minus_i_dev, int64_t naux, int nfreq,
                             const double *omega_weights_dev, void *stream);

/* The self-energy adjoint: gradients/rpa/space_time_adjoint.py:795-875
 * (`selfenergy_diag_backward`), its per-tau part :836-856 and the bra
 * slices' share :866-871. For the branch adjoints sl_bar, sg_bar (ntau x
 * nstates, device; the reverse of the tau -> omega weights :830-833, formed
 * by the caller) of Sigma^<, Sigma^> at the time points tau_host, on W(tau)
 * = Wt_dev (ntau, naux, naux; symmetric), it overwrites eps_bar (norb),
 * X_bar (M x norb), D_bar (M x naux) with the self-energy sweep's share and
 * writes Wt_bar_dev (ntau, naux, naux), which the Dyson and chi0 reverses
 * (mbpt_dyson_backward, mbpt_transform, mbpt_chi0_backward) take on.
 * states_dev: nstates int64 orbital indices. mode: MBPT_MODE_FP64 or
 * MBPT_MODE_FP64_INT8. */
size_t mbpt_sigma_backward_workspace_bytes(int64_t M, int64_t norb, int64_t nocc,
                                           int64_t naux, int nstates);
int mbpt_sigma_backward(const double *X_dev, int64_t M, int64_t norb, int64_t nocc,
                        const double *eps_dev, double mu, const double *D_dev, int64_t naux,
                        const double *tau_host, int ntau, const double *Wt_dev,
                        const int64_t *states_dev, int nstates, const double *sl_bar_dev,
                        const double *sg_bar_dev, int mode, double *eps_bar_dev,
                        double *X_bar_dev,
                        double *D_bar_dev, double *Wt_bar_dev, void *workspace,
                        size_t ws_bytes, int *err_dev, void *stream);

/* The self-energy's two branches as full AO matrices: per time point tau_k
 *   Sigma^<(tau_k) = X_ao^T (G_occ(tau_k) o Zt_k) X_ao,
 *   Sigma^>(tau_k) = -X_ao^T (G_virt(tau_k) o Zt_k) X_ao,
 * G from the MO collocation X_ao mo_coeff (occupied/virtual split at nocc,
 * eps - mu), Zt_k = D Wt_k D^T: GW/imaginary_time.py:403-533
 * (`self_energy_matrix_imaginary_time`, before its tau -> omega fold).
 * out_dev: (2, ntau, nao, nao), lesser branch first, FP64. mode: FP64 (or
 * its int8 emulation): DGEMMs and Hadamard passes; MBPT_MODE_MIXED: the
 * split BF16 products of the self-energy sweep (U = D Wt, one pass forming
 * G_occ o Zt and G_virt o Zt, X_ao^T H X_ao as two products, the last one
 * stored in FP64 by its epilogue), ~1e-5 relative. */
size_t mbpt_sigma_ao_workspace_bytes(int64_t M, int64_t nao, int64_t norb, int64_t nocc,
                                     int64_t naux, int mode);
int mbpt_sigma_ao(const double *X_ao_dev, int64_t M, int64_t nao, const double *mo_coeff_dev,
                  int64_t norb, int64_t nocc, const double *eps_dev, double mu,
                  const double *D_dev, int64_t naux, const double *Wt_dev,
                  const double *tau_host, int ntau, int mode, double *out_dev,
                  void *workspace, size_t ws_bytes, int *err_dev, void *stream);

/* ---- contour deformation (GW/contour_deformation.py), FP64 ----------------
 * Three-index slices B_s = D^T diag(X[:, p_s]) X of the states p_s
 * (LinearResponse/space_time.py:804-815 `three_index_slice`), written to
 * B_dev as (nstates, naux, norb) row-major; states_host: nstates int64. */
size_t mbpt_three_index_slices_workspace_bytes(int64_t M, int64_t norb);
int mbpt_three_index_slices(const double *X_dev, int64_t M, int64_t norb, const double *D_dev,
                            int64_t naux, const int64_t *states_host, int nstates,
                            double *B_dev, void *workspace, size_t ws_bytes, void *stream);

/* (1 - chi0) y = b from mbpt_dyson's Cholesky factor (want_w = 0: the
 * column-major lower factor L of 1 - chi0 in the chi0 slice), in place on b
 * (column-major n x nrhs): the contour residues' W(freq) b
 * (GW/real_screening.py:147-150 `LaplaceRealScreening.apply`, which solves
 * against 1 - chi0), without forming W. FP64. */
int mbpt_chol_solve(const double *L_dev, int64_t n, double *b_dev, int nrhs, void *stream);

/* The contour deformation's imaginary-axis term and its slope at nq points
 * (state slot slot_dev[j], real frequency omega_dev[j]): value[j] =
 * -(1/pi) sum_(k,q) c_k(omega - eps_q) wc[slot][k][q] with the Gauss-Legendre
 * weights of the Lorentzian kernel and the closed-form correction of its
 * singular part (wc(0) = e1 wc[k1] + e2 wc[k2], model a^2 / (a^2 + nu^2)),
 * slope[j] its omega derivative (GW/contour_deformation.py:150-202
 * `cd_integral_weights` contracted as in :310-373 `sigma_cd`,
 * `sigma_cd_slope`). wc_dev: (nslots, nfreq, norb) FP64. */
int mbpt_cd_integral_terms(const double *wc_dev, int nslots, int nfreq, int64_t norb,
                           const double *eps_dev, const double *nu_dev, const double *nu_w_dev,
                           int k1, int k2, double e1, double e2, double a, double on_tol,
                           const int *slot_dev, const double *omega_dev, int64_t nq,
                           double *value_dev, double *slope_dev, void *stream);
/* err[i] = max over the pair energies d and both signs of y = d -+ freq[i] of
 * |y sum_k tau_w[k] e^(-y tau[k]) - 1|, infinity where some y <= 0: whether
 * the imaginary-time grid carries a real frequency
 * (LinearResponse/space_time.py:908-931 `laplace_representation_error`). */
int mbpt_laplace_representation_error(const double *d_dev, int64_t npairs,
                                       const double *tau_dev, const double *tau_w_dev, int ntau,
                                       const double *freq_dev, int64_t nf, double *err_dev,
                                       void *stream);

/* The explicit particle-hole response of one block (continuation 'cd'),
 * LinearResponse/space_time.py:934-953 `chi0_aux` as GW/real_screening.py:
 * 171-181 `screening_aux` calls it:
 *   chi0 = spin_factor (C diag(f)) C^T   (+ chi0 when accumulate, FP64 only),
 * C_dev (naux, nov) row-major with leading dimension ldc, f_dev (nov) the
 * pairs' frequency factor (LinearResponse/imaginary_frequency.py:25-59),
 * chi0_dev (naux, naux) FP64, symmetric on return. mode MBPT_MODE_FP64: a
 * symmetric rank-k DGEMM over column chunks; MBPT_MODE_MIXED: one split
 * BF16x3 tensor-core product (FP32 accumulation, ~1e-5 relative). */
size_t mbpt_chi0_aux_workspace_bytes(int64_t naux, int64_t nov, int mode);
int mbpt_chi0_aux(const double *C_dev, int64_t naux, int64_t nov, int64_t ldc,
                  const double *f_dev, double spin_factor, int accumulate, int mode,
                  double *chi0_dev, void *workspace, size_t ws_bytes, int *err_dev,
                  void *stream);

/* The imaginary-axis screening contraction of the contour deformation:
 * wc[k, c] = B[:, c]^T (W - I)_k B[:, c] for W - I (nfreq, naux, naux) from the
 * Dyson step and B (naux x ncols, row-major; the states' slices side by side):
 * GW/contour_deformation.py:229-237 `screening_contraction` and :248-290
 * `cd_screening_contraction_multi` (one W per frequency serving every
 * state). wc_dev: nfreq x ncols, overwritten. mode: FP64 (cuBLAS DGEMM per
 * frequency) or MIXED ((W - I)_k B as a split-BF16 tensor-core product with
 * FP32 output, the column dots in FP64). */
size_t mbpt_screening_contraction_workspace_bytes(int64_t naux, int64_t ncols, int mode);
int mbpt_screening_contraction(const double *w_minus_i_dev, int nfreq, int64_t naux,
                               const double *B_dev, int64_t ncols, int mode, double *wc_dev,
                               void *workspace, size_t ws_bytes, int *err_dev, void *stream);

/* The contour deformation's reverse (gradients/gwbse/qp_space_time.py:328-361,
 * the integral term's adjoint): for adjoints wc_bar (nfreq x norb) on
 * wc[k, q] = b_q^T (W - I)_k b_q, accumulates B_bar += 2 (W - I)_k B
 * diag(wc_bar[k]) over k and writes W_bar_k = B diag(wc_bar[k]) B^T
 * (nfreq, naux, naux). B, B_bar: naux x norb. FP64. */
size_t mbpt_cd_integral_backward_workspace_bytes(int64_t naux, int64_t norb);
int mbpt_cd_integral_backward(const double *w_minus_i_dev, int nfreq, int64_t naux,
                              const double *B_dev, int64_t norb, const double *wc_bar_dev,
                              double *B_bar_dev, double *W_bar_dev, void *workspace,
                              size_t ws_bytes, void *stream);

/* The three-index slice's reverse (gradients/rpa/space_time_adjoint.py:593-624):
 * for an adjoint B_bar (naux x norb) on B_p = D^T diag(X[:, p]) X, accumulates
 * X_bar (M x norb) and D_bar (M x naux). FP64. */
size_t mbpt_three_index_slice_backward_workspace_bytes(int64_t M, int64_t norb, int64_t naux);
int mbpt_three_index_slice_backward(const double *X_dev, int64_t M, int64_t norb,
                                    const double *D_dev, int64_t naux, int64_t p,
                                    const double *B_bar_dev, double *X_bar_dev,
                                    double *D_bar_dev, void *workspace, size_t ws_bytes,
                                    void *stream);

/* The reverse of the Dyson step W = [1 - chi0]^-1: chi0_bar_f = W_f W_bar_f W_f
 * (gradients/rpa/space_time_adjoint.py:679-685), in place over wbar_dev
 * (nfreq, naux, naux), from W - I (w_minus_i_dev, the Dyson output). mode:
 * MBPT_MODE_FP64 or MBPT_MODE_FP64_INT8. */
size_t mbpt_dyson_backward_workspace_bytes(int64_t naux);
int mbpt_dyson_backward(const double *w_minus_i_dev, double *wbar_dev, int64_t naux, int nfreq,
                        int mode, void *workspace, size_t ws_bytes, void *stream);

/* ---- quasiparticle-shift network (learned warm start) --------------------
 * A 4 -> H -> H -> 1 perceptron with SiLU, FP32, parameters packed as
 * [W1 (H x 4), b1 (H), W2 (H x H), b2 (H), W3 (H), b3 (1)].
 * forward: y (B) from x (B x 4); the activations needed by backward are
 * written to act_dev (B x 4H floats). backward: grad (same packing) of
 * 0.5/B sum (y - t)^2, loss_dev (1) the loss. adamw: one AdamW step. */
int mbpt_mlp_param_count(int hidden);
int mbpt_mlp_forward(const float *params_dev, int hidden, const float *x_dev, int batch,
                     float *y_dev, float *act_dev, void *stream);
int mbpt_mlp_backward(const float *params_dev, int hidden, const float *x_dev, int batch,
                      const float *act_dev, const float *y_dev, const float *target_dev,
                      float *grad_dev, float *loss_dev, void *stream);
int mbpt_mlp_adamw(float *params_dev, const float *grad_dev, float *m_dev, float *v_dev,
                   int count, float lr, float beta1, float beta2, float eps, float weight_decay,
                   int step, void *stream);

/* ---- split-precision GEMM (diagnostic entry of the tensor-core engine) ---
 * C (m x n, FP32, ldc) = alpha * A B^T with A (m x k) and B (n x k) FP64,
 * each rounded to a BF16 pair and multiplied with three tcgen05 products.
 * m, n, k are padded internally to multiples of 128 / 128 / 64. Extents
 * above 2^24 are refused (MBPT_ERR_SHAPE; the sizing call returns SIZE_MAX). */
size_t mbpt_gemm_split_workspace_bytes(int64_t m, int64_t n, int64_t k);
int mbpt_gemm_split(const double *A_dev, const double *B_dev, int64_t m, int64_t n, int64_t k,
                    double alpha, float *C_dev, int64_t ldc, void *workspace, size_t ws_bytes,
                    int *err_dev, void *stream);
/* The same with TF32 hi/lo pairs (22 significant bits, tcgen05 kind::tf32):
 * the product form of the chi0 sweep's G_occ / G_virt stage in mixed mode.
 * k is padded to a multiple of 32. */
size_t mbpt_gemm_split_tf32_workspace_bytes(int64_t m, int64_t n, int64_t k);
int mbpt_gemm_split_tf32(const double *A_dev, const double *B_dev, int64_t m, int64_t n,
                         int64_t k, double alpha, float *C_dev, int64_t ldc, void *workspace,
                         size_t ws_bytes, int *err_dev, void *stream);

/* ---- FP64-accurate GEMM on the int8 tensor cores ---------------------------
 * C (m x n, row-major, ldc) = alpha op(A) op(B) + beta C, op(A) = A (m x k,
 * lda) or A^T (ta: A is k x m), op(B) = B (k x n, ldb) or B^T (tb: B is
 * n x k), all FP64 row-major. The Ozaki scheme: each row of op(A) and each
 * column of op(B) is scaled by a power of two above its largest magnitude
 * and cut into `slices` (7 or 8) signed 7-bit digits; the digit products are
 * exact int32 tcgen05 products, combined in FP64 (error about 2^-7S K
 * max|row| max|column| per entry: FP64 level at 8 digits). The FP64
 * products of the reverse sweeps (the NumPy matrix products of
 * gradients/rpa/space_time_adjoint.py:167-218, 795-875) run on it.
 * K is taken in passes of at most 32768. */
size_t mbpt_dgemm_ozaki_workspace_bytes(int64_t m, int64_t n, int64_t k, int slices);
int mbpt_dgemm_ozaki(int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha,
                     const double *A_dev, int64_t lda, const double *B_dev, int64_t ldb,
                     double beta, double *C_dev, int64_t ldc, int slices, void *workspace,
                     size_t ws_bytes, int *err_dev, void *stream);

/* ---- split-precision GEMM without caller scratch -------------------------
 * No counterpart in MBPTcode: an addition of this library for callers that
 * cannot allocate device memory, typically hosts whose device memory is all
 * owned by their own allocator (a framework's caching pool, a fixed memory
 * budget) and which therefore can neither pass a workspace nor let the
 * library call cudaMalloc. Same product as mbpt_gemm_split (C = alpha A B^T,
 * A m x k, B n x k FP64, C FP32 with ldc), but its scratch is a 32 MiB
 * file-scope device array inside the library, which every GPU that loads
 * the library holds until the process exits; the call itself allocates
 * nothing. Limit: the padded operands and product must fit,
 * 4 (mp kp + np kp) + 4 mp np <= 32 MiB with mp, np = m, n rounded up to
 * 128 and kp = k rounded up to 64 (each part 1024-byte aligned); larger sizes
 * return MBPT_ERR_WORKSPACE and compute nothing.
 * The first call on a device looks up that array's device address (with
 * the device current) and keeps it; make that first call before any stream
 * capture. All calls share the one array and each overwrites it: calls whose
 * work overlaps on the GPU (other streams, other host threads) race and must
 * be serialised by the caller. mbpt_gemm_split_static_capacity returns the
 * array's size in bytes. */
size_t mbpt_gemm_split_static_capacity(void);
int mbpt_gemm_split_static(const double *A_dev, const double *B_dev, int64_t m, int64_t n,
                           int64_t k, double alpha, float *C_dev, int64_t ldc, int *err_dev,
                           void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MBPT_B200_H */
