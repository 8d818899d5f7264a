/*
 * pci_gpu.h -- C ABI of the B200 engine for pconf's two hot stages:
 * the determinant-pair Hamiltonian build (FormH / FormJ) and the Davidson
 * eigensolver (Diag4).
 *
 * Every argument is ISO_C_BINDING-interoperable (int32_t, int64_t, double,
 * plain pointers).  Index conventions are the Fortran ones: m-state, orbital
 * and determinant indices are 1-based values, arrays are passed as the
 * column-major Fortran arrays they are in pconf (Iarr(Ne,Nd) is Ne
 * consecutive m-states per determinant).  Host arrays are borrowed for the
 * duration of a call; device buffers (tables, CSR, vectors) belong to the
 * handle until pci_gpu_destroy.  Calls on one handle must come from one host
 * thread; all calls are synchronous.
 *
 * Every int-returning entry point returns PCI_OK (0) or one of the PCI_E_*
 * codes below; pci_gpu_last_error() then holds a message.
 */
#ifndef PCI_GPU_H
#define PCI_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCI_OK                 0
#define PCI_E_INPUT            1  /* inconsistent sizes or indices (pconf Stop) */
#define PCI_E_OOM              2  /* device allocation failed */
#define PCI_E_MISSING_INTEGRAL 3  /* Gint: integral is absent (integrals.f90:256-261) */
#define PCI_E_ORTHO_FAIL       4  /* Fail of orthogonalization/normalization (davidson.f90:718-737) */
#define PCI_E_TIMEOUT          5  /* a bounded device wait gave up */
#define PCI_E_CUDA             6  /* CUDA runtime / library error */
#define PCI_E_STATE            7  /* call out of order (e.g. davidson before form_h) */
#define PCI_E_NOT_CONVERGED    8  /* N_it reached with a residual above Crt4 (info only) */

#define PCI_MAT_H   0
#define PCI_MAT_J2  1

typedef struct pci_gpu pci_gpu_t;

/* Davidson settings.  Field meanings follow CONF.INP / ci.in keys
 * (conf_init.f90:37-213). */
typedef struct {
    int32_t Nlv;        /* number of levels (NLV) */
    int32_t N_it;       /* iteration limit (N_IT) */
    int32_t Kl4;        /* 1: initial vectors from the Nd0 block; 2: from X0 (CONF.XIJ) */
    int32_t Kv;         /* 4: no J selection; 3: select and project on J = XJ_av */
    int32_t Nc4;        /* configurations eligible for the initial block */
    int32_t MaxNd0;     /* largest initial block (ci.in MaxNd0, default 3000) */
    int32_t mode;       /* PCI_DVD_FP64 (reference algorithm) or PCI_DVD_FP32: H stored in FP32
                           (form_h value_prec 32), SpMM on float vectors with FP32 accumulation;
                           orthogonalisation, projections, Rayleigh quotients, residual norms and
                           the projected eigensolve stay FP64 */
    int32_t KXIJ;       /* unused by the library; kept for the caller's CONF.XIJ cadence */
    double  Crt4;       /* residual-norm convergence threshold (CRT4) */
    double  XJ_av;      /* target J for Kv = 3 */
    double  admix_crit; /* stop when max admixture <= this (pconf.F90:2015, 1e-6); 0 disables */
} pci_dvd_params;

#define PCI_DVD_FP64 0
#define PCI_DVD_FP32 1
#define PCI_DVD_LEARNED 2   /* FP64; on rows >= Nd0 the correction takes the attached model's
                               direction and the diagonal correction's length; a level whose
                               residual stops decreasing falls back to the diagonal correction */

/* Replaces: the device has no counterpart in pconf; this opens a handle on
 * CUDA device `device` (the MPI rank's process is the reference's unit). */
int pci_gpu_create(int32_t device, pci_gpu_t **h);

/* Replaces: the broadcast of the determinant basis in InitFormH
 * (pconf.F90:1096-1118) -- Iarr, Nh, Jz, Nn, Kk, Ll, Jj, Ndc, Nc, Ne, Nd,
 * Nst, Nso, Nx, Mj, Gj.  Nsu is the number of orbitals in Nn/Kk/Ll/Jj.
 * Determinants must be grouped by configuration in Ndc order and each sorted
 * ascending (Det_List, determinants.f90:144-183). */
int pci_gpu_set_basis(pci_gpu_t *h, int32_t Ne, int64_t Nd, int32_t Nst, int32_t Nsu,
                      int32_t Nso, int32_t Nx, int32_t Mj,
                      const int32_t *Iarr, const int32_t *Nh, const int32_t *Jz,
                      const int32_t *Nn, const int32_t *Kk, const int32_t *Ll, const int32_t *Jj,
                      int32_t Nc, const int32_t *Ndc, double Gj);

/* Replaces: BuildHintLUT, BuildGauntLUT and BuildGintHash
 * (integrals.f90:604-632, 663-674, 702-715) fed by Rint (integrals.f90:13-120)
 * and CONF.GNT (pconf.F90:383-406).  HintLUT has Nx*Nx entries, GauntLUT
 * nGauntLUT entries (index 0..max(In)), Rint2 holds Ngint values (two per
 * integral, interleaved, when kbrt /= 0) as float (r2_is_f64 = 0, the
 * reference's default type2_real) or double (USE_DP_INTEGRALS). */
int pci_gpu_set_integrals(pci_gpu_t *h, const double *HintLUT, int32_t Nlx,
                          int64_t nGauntLUT, const double *GauntLUT,
                          int64_t Ngint, int32_t kbrt, int32_t r2_is_f64,
                          const void *Rint2, const int32_t *Iint2, const int32_t *Iint3);

/* Replaces: Call FormH + RedistributeHamCSR (pconf.F90:217-219).  Builds the
 * lower triangle (diagonal included, columns ascending, exact zeros dropped:
 * npes = 1 semantics, pconf.F90:1259) as device-resident CSR with values in
 * FP64 (value_prec = 64) or FP32 (32).  Returns NumH (stored elements),
 * numzero (difference <= 2 pairs whose element is exactly 0) and Hmin (the
 * minimum stored value, Hamil%minval).  A matrix the handle held before
 * (from an earlier pci_gpu_form_h, dropped by pci_gpu_set_basis or
 * pci_gpu_set_integrals) lends its device buffers to the new one when they
 * fit, instead of being freed and allocated again; buffers left over are
 * freed when the build ends, and any allocation that fails first frees them
 * and retries. */
int pci_gpu_form_h(pci_gpu_t *h, int32_t value_prec, int64_t *NumH, int64_t *numzero, double *Hmin);

/* Replaces: Call FormJ + RedistributeJsqCSR (pconf.F90:224-225).  J^2 in units
 * of (2j)^2 over pairs inside one configuration block. */
int pci_gpu_form_j(pci_gpu_t *h, int64_t *NumJ);

/* Sizes of a resident matrix: rows (Nd) and stored elements. */
int pci_gpu_csr_info(pci_gpu_t *h, int32_t which, int64_t *nrows, int64_t *nnz);

/* Replaces: the Hamil%col/val + HamilCSR_rowptr globals that WriteMatrixCSR
 * streams to pCONF.HIJ (matrix_io.f90:689-799).  Copies the resident CSR out:
 * rowptr[Nd+1] 0-based prefix (HamilCSR_rowptr(0:Nd)), col 1-based, val as
 * double.  Any pointer may be NULL to skip that array. */
int pci_gpu_get_csr(pci_gpu_t *h, int32_t which, int64_t *rowptr, int32_t *col, double *val);

/* Replaces: the row range of Hamil%col/val that one rank holds after
 * RedistributeHamCSR (matrix_io.f90:260-502) and streams to pCONF.HIJ.
 * Copies rows row_lo..row_hi (1-based, inclusive) of the resident matrix:
 * rowptr[row_hi-row_lo+2] as a 0-based prefix within the range, col 1-based,
 * val as double.  col and val may be NULL (size them from rowptr's last
 * entry first). */
int pci_gpu_get_csr_rows(pci_gpu_t *h, int32_t which, int64_t row_lo, int64_t row_hi, int64_t *rowptr, int32_t *col,
                         double *val);

/* Replaces: ReadMatrixCSR (matrix_io.f90:801-939) for Kl = 1 restarts:
 * uploads a lower-triangle CSR (same layout as pci_gpu_get_csr) and its Hmin. */
int pci_gpu_set_csr(pci_gpu_t *h, int32_t which, int64_t Nd, int64_t nnz, const int64_t *rowptr,
                    const int32_t *col, const double *val, double Hmin);

/* Replaces: Call Diag4 (pconf.F90:238) with Init4, DiagInitApprox, FormB0 and
 * the Davidson module (davidson.f90).  X0 (Nd x Nlv column-major, Kl4 = 2) may
 * be NULL.  Outputs: Tk (energies, -(E + Hmin)), Tj (J of each level, J_av),
 * Iconverge, X (Nd x Nlv column-major eigenvectors, may be NULL), the
 * iteration count and, if non-NULL, the final residual norms (length Nlv).
 * Kv = 3 selects initial vectors with J = XJ_av, averages the diagonal over
 * configurations (AvgDiag) and filters new vectors onto J = XJ_av (Prj_J with
 * the terms of pci_gpu_jterms); if fewer than Nlv initial vectors have that
 * J, the reference lowers Nlv, and the levels past that number come back with
 * Iconverge = -1 and zero Tk, Tj and X. */
int pci_gpu_davidson(pci_gpu_t *h, const pci_dvd_params *p, const double *X0,
                     double *Tk, double *Tj, int32_t *Iconverge, double *X,
                     int32_t *iters, double *resid);

/* Replaces: J_av (formj2.f90:355-387), the J of each vector from
 * <x|J^2|x> over rows and columns 1..nlim of the resident J^2 matrix, as
 * WriteFinalXIJ (pconf.F90:2566-2602) and FormB0 (davidson.f90:107-135) use
 * it.  X is Nd x nv column-major on the host (1 <= nv <= 64); Tj[nv] receives
 * J = (sqrt(1 + <x|J^2|x>) - 1) / 2. */
int pci_gpu_j_av(pci_gpu_t *h, const double *X, int32_t nv, int64_t nlim, double *Tj);

/* Replaces: lsj / calcLSJ / lsj_det (pconf.F90:2672-2962), the kLSJ = 1
 * step: for each vector the quantum numbers J, L, S from <x|X^2|x> over the
 * determinant pairs of equal non-relativistic configuration (CompNRC = 0)
 * and relativistic CompC <= 2, x = (sqrt(<X^2> + 1) - 1) / 2.  X is Nd x nv
 * column-major on the host (1 <= nv <= 64), normalised as the caller wants
 * (the reference passes the eigenvectors).  Needs the principal numbers Nn
 * passed to pci_gpu_set_basis (PCI_E_STATE without them). */
int pci_gpu_lsj(pci_gpu_t *h, const double *X, int32_t nv, double *xj, double *xl, double *xs);

/* Replaces: the density-matrix pass of pdtm's FormDM (pdtm.f90:1134-1336):
 * for each vector of X (Nd x nv column-major, host) the one-particle density
 * matrix over the m-states, from the determinant pairs n >= k whose
 * relativistic configurations differ by at most one orbital and whose
 * coefficients satisfy |b_n| > trd and |b_n b_k| > trd (pdtm's Trd, default
 * 1e-10).  Ro (Nst x Nst x nv, column-major per vector, host) receives
 * Ro(i, j) for 1-based m-states i, j at Ro[(v*Nst + j-1)*Nst + i-1]; the
 * reference's Ro is this shifted by Npo (the core m-states). */
int pci_gpu_density(pci_gpu_t *h, const double *X, int32_t nv, double trd, double *Ro);

/* Replaces: the transition-density pass of pdtm's FormTM (pdtm.f90:
 * 1538-1605) for one initial level (vector bi over the basis of handle hi)
 * and one final level (bf over the basis of hf; the two bases share Ne and
 * the m-states, e.g. opposite parities): the determinant pairs whose
 * relativistic configurations differ by at most one orbital, |b_n| > trd
 * and |b_n b_k| > trd.  Ro (Nst x Nst column-major, host) receives Ro(i, j)
 * with i the initial determinant's m-state and j the final's (1-based, at
 * Ro[(j-1)*Nst + i-1]). */
int pci_gpu_transition_density(pci_gpu_t *hi, pci_gpu_t *hf, const double *bi, const double *bf, double trd,
                               double *Ro);

/* Replaces: the kCSF = 1 path, jbasis + formh_sym (csf.f90:17-407, 538-1006;
 * pconf.F90:146-148, 211-214).  From the resident FP64 determinant H
 * (pci_gpu_form_h(64)) and J^2 (pci_gpu_form_j): each configuration's CSFs
 * are the eigenvectors of its J^2 block with 2J = Mj, and the CSF
 * Hamiltonian C^T H C replaces H on the handle (lower triangle, FP64; CSFs
 * in configuration order).  *ncsf receives the number of CSFs, *numh the
 * stored elements.  Solve it with the batched solver (pci_batch_add_block);
 * pci_gpu_davidson refuses it.  Configurations of up to 112 determinants. */
int pci_gpu_form_csf(pci_gpu_t *h, int64_t *ncsf, int64_t *numh);
/* CSFs of each configuration (Nc entries) after pci_gpu_form_csf. */
int pci_gpu_csf_counts(pci_gpu_t *h, int32_t *per_conf);
/* Replaces: unsym (csf.f90:1088-1134).  Y is Ncsf x nv column-major on the
 * host (1 <= nv <= 64); X (Nd x nv, column-major, host) receives the
 * determinant vectors. */
int pci_gpu_csf_to_det(pci_gpu_t *h, const double *Y, int32_t nv, double *X);

/* Replaces: conf_pt's PTE (conf_pt.f90:751-952), second-order CI+PT, for PT
 * spaces whose Hamiltonian the device holds: the resident determinant H
 * (pci_gpu_form_h over the CI determinants followed by the PT ones) and the
 * CI vectors X0 over the first nd0 determinants (nd0 x nv column-major,
 * host; nd0 <= nd1 <= Nd, both at configuration ends).  For every
 * determinant i > nd1: x = sum_(k <= nd0) H_ik X0_kn, dE[n] += x^2 /
 * (E[n] - H_ii), and Xpt (Nd x nv column-major, may be NULL; rows <= nd1
 * zero) receives c_in = x / (E[n] - H_ii).  E are the levels' energies as
 * eigenvalues of H; dE is negative for a lowest level (the reference's
 * Ey(n) is -dE[n] in its binding convention).  avg_diag = 1 applies
 * average_diag as the reference does (conf_pt.f90:710-724: the mean goes to
 * each PT configuration's last determinant).  H must be built with Gj = 0
 * (conf_pt's Hmltn has no J^2 term; its energies E take the Gj shift off,
 * conf_pt.f90:737). */
int pci_gpu_pt2(pci_gpu_t *h, int64_t nd1, int64_t nd0, const double *X0, int32_t nv, const double *E,
                int32_t avg_diag, double *dE, double *Xpt);

/* Replaces: PTE's contributions of the non-relativistic configurations
 * (dE(n,ic), dV(n,ic), conf_pt.f90:871-872, from which it prints DEnr and
 * DVnr).  pci_gpu_pt2 plus, for ngrp groups of PT rows given as ascending
 * determinant offsets grp[0..ngrp] (group g holds rows grp[g]..grp[g+1]-1,
 * all within nd1..Nd; NR_Init's non-relativistic configurations,
 * conf_pt.f90:500-570, are the reference's groups), dEg[g*nv + n] = the
 * group's sum of x^2 / (E[n] - H_ii) and dVg[g*nv + n] = its sum of c_in^2
 * (both ngrp x nv, host).  On a PT block of pci_gpu_form_h_pt_rows the
 * sums cover that block's rows. */
int pci_gpu_pt2_groups(pci_gpu_t *h, int64_t nd1, int64_t nd0, const double *X0, int32_t nv, const double *E,
                       int32_t avg_diag, const int64_t *grp, int32_t ngrp, double *dE, double *dEg, double *dVg,
                       double *Xpt);

/* Replaces: conf_pt's own FormH (conf_pt.f90:1319-1351), which forms for
 * each PT determinant only its row against the first nd0 determinants.
 * Builds, in place of H, the block pci_gpu_pt2 reads: the rows of the
 * determinants beyond nd1 against columns below nd0, plus each PT
 * configuration's own diagonal block (for H_ii); rows up to nd1 stay empty
 * and the PT x PT block between different configurations is not formed, so
 * the stored elements grow with the PT space times the zero-order space's
 * neighbours instead of the PT space squared.  Elements are bit-identical to
 * the same positions of pci_gpu_form_h's H.  nd0 <= nd1 < Nd, both at
 * configuration ends; value_prec 64 or 32.  pci_gpu_pt2 must then be called
 * with the same nd1 and nd0; the Davidson entry points, the batched solver
 * and pci_gpu_form_csf refuse this matrix. */
int pci_gpu_form_h_pt(pci_gpu_t *h, int64_t nd1, int64_t nd0, int32_t value_prec, int64_t *NumH);

/* No counterpart in the reference, whose PTE shares each PT configuration's
 * determinants out over its MPI ranks and reduces the sums
 * (conf_pt.f90:825-860); here a share is a range of whole PT configurations,
 * so that each block holds whole diagonal blocks.  pci_gpu_form_h_pt for the PT rows
 * row_lo..row_hi-1 only (nd1 <= row_lo < row_hi <= Nd, all at configuration
 * ends): for a PT space whose whole PT block exceeds the device, or for one
 * range per GPU.  pci_gpu_pt2 on it gives that range's share: the ranges' dE
 * add up to the whole PT space's, and Xpt is zero outside the range. */
int pci_gpu_form_h_pt_rows(pci_gpu_t *h, int64_t nd1, int64_t nd0, int64_t row_lo, int64_t row_hi,
                           int32_t value_prec, int64_t *NumH);

/* No counterpart in the reference.  The J_av of pci_gpu_j_av for callers that
 * cannot allocate device memory (a host that owns all device memory through
 * its own pool or a framework's caching allocator, or a path where
 * cudaMalloc's implicit synchronisation is not acceptable).  Every array is
 * device memory the caller already holds: the J^2 matrix in the
 * pci_gpu_get_csr layout (rowptr[nrows+1] 0-based prefix, col 1-based, val
 * the FP64 values pci_gpu_get_csr(h, PCI_MAT_J2, ...) returns -- an FP32
 * copy is read as doubles and gives wrong J), X column-major with leading
 * dimension ldx >= nrows, and Tj[nv] for the result.  No handle and no allocation: the only scratch is a static device
 * array of 64 doubles, so nv is limited to 1..64 (larger nv returns
 * PCI_E_INPUT).  Work is enqueued on `stream` (NULL = default stream) and not
 * waited for.  All calls on a device share the scratch; calls that overlap on
 * the GPU race.  The first call on a device resolves the scratch address and
 * should come before any stream capture; that address belongs to the device's
 * primary context and stays valid until the process exits or the device is
 * reset (after cudaDeviceReset, or under another driver context, do not call
 * this entry point again in the same process).  On error, errbuf (errlen bytes, may
 * be NULL) receives a message. */
int pci_gpu_j_av_noalloc(const int64_t *rowptr, const int32_t *col, const double *val, int64_t nrows,
                         const double *X, int64_t ldx, int32_t nv, int64_t nlim, double *Tj,
                         void *stream, char *errbuf, int32_t errlen);

/* Replaces: FormBarr (src/determinants.f90:839-864), the bit-string form of
 * the determinant list that pconf builds when Ne >= num_ints_bit_rep or
 * CONF_USE_BIT_DET is set: Barr(nint, Nd), nint = ceil(Nst / 32), bit
 * (m-1) mod 32 of word (m-1)/32 + 1 set for every occupied m-state m.  Kept
 * on the device; *nint receives nint; barr (nint x Nd int32, may be NULL)
 * receives a copy. */
int pci_gpu_form_barr(pci_gpu_t *h, int32_t *nint, int32_t *barr);

/* Replaces: compare_bit_dets + get_det_indexes (src/determinants.f90:933-1034)
 * on the device for n determinant pairs (pairs[2i], pairs[2i+1], 1-based):
 * ndiffs (3 for three or more), the phase is and the differing m-states
 * idx1[3i..3i+2], idx2[3i..3i+2] of each determinant in the reference's slot
 * order (slot 1 unused, 0 where absent).  The reference's phase rule is kept
 * as it is, including its disagreement with Rspq on some single
 * differences.  Needs pci_gpu_form_barr. */
int pci_gpu_bit_compare(pci_gpu_t *h, int64_t n, const int64_t *pairs, int32_t *ndiffs, int32_t *is, int32_t *idx1,
                        int32_t *idx2);

/* Jt(1:Njd) of the basis set by pci_gpu_set_basis: the sorted 2J values of
 * the terms its configurations hold, as Dinit lists them
 * (src/determinants.f90:227-325); Prj_J of the Kv = 3 Davidson filters
 * them.  Copies up to cap values into out (may be NULL) and returns Njd, or
 * -1 before set_basis. */
int32_t pci_gpu_jterms(pci_gpu_t *h, int32_t *out, int32_t cap);

/* ---- Learned Davidson correction ------------------------------------------
 * A small MLP (nin -> 128 -> 128 -> 128 -> 1, ReLU) whose forward and
 * backward products run on the tensor cores with BF16 weights, FP32
 * activations split into two BF16 terms (hi + lo) and FP32 accumulation, with
 * FP32 master weights and Adam moments; trained on the GPU.  No counterpart in
 * the reference, which has only the diagonal correction of Dvdsn
 * (davidson.f90:436-570).  Parameters are laid out layer by layer as
 * W (din x dout, row-major) then b (dout). */
typedef struct pci_mlp pci_mlp_t;
int pci_mlp_create(int32_t device, int32_t nin, int32_t seed, pci_mlp_t **m);
int64_t pci_mlp_num_params(pci_mlp_t *m);
int pci_mlp_set_params(pci_mlp_t *m, const float *p, int64_t n);
int pci_mlp_get_params(pci_mlp_t *m, float *p, int64_t n);
/* y[n] from X[n x nin] (host arrays). */
int pci_mlp_forward(pci_mlp_t *m, const float *X, int64_t n, float *y);
/* y[n] from the compact inputs the solver uses, on the tensor-core path of
 * the batched solver's learned correction: orbs[n x 8] holds each row's
 * occupied orbitals (0-based, an orbital listed once per electron in it,
 * 0xff = empty slot; these are the non-zero occupation counts of inputs
 * 0..nin-4), f[n x 3] inputs nin-3, nin-2 and nin-1 (host arrays).  The
 * hidden activations are rounded to BF16 for the tensor-core products, so
 * y agrees with pci_mlp_forward on the same rows to about 1e-2 relative. */
int pci_mlp_forward_occ(pci_mlp_t *m, const uint8_t *orbs, const float *f, int64_t n, float *y);
/* Mean squared error against T[n] and its gradient (length num_params,
 * may be NULL) for X[n x nin] (host arrays). */
int pci_mlp_loss_grad(pci_mlp_t *m, const float *X, const float *T, int64_t n, float *loss, float *grad);
/* Adam (lr, betas 0.9/0.999) over shuffled batches for `epochs` passes of
 * (X, T); *loss_out receives the last epoch's mean batch loss. */
int pci_mlp_train(pci_mlp_t *m, const float *X, const float *T, int64_t n, int32_t epochs, int32_t batch, float lr,
                  int32_t seed, float *loss_out);
const char *pci_mlp_last_error(pci_mlp_t *m);
void pci_mlp_destroy(pci_mlp_t *m);
/* The FP64 Davidson with every unconverged level's correction rows >= Nd0
 * recorded as samples for the model: features (Nsu occupation counts,
 * D_n - theta, residual entry times sqrt(Nd)/|r|; Nsu + 2 floats per
 * sample) into feat, and after the solve the targets (converged vector
 * minus that iteration's vector, signs aligned, scaled to unit RMS over the
 * rows >= Nd0 of that level and iteration) into target.  The converged vectors are Xref (Nd x Nlv, column-major, e.g.
 * from a solve whose initial block covers every determinant) or, when Xref
 * is NULL, the solve's own final vectors.  Up to cap samples are written;
 * *count receives the number recorded.  Tk, Iconverge (Nlv each) and iters
 * as pci_gpu_davidson. */
int pci_gpu_davidson_harvest(pci_gpu_t *h, const pci_dvd_params *p, const double *Xref, float *feat, float *target,
                             int64_t cap, int64_t *count, double *Tk, int32_t *Iconverge, int32_t *iters);
/* Attach a trained model to the handle for the learned Davidson form
 * (mode PCI_DVD_LEARNED); NULL detaches.  The model must outlive its use. */
int pci_gpu_set_correction_model(pci_gpu_t *h, pci_mlp_t *m);

/* Per-stage device times (milliseconds) and counters of the last calls:
 * [0] FormH total (adjacency + count + fill + compaction), [1] FormH count
 * pass (candidate bound in the single-evaluation build), [2] FormH fill
 * pass, [3] FormJ, [4] Davidson total, [5] SpMM total in the last Davidson,
 * [6] number of SpMM launches, [7] Init4 + DiagInitApprox, [8] configuration
 * adjacency build, [9] determinant pairs with difference <= 2, [10]
 * determinant pairs compared, [11] kernel launches of the last FormH,
 * [12] FormH compaction, [13] 1 when the last FormH took the single-
 * evaluation build, 0 for the two-pass build, [14] element slots of the
 * padded rows in the single-evaluation build.  n is the capacity of `out`;
 * returns the number written. */
int32_t pci_gpu_stats(pci_gpu_t *h, double *out, int32_t n);

const char *pci_gpu_last_error(pci_gpu_t *h);
void pci_gpu_destroy(pci_gpu_t *h);

#ifdef __cplusplus
}
#endif
#endif /* PCI_GPU_H */
