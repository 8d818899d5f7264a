/*
 * pci_batch.h -- C ABI of the batched form: many independent CI blocks
 * (different ions, M_J and parity), each with its own lower-triangle
 * Hamiltonian, solved for their lowest roots together on one GPU.
 *
 * The reference solves one block per pconf run: Diag4 (pconf.F90:238, with
 * the Davidson module davidson.f90) takes Nlv, N_it and the residual criterion
 * Crt4 and returns the energies Tk(1:Nlv) and vectors ArrB.  This interface
 * keeps those meanings per block (nlv, max_it, tol; energies and vectors in
 * the same order), with H stored in FP32 (or FP64) and FP64 vectors.
 *
 * Every iteration step of the solve is one kernel launch over all blocks,
 * the SpMM one persistent kernel over the rows of every block, and the
 * iterations are replayed from a CUDA graph.  Blocks are added from
 * pci_gpu_t handles whose Hamiltonian is resident (pci_gpu_form_h or
 * pci_gpu_set_csr); the batch takes over that matrix.
 *
 * Every int-returning entry point returns PCI_OK (0) or a PCI_E_* code of
 * pci_gpu.h; pci_batch_last_error() then holds a message.
 */
#ifndef PCI_BATCH_H
#define PCI_BATCH_H

#include <stdint.h>

#include "pci_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pci_batch pci_batch_t;

#define PCI_BATCH_MAX_LV   12   /* roots per block */
#define PCI_BATCH_MAX_SUB  112  /* subspace vectors per block (the projected eigensolve keeps two
                                   112 x 112 FP64 arrays in shared memory) */

#define PCI_BATCH_FP64  0   /* SpMM on FP64 vectors with FP64 sums throughout */
#define PCI_BATCH_MIXED 1   /* SpMM on FP32 vectors with FP32 sums (FP32 values) until every root of a
                               block is at or below switch_tol, or the largest residual stops dropping
                               (stall_max iterations without a 10% drop); then a restart on the Ritz
                               vectors and the FP64 SpMM (FP64 values, or hi + lo of a split block) to
                               tol.  Basis, projections, eigensolve and residual norms stay FP64. */

#define PCI_BATCH_CORR_DIAG    0   /* t = r / (theta - H_nn), as Dvdsn (davidson.f90:436-570) */
#define PCI_BATCH_CORR_LEARNED 1   /* t = output of the attached model (pci_batch_set_correction_model)
                                      per row; a root whose residual does not drop from one iteration
                                      to the next takes the diagonal correction for the rest of the
                                      solve */

typedef struct {
    int32_t nlv;            /* roots per block, 1..PCI_BATCH_MAX_LV (Nlv) */
    int32_t max_sub;        /* subspace size at which a block restarts, 2*nlv..PCI_BATCH_MAX_SUB */
    int32_t keep;           /* Ritz vectors kept at a restart, nlv..max_sub-nlv */
    int32_t max_it;         /* iteration limit per block (N_it) */
    double tol;             /* residual 2-norm per root (Crt4) */
    int32_t it_per_graph;   /* iterations captured in one CUDA graph, >= 1 */
    int32_t spmm_variant;   /* SpMM variant (pci_batch_tune), -1 = tuned or default */
    int32_t precision;      /* PCI_BATCH_FP64 or PCI_BATCH_MIXED */
    int32_t stall_max;      /* PCI_BATCH_MIXED: see above; 0 = 8 */
    double switch_tol;      /* PCI_BATCH_MIXED: residual that ends the FP32 phase (>= tol) */
    int32_t correction;     /* PCI_BATCH_CORR_DIAG or PCI_BATCH_CORR_LEARNED */
    int32_t pad;
} pci_batch_params;

/* One sample for training the learned correction: the state of one root of
 * one block at one iteration, seen at one sampled row. */
typedef struct {
    int32_t blk, iter, root, phase;   /* block, iteration (1-based), root, SpMM phase */
    int64_t row;                      /* row within the block, 0-based */
    double x;                         /* entry of the root's Ritz vector at this iteration */
    double r;                         /* entry of its residual H x - theta x */
    double theta;                     /* Ritz value */
    double rnorm;                     /* residual 2-norm */
    double diag;                      /* H_nn */
} pci_batch_sample;

int pci_batch_create(int32_t device, pci_batch_t **out);

/* Append the Hamiltonian resident in `h` as the next block and take it over
 * (h keeps its basis and integrals but no longer holds H; on an error return
 * the matrix is released and h no longer holds it either).  FP64 values are
 * rounded to FP32, kept, or split into FP32 pairs as pci_batch_set_value_prec
 * says.  When h holds a determinant basis, the occupied orbitals of every row
 * are kept as the learned correction's inputs.  *index receives the block's
 * index. */
int pci_batch_add_block(pci_batch_t *b, pci_gpu_t *h, int32_t *index);

/* Value precision of blocks added from now on: 32 (default) rounds FP64
 * values to FP32 when a block is added; 64 keeps each block's values as its
 * handle built them (FP64 from pci_gpu_form_h with value_prec 64); 48 splits
 * each FP64 value v in place into the FP32 pair hi = fl(v), lo = fl(v - hi)
 * (same memory as FP64; hi + lo = v to about 2^-48 relative): the FP32 SpMM
 * of PCI_BATCH_MIXED reads hi, the FP64 SpMM hi + lo. */
int pci_batch_set_value_prec(pci_batch_t *b, int32_t value_prec);

/* Storage of the blocks' matrices for the solve: 0 (default) = lower
 * triangles only (the SpMM adds the transpose part by global reductions);
 * 1 = blocks, largest first, get a symmetric copy of both triangles (the
 * SpMM then gathers rows with no reductions, reading every element twice)
 * while it fits in free device memory beside the solve buffers with a 4 GiB
 * margin.  Takes effect at the next pci_batch_tune or pci_batch_davidson;
 * cannot be switched back to 0 once copies exist. */
int pci_batch_set_storage(pci_batch_t *b, int32_t mode);

/* Blocks, total rows and total stored (lower-triangle) elements. */
int pci_batch_info(pci_batch_t *b, int32_t *nblocks, int64_t *rows, int64_t *nnz);

/* Pick the SpMM variant for nv vectors by timing each candidate on the
 * batch's matrix (ms = the chosen variant's time per SpMM), or take it from
 * the cache file `cache_path` (NULL = no cache) when it holds a line for the
 * same device and matrix; new results are appended there.  The pick is used
 * by later pci_batch_davidson calls with spmm_variant = -1. */
int pci_batch_tune(pci_batch_t *b, int32_t nv, const char *cache_path, int32_t *variant, double *ms,
                   int32_t *from_cache);

/* Parameters of SpMM variant `variant` (lanes per row, thread blocks per SM);
 * returns the number of variants when `variant` is out of range.  A variant
 * whose lanes per row are fewer than the vectors is not used. */
int pci_batch_variant(int32_t variant, int32_t *lanes_per_row, int32_t *blocks_per_sm);

/* Solve every block.  E[blk*nlv + j] = energy of root j, rnorm likewise its
 * final residual 2-norm, iters[blk] = iterations the block took, status[blk]
 * = 1 converged, 2 iteration limit, 3 no new direction left.  graph_launches
 * (may be NULL) receives the number of graph replays. */
int pci_batch_davidson(pci_batch_t *b, const pci_batch_params *p, double *E, double *rnorm, int32_t *iters,
                       int32_t *status, int32_t *graph_launches);

/* Ritz vectors of block blk after pci_batch_davidson: X[nd_blk x nlv],
 * column-major, unit 2-norm. */
int pci_batch_vectors(pci_batch_t *b, int32_t blk, double *X);

/* Timings of the last solve: out[0] total ms, [1] iterations (largest over
 * blocks), [2] SpMM ms per call on FP64 vectors (measured outside the
 * graph), [3] SpMM variant used, [4] setup ms, [5] kernel launches per
 * iteration, [6] share of the lower-triangle elements held as full copies,
 * [7] SpMM ms per call on FP32 vectors (PCI_BATCH_MIXED), [8] largest number
 * of FP32-phase iterations of a block, [9] blocks that reached the FP64
 * phase (PCI_BATCH_MIXED); n <= 10. */
int pci_batch_stats(pci_batch_t *b, double *out, int32_t n);

/* Attach a trained model (pci_gpu.h) for correction = PCI_BATCH_CORR_LEARNED;
 * NULL detaches.  Its first nin - 3 inputs are the occupation counts of the
 * orbitals; with s = sqrt(nd) / |r|, input nin - 3 is H_nn - theta, input
 * nin - 2 the residual entry r_n s and input nin - 1 the diagonal correction
 * r_n s / (theta - H_nn) (denominator at least 1e-8 in size, value clipped to
 * +-1e4); every block must come from a handle with a basis of at most
 * nin - 3 orbitals.  The model must outlive its use.  No
 * counterpart in the reference, whose only correction is Dvdsn's diagonal one
 * (davidson.f90:436-570). */
int pci_batch_set_correction_model(pci_batch_t *b, pci_mlp_t *m);

/* Record training samples in the next solves: rows_per_block rows of every
 * block (all rows of smaller blocks) drawn with `seed`, up to `capacity`
 * samples (later ones are counted, not kept); 0 rows switches it off. */
int pci_batch_set_harvest(pci_batch_t *b, int32_t rows_per_block, int64_t capacity, int32_t seed);

/* Samples of the last solve: up to cap into out (may be NULL); *count
 * receives the number recorded (above the capacity, the rest were dropped). */
int pci_batch_harvest(pci_batch_t *b, pci_batch_sample *out, int64_t cap, int64_t *count);

/* Measured throughput of the SpMM's transpose part on this device: FP64
 * reductions by teams of nv lanes onto nv consecutive words at random rows of
 * a rows x nv array (rows = the SpMM's row count), as GB/s of reduced data.
 * The lower-triangle SpMM adds nnz * nv such words per call, so this is the
 * roofline that bounds it.  Allocates rows * nv * 8 bytes for the probe. */
int pci_batch_probe_reduction(int32_t device, int64_t rows, int32_t nv, double *gbs);

const char *pci_batch_last_error(pci_batch_t *b);
void pci_batch_destroy(pci_batch_t *b);

#ifdef __cplusplus
}
#endif

#endif
