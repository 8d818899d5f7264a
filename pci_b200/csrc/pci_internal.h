// Internal declarations shared by the translation units of libpci_gpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/pci_gpu.h"

#define PCI_NE_MAX 8
#define PCI_MAX_PROBE 4096

// Device error bits (OR-ed into Handle::d_err by kernels)
#define DERR_MISSING_INTEGRAL 1u
#define DERR_M_NOT_CONSERVED  2u
#define DERR_BAD_INDEX        4u
#define DERR_ROW_SLOTS        8u   // a row produced more elements than its slots

struct Csr {
    int64_t nrows = 0, nnz = 0;
    int64_t *rowptr = nullptr;   // [nrows+1], 0-based prefix
    int32_t *col = nullptr;      // 0-based column
    void *val = nullptr;         // double or float
    int val_f32 = 0;
    int64_t cap = 0;             // col/val slots allocated when more than nnz (padded build), else 0
};

// Everything the H-build kernels read; plain pointers so it can be passed by value.
struct DevSys {
    int ne, nst, nsu, nso, nx, mj, nc, nlx, kbrt, kdim, ntype;
    int plans;   // per-tile term lists allowed: no Breit term, m-states numbered orbital by orbital
    int64_t nd;
    double gj;
    const uint16_t *occ;        // [nd*ne] 0-based m-state, ascending per determinant
    const int32_t *conf_of;     // [nd]
    const int64_t *conf_start;  // [nc+1]
    const uint16_t *conf_orb;   // [nc*ne] 0-based orbitals of the configuration, ascending
    const int64_t *adj_ptr;     // [nc+1]
    const int32_t *adj;         // connected configurations c2 <= c1, ascending
    const int16_t *ms_orb;      // [nst] orbital (0-based) of each m-state
    const int8_t *ms_jz;        // [nst] 2m
    const uint8_t *ms_type;     // [nst] (j,m) type index into the Gaunt table
    const uint32_t *msd;        // [nst] packed: orbital, type, 2m+128, l, (2j-1)/2
    const int8_t *orb_l;        // [nsu]
    const int8_t *orb_j;        // [nsu] 2j
    const double *h1;           // [nsu*nsu] one-electron integrals, 0 unless kappa equal
    const double *gaunt;        // [kdim][ntype][ntype]
    // radial-integral hash: slot s = 2 (or 4 with the Breit term) 64-bit
    // words at htab + s * hw: key, value(s); key 0 = empty
    const unsigned long long *htab;
    int hw;
    unsigned long long hmask;
    unsigned int *err;
};

struct pci_gpu {
    int device = 0;
    cudaStream_t st = nullptr;
    std::string err;
    // basis
    int ne = 0, nst = 0, nsu = 0, nso = 0, nx = 0, mj = 0, nc = 0;
    int64_t nd = 0;
    double gj = 0.0;
    bool have_basis = false, have_ints = false;
    std::vector<int32_t> h_ndc;       // host copy of Ndc
    std::vector<int32_t> h_orb_j, h_orb_l, h_orb_k;
    std::vector<int32_t> h_orb_n;     // principal numbers Nn (empty when not given)
    int8_t *d_orb_n = nullptr;
    // CSF basis (pci_gpu_form_csf): coefficients C_c (ndc x ncsf per
    // configuration, column-major at csf_coff[c]) and the first CSF of each
    // configuration
    double *d_csf_C = nullptr;
    int64_t *d_csf_start = nullptr, *d_csf_coff = nullptr;
    std::vector<int64_t> h_csf_start;
    int64_t ncsf = 0;
    // LSJ's configuration pairs (pci_gpu_lsj), built once per basis
    int2 *d_lsj_items = nullptr;
    int64_t lsj_nitems = -1;
    std::vector<int32_t> h_nh, h_jz;
    std::vector<int32_t> h_jterms;    // Jt(1:Njd): sorted 2J of the terms present
    std::vector<unsigned long long> h_rowwork;   // determinant pairs per row, per configuration
    uint32_t *d_msd = nullptr;                   // packed m-state descriptors
    int32_t *d_barr = nullptr;                   // Barr(nint, Nd) bit strings (pci_gpu_form_barr), or null
    int nint = 0;
    uint16_t *d_occ = nullptr;
    int32_t *d_conf_of = nullptr;
    int64_t *d_conf_start = nullptr;
    uint16_t *d_conf_orb = nullptr;
    int64_t *d_adj_ptr = nullptr;
    int32_t *d_adj = nullptr;
    int64_t n_adj = 0;
    // window of the adjacency in use: rows of configurations adj_win_c1 <= c
    // < adj_win_c2 against configurations < adj_win_c0 and themselves (-1:
    // full lower triangle)
    int adj_win_c1 = -1, adj_win_c0 = 0, adj_win_c2 = 0;
    int16_t *d_ms_orb = nullptr;
    int8_t *d_ms_jz = nullptr;
    uint8_t *d_ms_type = nullptr;
    int8_t *d_orb_l = nullptr, *d_orb_j = nullptr;
    // integrals
    double *d_h1 = nullptr;
    double *d_gaunt = nullptr;
    int kdim = 0, ntype = 0, nlx = 0, kbrt = 0;
    unsigned long long *d_htab = nullptr;   // interleaved key/value slots
    int hw = 2;
    unsigned long long hcap = 0;
    // matrices
    Csr H, J, Hfull;
    // device buffers of the last retired H (csr_retire), reused by the next
    // FormH instead of a cudaFree and cudaMalloc of the whole CSR; released
    // by dev_alloc when an allocation fails, and by pci_gpu_destroy
    struct Spare {
        void *rowptr = nullptr, *col = nullptr, *val = nullptr;
        size_t rowptr_bytes = 0, col_bytes = 0, val_bytes = 0;
    } spare;
    double hmin = 0.0;
    int64_t numh = 0, numzero = 0, numj = 0;
    unsigned int *d_err = nullptr;
    // scratch
    void *d_tmp = nullptr;
    size_t tmp_bytes = 0;
    // stats (ms)
    double st_formh = 0, st_formh_count = 0, st_formh_fill = 0, st_formj = 0;
    double st_dvd = 0, st_spmm = 0, st_spmm_calls = 0, st_init = 0;
    double st_adj = 0, st_pairs = 0, st_scanned = 0, st_launches = 0;
    double st_formh_compact = 0, st_formh_padded = 0, st_formh_compact_launches = 0, st_formh_slots = 0;
    bool h_from_tiles = false;  // H was built here by form_h: its rows follow the adjacency tiles
    // H is conf_pt's PT block of pci_gpu_form_h_pt (rows h_pt_lo..h_pt_hi-1,
    // all >= h_pt_nd1, against columns < h_pt_nd0); -1: H is not a PT block
    int64_t h_pt_nd1 = -1, h_pt_nd0 = 0, h_pt_lo = 0, h_pt_hi = 0;
    pci_mlp *corr_model = nullptr;   // learned Davidson correction (not owned)
    int spmm_mode = 0;        // 0 auto, 1 full symmetric copy, 2 lower triangle (env PCI_SPMM)
    int spmm_lower_used = 0;
};

// learned correction model (mlp.cu)
int mlp_forward_device(pci_mlp *m, const float *dX, int64_t n, float *dy, cudaStream_t st);
int mlp_num_inputs(const pci_mlp *m);
namespace mlptc { struct Weights; }
mlptc::Weights mlp_tc_weights(const pci_mlp *m);

// error helpers
int set_err(pci_gpu *h, int code, const std::string &msg);
int cuda_err(pci_gpu *h, cudaError_t e, const char *what);
#define PCI_CUDA(h, call)                                         \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return cuda_err((h), _e, #call);   \
    } while (0)

void *dev_alloc(pci_gpu *h, size_t bytes, int *rc);
void dev_free(void *p);
int ensure_tmp(pci_gpu *h, size_t bytes);
DevSys make_devsys(const pci_gpu *h);

// hbuild.cu
struct RowStatsOut {
    unsigned long long numzero = 0, pairs = 0, scanned = 0;
    double hmin = 0.0;
};
int hb_build_hash(pci_gpu *h, int64_t ngint, int kbrt, int r2_is_f64, const void *rint2,
                  const int32_t *iint2, const int32_t *iint3);
int hb_build_adjacency(pci_gpu *h, int w_c1 = -1, int w_c0 = 0, int w_c2 = 0);
// Squeeze the padded rows of the single-evaluation FormH (row r's entries at
// pptr[r], rowptr[r+1]-rowptr[r] of them) into plain CSR order in place,
// through a buffer of `chunk` entries.
int hb_compact(pci_gpu *h, const int64_t *pptr, const int64_t *rowptr, int64_t nrows, int32_t *col, void *val,
               int vbytes, int64_t chunk);
int hb_form_h(pci_gpu *h, int value_prec, int64_t *numh, int64_t *numzero, double *hmin);
int hb_form_j(pci_gpu *h, int64_t *numj);
int hb_form_h_pt(pci_gpu *h, int64_t nd1, int64_t nd0, int64_t row_lo, int64_t row_hi, int value_prec, int64_t *numh);
double host_gaunt(int nlx, const double *lut, int64_t nlut, int k, double xj1, double xm1,
                  double xj2, double xm2);

// spmm.cu
int sp_build_full(pci_gpu *h);
// Y = (H - hmin I) X on row-major blocks: X[n*ldx + v], Y[n*ldy + v], v < nv
int sp_spmm(pci_gpu *h, const double *X, int ldx, double *Y, int ldy, int nv, cudaStream_t st);
int sp_spmm_f32(pci_gpu *h, const float *X, int ldx, float *Y, int ldy, int nv, cudaStream_t st);
// y = J x restricted to rows/cols < nlim, returned as <x|J|x>
int sp_jav(pci_gpu *h, const double *X, int ldx, int nv, int64_t nlim, double *out_host);
int sp_jav_strided(pci_gpu *h, const double *X, int64_t sn, int64_t sv, int nv, int64_t nlim, double *out_host);
void csr_free(Csr &c);
// Free c, keeping its buffers in h->spare (releasing what the spare held).
void csr_retire(pci_gpu *h, Csr &c);
// A spare buffer of at least `bytes` (0: rowptr, 1: col, 2: val), taken out of
// the spare, or nullptr.
void *spare_take(pci_gpu *h, int which, size_t bytes);
void spare_release(pci_gpu *h);
size_t spare_bytes(const pci_gpu *h);

// davidson.cu
// Samples of the learned correction recorded during a solve (features of
// rows >= Nd0 for each unconverged level and iteration, and after the solve
// their targets); see pci_gpu_davidson_harvest.
struct DvdHarvest {
    float *feat = nullptr, *target = nullptr;
    const double *xref = nullptr;   // reference vectors (Nd x Nlv, column-major) or null: the solve's own
    int64_t cap = 0, count = 0;
};
int dv_run(pci_gpu *h, const pci_dvd_params *p, const double *X0, double *Tk, double *Tj,
           int32_t *Iconverge, double *X, int32_t *iters, double *resid, DvdHarvest *hv = nullptr);
