/* pci_io.h -- readers and writers of the pconf files the drop-in keeps
 * compatible: the CSR matrix stream pCONF.HIJ / pCONF.JJJ, the eigenvector
 * file CONF.XIJ, the energy table CONF.RES, the determinant list CONF.DET,
 * the angular-factor file CONF.GNT and the radial-integral file CONF.INT.
 *
 * Host code only (no device, no CUDA context needed).  "Sequential" files
 * are Fortran unformatted sequential files as gfortran writes them: every
 * record is framed by a 4-byte little-endian length before and after it;
 * records longer than 2^31-1 bytes are split into subrecords whose leading
 * marker is negative when another subrecord follows (and whose trailing
 * marker is negative when one precedes).  "Stream" files have no framing.
 *
 * All functions return PCI_OK (0) or PCI_E_INPUT (1, bad arguments or a
 * file whose layout does not match) and write a message into errbuf (when
 * errbuf is not NULL, at most errlen bytes including the terminating NUL).
 */
#ifndef PCI_IO_H
#define PCI_IO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- pCONF.HIJ / pCONF.JJJ (stream) --------------------------------------
 * Layout of WriteMatrixCSR (src/matrix_io.f90:689-799): int64 Nd, int64 nnz,
 * int64 rowptr(0:Nd) (0-based prefix), int32 col(nnz) (1-based),
 * real val(nnz) with val_bytes = 8 (type_real = dp) or 4 (sp). */
int pci_io_write_csr(const char *path, int64_t nd, int64_t nnz, const int64_t *rowptr, const int32_t *col,
                     const void *val, int32_t val_bytes, char *errbuf, int32_t errlen);
/* Header of a CSR stream: Nd and nnz; *val_bytes is inferred from the file
 * size (8 or 4). */
int pci_io_read_csr_header(const char *path, int64_t *nd, int64_t *nnz, int32_t *val_bytes, char *errbuf,
                           int32_t errlen);
/* Body of a CSR stream into caller arrays sized from the header (the reader
 * of src/matrix_io.f90:801-939 with npes = 1).  Checks that rowptr starts at
 * 0, never decreases and ends at nnz. */
int pci_io_read_csr(const char *path, int64_t nd, int64_t nnz, int64_t *rowptr, int32_t *col, void *val,
                    int32_t val_bytes, char *errbuf, int32_t errlen);

/* ---- CONF.HIJ / CONF.JJJ (stream) ------------------------------------------
 * The sorted element stream that pCI's sort program writes from pconf's
 * parallel matrix file (src/sort.f90:16-80) and that pol / ine read
 * (ReadHIJ, src/pol.f90:766-797): int64 count, then count records of int32
 * row, int32 column (1-based, column <= row) and real64 value, rows
 * ascending and columns ascending within a row, exact zeros left out.
 * rowptr/col/val are a lower-triangle CSR as pci_gpu_get_csr returns it
 * (0-based row prefix, 1-based columns). */
int pci_io_write_hij(const char *path, int64_t nd, const int64_t *rowptr, const int32_t *col, const double *val,
                     char *errbuf, int32_t errlen);
/* The same stream written in row ranges (to stream a matrix too large for
 * host memory, e.g. from pci_gpu_get_csr_rows): rows row0+1 .. row0+nrows of
 * a CSR slice (rowptr[nrows+1], any base; col/val indexed from rowptr[0]).
 * row0 = 0 creates the file; later ranges must follow in row order. */
int pci_io_append_hij(const char *path, int64_t row0, int64_t nrows, const int64_t *rowptr, const int32_t *col,
                      const double *val, char *errbuf, int32_t errlen);
/* *count = the file's record count; up to cap records into row/col/val. */
int pci_io_read_hij(const char *path, int64_t cap, int32_t *row, int32_t *col, double *val, int64_t *count,
                    char *errbuf, int32_t errlen);

/* ---- CONF.XIJ (sequential) -----------------------------------------------
 * One record per level n: Tk(n) (r8), Tj(n) (r8), Nd (i4), x(1:Nd) (r8), as
 * WriteXIJ / WriteFinalXIJ write them (src/pconf.F90:2536-2602).  X is
 * column-major Nd x nlv. */
int pci_io_write_xij(const char *path, int32_t nlv, int64_t nd, const double *Tk, const double *Tj, const double *X,
                     char *errbuf, int32_t errlen);
/* Reads up to nlv_max records with this Nd into Tk, Tj, X (column-major,
 * leading dimension nd); *nread receives the number read. */
int pci_io_read_xij(const char *path, int32_t nlv_max, int64_t nd, double *Tk, double *Tj, double *X,
                    int32_t *nread, char *errbuf, int32_t errlen);

/* ---- CONF.RES (text) -----------------------------------------------------
 * The energy table PrintEnergies writes (src/pconf.F90:3152-3242) for pure
 * CI in the determinant basis (Ksig = 0, kCSF = 0, no isotope shift): header
 * with the interaction label (kbrt 0 Coulomb, 1 Gaunt, 2 Breit), Nc, Nd and
 * Gj, then one line (3X,I3,F14.9,F14.8,F18.6,F15.2) per level: n, J, EV, ET,
 * DEL(cm^-1), where EV = Tk + 4 Gj J(J+1), ET = EV - Ecore and
 * DEL = (EV(1) - EV(n)) * 2 * 109737.315709.  Appends when append != 0. */
int pci_io_write_res(const char *path, int32_t append, int32_t kbrt, int32_t nc, int64_t nd, double gj, int32_t nlv,
                     const double *Tj, const double *Tk, double ecore, char *errbuf, int32_t errlen);

/* ---- CONF.DET (sequential) -----------------------------------------------
 * Wdet / Rdet (src/determinants.f90:448-500): record 1 Nd, Nsu (i4); then one
 * record Iarr(1:Ne, i) (i4) per determinant.  Iarr is column-major Ne x Nd. */
int pci_io_write_det(const char *path, int32_t ne, int64_t nd, int32_t nsu, const int32_t *Iarr, char *errbuf,
                     int32_t errlen);
int pci_io_read_det_header(const char *path, int64_t *nd, int32_t *nsu, int32_t *ne, char *errbuf, int32_t errlen);
int pci_io_read_det(const char *path, int32_t ne, int64_t nd, int32_t *Iarr, char *errbuf, int32_t errlen);

/* ---- CONF.GNT (sequential) -----------------------------------------------
 * Records Nlx, Ngaunt; num_gaunts_per_partial_wave(Nlx+1); In(Ngaunt) (i4);
 * Gnt(Ngaunt) (r8) (src/breit.f90:96-101, read at src/pconf.F90:383-406).
 * The LUT helper builds GauntLUT(0:max(In)) = Gnt at In as BuildGauntLUT
 * (src/integrals.f90:702-715). */
int pci_io_write_gnt(const char *path, int32_t nlx, int32_t ngaunt, const int32_t *per_wave, const int32_t *In,
                     const double *Gnt, char *errbuf, int32_t errlen);
int pci_io_read_gnt_header(const char *path, int32_t *nlx, int32_t *ngaunt, char *errbuf, int32_t errlen);
int pci_io_read_gnt(const char *path, int32_t nlx, int32_t ngaunt, int32_t *per_wave, int32_t *In, double *Gnt,
                    char *errbuf, int32_t errlen);
/* lut has max(In)+1 entries (*nlut on return when lut is NULL). */
int pci_io_gaunt_lut(int32_t ngaunt, const int32_t *In, const double *Gnt, double *lut, int64_t *nlut);

/* ---- CONF.INT (sequential) -----------------------------------------------
 * The records Rint reads (src/integrals.f90:35-106; written by
 * src/pbasc.f90:1170-1189): Ns, Nso, Nsp, Nsx (i4), Ecore (r8);
 * (Nn, Kk, Ll, Jj) x Nsx (i4); a record skipped by the reader; Nhint, Kbrt
 * (i4); Rint1(Nhint) (r8); Iint1(Nhint) (i4); Ngint (i8), Nlist (i4),
 * nrd = Nx^2 (i4); Rint2 (r4, or r8 with r2_bytes = 8; two values per
 * integral when Kbrt > 0); Iint2(Ngint), Iint3(Ngint) (i4); IntOrd(nrd) (i8).
 * The optional isotope-shift records are not read. */
typedef struct {
    int32_t ns, nso, nsp, nsx;
    double ecore;
    int32_t nhint, kbrt;
    int64_t ngint;
    int32_t nlist, nrd;
    int32_t r2_bytes;   /* 4 or 8, from the Rint2 record length */
} pci_int_header;
int pci_io_read_int_header(const char *path, pci_int_header *hdr, char *errbuf, int32_t errlen);
/* Arrays sized from the header: NnKkLlJj 4 x nsx (interleaved per orbital as
 * in the file), Rint1/Iint1 nhint, Rint2 ngint x (kbrt ? 2 : 1) of r2_bytes,
 * Iint2/Iint3 ngint, IntOrd nrd.  Any pointer may be NULL to skip a field. */
int pci_io_read_int(const char *path, const pci_int_header *hdr, int32_t *NnKkLlJj, double *Rint1, int32_t *Iint1,
                    void *Rint2, int32_t *Iint2, int32_t *Iint3, int64_t *IntOrd, char *errbuf, int32_t errlen);
int pci_io_write_int(const char *path, const pci_int_header *hdr, const int32_t *NnKkLlJj, const double *Rint1,
                     const int32_t *Iint1, const void *Rint2, const int32_t *Iint2, const int32_t *Iint3,
                     const int64_t *IntOrd, char *errbuf, int32_t errlen);
/* HintLUT(Nx*Nx) = Rint1 at Iint1 (1-based), as BuildHintLUT
 * (src/integrals.f90:663-674). */
int pci_io_hint_lut(int32_t nhint, const double *Rint1, const int32_t *Iint1, int32_t nx, double *lut);

#ifdef __cplusplus
}
#endif

#endif
