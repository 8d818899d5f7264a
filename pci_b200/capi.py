"""ctypes binding of libpci_gpu.so (include/pci_gpu.h).

This is the same boundary a Fortran ``pconf`` binds through ISO_C_BINDING:
plain pointers and sizes, 1-based Fortran indices.  There is no fallback: if
the library is missing or fails to load, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB

PCI_OK = 0
ERRORS = {1: "PCI_E_INPUT", 2: "PCI_E_OOM", 3: "PCI_E_MISSING_INTEGRAL", 4: "PCI_E_ORTHO_FAIL",
          5: "PCI_E_TIMEOUT", 6: "PCI_E_CUDA", 7: "PCI_E_STATE", 8: "PCI_E_NOT_CONVERGED"}
PCI_MAT_H, PCI_MAT_J2 = 0, 1
PCI_DVD_FP64, PCI_DVD_FP32, PCI_DVD_LEARNED = 0, 1, 2

EXPORTS = ["pci_gpu_create", "pci_gpu_set_basis", "pci_gpu_set_integrals", "pci_gpu_form_h",
           "pci_gpu_form_j", "pci_gpu_csr_info", "pci_gpu_get_csr", "pci_gpu_set_csr",
           "pci_gpu_davidson", "pci_gpu_j_av", "pci_gpu_j_av_noalloc", "pci_gpu_lsj", "pci_gpu_density", "pci_gpu_transition_density", "pci_gpu_form_csf", "pci_gpu_csf_counts",
           "pci_gpu_csf_to_det", "pci_gpu_pt2", "pci_gpu_pt2_groups", "pci_gpu_form_h_pt", "pci_gpu_form_h_pt_rows", "pci_gpu_jterms", "pci_gpu_stats",
           "pci_gpu_last_error", "pci_gpu_destroy", "pci_mlp_create", "pci_mlp_num_params", "pci_mlp_set_params",
           "pci_mlp_get_params", "pci_mlp_forward", "pci_mlp_loss_grad", "pci_mlp_train", "pci_mlp_last_error",
           "pci_mlp_destroy", "pci_gpu_set_correction_model", "pci_gpu_davidson_harvest", "pci_mlp_forward_occ",
           "pci_gpu_get_csr_rows", "pci_gpu_form_barr", "pci_gpu_bit_compare"]
BATCH_EXPORTS = ["pci_batch_create", "pci_batch_add_block", "pci_batch_set_storage", "pci_batch_set_value_prec",
                 "pci_batch_info", "pci_batch_tune",
                 "pci_batch_variant", "pci_batch_davidson", "pci_batch_vectors", "pci_batch_stats",
                 "pci_batch_last_error", "pci_batch_destroy", "pci_batch_set_correction_model",
                 "pci_batch_set_harvest", "pci_batch_harvest", "pci_batch_probe_reduction"]
PCI_BATCH_FP64, PCI_BATCH_MIXED = 0, 1
PCI_BATCH_CORR_DIAG, PCI_BATCH_CORR_LEARNED = 0, 1
SAMPLE_DTYPE = np.dtype([("blk", np.int32), ("iter", np.int32), ("root", np.int32), ("phase", np.int32),
                         ("row", np.int64), ("x", np.float64), ("r", np.float64), ("theta", np.float64),
                         ("rnorm", np.float64), ("diag", np.float64)])
BATCH_STATUS = {1: "converged", 2: "iteration limit", 3: "no new direction"}


class BatchParams(C.Structure):
    _fields_ = [("nlv", C.c_int32), ("max_sub", C.c_int32), ("keep", C.c_int32), ("max_it", C.c_int32),
                ("tol", C.c_double), ("it_per_graph", C.c_int32), ("spmm_variant", C.c_int32),
                ("precision", C.c_int32), ("stall_max", C.c_int32), ("switch_tol", C.c_double),
                ("correction", C.c_int32), ("pad", C.c_int32)]


class PciError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class DvdParams(C.Structure):
    _fields_ = [("Nlv", C.c_int32), ("N_it", C.c_int32), ("Kl4", C.c_int32), ("Kv", C.c_int32),
                ("Nc4", C.c_int32), ("MaxNd0", C.c_int32), ("mode", C.c_int32), ("KXIJ", C.c_int32),
                ("Crt4", C.c_double), ("XJ_av", C.c_double), ("admix_crit", C.c_double)]


_lib = None


def load(path: str = LIB):
    """Load the library (raises if it is absent: build it with pci_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libpci_gpu.so not found at {path}; run `python -m pci_b200.build`")
    L = C.CDLL(path)
    P = C.c_void_p
    i32, i64, f64 = C.c_int32, C.c_int64, C.c_double
    L.pci_gpu_create.argtypes = [i32, C.POINTER(P)]
    L.pci_gpu_set_basis.argtypes = [P, i32, i64, i32, i32, i32, i32, i32, P, P, P, P, P, P, P, i32, P, f64]
    L.pci_gpu_set_integrals.argtypes = [P, P, i32, i64, P, i64, i32, i32, P, P, P]
    L.pci_gpu_form_h.argtypes = [P, i32, C.POINTER(i64), C.POINTER(i64), C.POINTER(f64)]
    L.pci_gpu_form_j.argtypes = [P, C.POINTER(i64)]
    L.pci_gpu_csr_info.argtypes = [P, i32, C.POINTER(i64), C.POINTER(i64)]
    L.pci_gpu_get_csr.argtypes = [P, i32, P, P, P]
    L.pci_gpu_set_csr.argtypes = [P, i32, i64, i64, P, P, P, f64]
    L.pci_gpu_davidson.argtypes = [P, C.POINTER(DvdParams), P, P, P, P, P, C.POINTER(i32), P]
    L.pci_gpu_j_av.argtypes = [P, P, i32, i64, P]
    L.pci_gpu_lsj.argtypes = [P, P, i32, P, P, P]
    L.pci_gpu_density.argtypes = [P, P, i32, f64, P]
    L.pci_gpu_transition_density.argtypes = [P, P, P, P, f64, P]
    L.pci_gpu_form_csf.argtypes = [P, P, P]
    L.pci_gpu_csf_counts.argtypes = [P, P]
    L.pci_gpu_csf_to_det.argtypes = [P, P, i32, P]
    L.pci_gpu_pt2.argtypes = [P, i64, i64, P, i32, P, i32, P, P]
    L.pci_gpu_pt2_groups.argtypes = [P, i64, i64, P, i32, P, i32, P, i32, P, P, P, P]
    L.pci_gpu_form_h_pt.argtypes = [P, i64, i64, i32, P]
    L.pci_gpu_form_h_pt_rows.argtypes = [P, i64, i64, i64, i64, i32, P]
    L.pci_gpu_j_av_noalloc.argtypes = [P, P, P, i64, P, i64, i32, i64, P, P, C.c_char_p, i32]
    L.pci_mlp_create.argtypes = [i32, i32, i32, C.POINTER(P)]
    L.pci_mlp_num_params.argtypes = [P]
    L.pci_mlp_num_params.restype = i64
    L.pci_mlp_set_params.argtypes = [P, P, i64]
    L.pci_mlp_get_params.argtypes = [P, P, i64]
    L.pci_mlp_forward.argtypes = [P, P, i64, P]
    L.pci_mlp_loss_grad.argtypes = [P, P, P, i64, P, P]
    L.pci_mlp_train.argtypes = [P, P, P, i64, i32, i32, C.c_float, i32, P]
    L.pci_mlp_last_error.argtypes = [P]
    L.pci_mlp_last_error.restype = C.c_char_p
    L.pci_mlp_destroy.argtypes = [P]
    L.pci_mlp_destroy.restype = None
    L.pci_gpu_set_correction_model.argtypes = [P, P]
    L.pci_gpu_davidson_harvest.argtypes = [P, C.POINTER(DvdParams), P, P, P, i64, C.POINTER(i64), P, P,
                                           C.POINTER(i32)]
    L.pci_gpu_jterms.argtypes = [P, P, i32]
    L.pci_gpu_jterms.restype = i32
    L.pci_gpu_stats.argtypes = [P, P, i32]
    L.pci_gpu_stats.restype = i32
    L.pci_gpu_last_error.argtypes = [P]
    L.pci_gpu_last_error.restype = C.c_char_p
    L.pci_gpu_destroy.argtypes = [P]
    L.pci_gpu_destroy.restype = None
    L.pci_batch_create.argtypes = [i32, C.POINTER(P)]
    L.pci_batch_add_block.argtypes = [P, P, C.POINTER(i32)]
    L.pci_batch_info.argtypes = [P, C.POINTER(i32), C.POINTER(i64), C.POINTER(i64)]
    L.pci_batch_set_storage.argtypes = [P, i32]
    L.pci_batch_set_value_prec.argtypes = [P, i32]
    L.pci_batch_tune.argtypes = [P, i32, C.c_char_p, C.POINTER(i32), C.POINTER(f64), C.POINTER(i32)]
    L.pci_batch_variant.argtypes = [i32, C.POINTER(i32), C.POINTER(i32)]
    L.pci_batch_davidson.argtypes = [P, C.POINTER(BatchParams), P, P, P, P, C.POINTER(i32)]
    L.pci_batch_vectors.argtypes = [P, i32, P]
    L.pci_batch_stats.argtypes = [P, P, i32]
    L.pci_batch_last_error.argtypes = [P]
    L.pci_batch_last_error.restype = C.c_char_p
    L.pci_batch_destroy.argtypes = [P]
    L.pci_batch_destroy.restype = None
    L.pci_batch_set_correction_model.argtypes = [P, P]
    L.pci_batch_set_harvest.argtypes = [P, i32, i64, i32]
    L.pci_batch_harvest.argtypes = [P, P, i64, C.POINTER(i64)]
    L.pci_batch_probe_reduction.argtypes = [i32, i64, i32, C.POINTER(f64)]
    L.pci_mlp_forward_occ.argtypes = [P, P, P, i64, P]
    L.pci_gpu_get_csr_rows.argtypes = [P, i32, i64, i64, P, P, P]
    L.pci_gpu_form_barr.argtypes = [P, C.POINTER(i32), P]
    L.pci_gpu_bit_compare.argtypes = [P, i64, P, P, P, P, P]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Engine:
    """One device handle: the drop-in for pconf's FormH, FormJ and Diag4 calls."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.h = C.c_void_p()
        rc = self.L.pci_gpu_create(device, C.byref(self.h))
        self._check(rc)

    def _check(self, rc):
        if rc != PCI_OK:
            msg = self.L.pci_gpu_last_error(self.h).decode() if self.h else ""
            raise PciError(rc, msg)

    def close(self):
        if self.h:
            self.L.pci_gpu_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- inputs ---------------------------------------------------------
    def set_basis(self, sysm):
        b = sysm.basis
        nsu = sysm.nsu
        arr = lambda x: np.ascontiguousarray(x, dtype=np.int32)
        self._basis = dict(iarr=arr(sysm.iarr), nh=arr(sysm.nh), jz=arr(sysm.jz), nn=arr(b.nn[:nsu]),
                           kk=arr(b.kk[:nsu]), ll=arr(b.ll[:nsu]), jj=arr(b.jj[:nsu]), ndc=arr(sysm.ndc))
        k = self._basis
        rc = self.L.pci_gpu_set_basis(self.h, sysm.ne, sysm.nd, sysm.nst, nsu, b.nso, sysm.nx, sysm.mj,
                                      _p(k["iarr"]), _p(k["nh"]), _p(k["jz"]), _p(k["nn"]), _p(k["kk"]),
                                      _p(k["ll"]), _p(k["jj"]), sysm.nc, _p(k["ndc"]), float(sysm.gj))
        self._check(rc)
        self._nd = int(sysm.nd)
        self._nst = int(sysm.nst)

    def set_integrals(self, sysm):
        hl = np.ascontiguousarray(sysm.hint_lut, np.float64)
        gl = np.ascontiguousarray(sysm.gaunt_lut, np.float64)
        r2 = np.ascontiguousarray(sysm.rint2)
        i2 = np.ascontiguousarray(sysm.iint2, np.int32)
        i3 = np.ascontiguousarray(sysm.iint3, np.int32)
        rc = self.L.pci_gpu_set_integrals(self.h, _p(hl), sysm.nlx, gl.size, _p(gl), sysm.ngint, sysm.kbrt,
                                          1 if r2.dtype == np.float64 else 0, _p(r2), _p(i2), _p(i3))
        self._check(rc)

    def load_system(self, sysm):
        self.set_basis(sysm)
        self.set_integrals(sysm)

    # --- FormH / FormJ --------------------------------------------------
    def form_h(self, value_prec: int = 64):
        numh, nz, hmin = C.c_int64(), C.c_int64(), C.c_double()
        self._check(self.L.pci_gpu_form_h(self.h, value_prec, C.byref(numh), C.byref(nz), C.byref(hmin)))
        return numh.value, nz.value, hmin.value

    def form_j(self):
        n = C.c_int64()
        self._check(self.L.pci_gpu_form_j(self.h, C.byref(n)))
        return n.value

    def get_csr(self, which: int = PCI_MAT_H):
        nrows, nnz = C.c_int64(), C.c_int64()
        self._check(self.L.pci_gpu_csr_info(self.h, which, C.byref(nrows), C.byref(nnz)))
        rowptr = np.zeros(nrows.value + 1, np.int64)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value, np.float64)
        self._check(self.L.pci_gpu_get_csr(self.h, which, _p(rowptr), _p(col), _p(val)))
        return rowptr, col, val

    def form_barr(self, copy=True):
        """FormBarr on the device; returns Barr as [Nd, nint] int32 (None without copy)."""
        nint = C.c_int32()
        self._check(self.L.pci_gpu_form_barr(self.h, C.byref(nint), None))
        if not copy:
            return None
        nd = self._nd
        out = np.zeros((nd, nint.value), np.int32)
        self._check(self.L.pci_gpu_form_barr(self.h, C.byref(nint), _p(out)))
        return out

    def bit_compare(self, pairs):
        """compare_bit_dets + get_det_indexes on the device for 1-based pairs [n, 2]:
        (ndiffs, is, idx1 [n, 3], idx2 [n, 3])."""
        pairs = np.ascontiguousarray(pairs, np.int64)
        n = pairs.shape[0]
        nf = np.zeros(n, np.int32)
        isg = np.zeros(n, np.int32)
        i1 = np.zeros((n, 3), np.int32)
        i2 = np.zeros((n, 3), np.int32)
        self._check(self.L.pci_gpu_bit_compare(self.h, n, _p(pairs), _p(nf), _p(isg), _p(i1), _p(i2)))
        return nf, isg, i1, i2

    def csr_info(self, which: int = PCI_MAT_H):
        """(rows, stored elements) of a resident matrix."""
        nrows, nnz = C.c_int64(), C.c_int64()
        self._check(self.L.pci_gpu_csr_info(self.h, which, C.byref(nrows), C.byref(nnz)))
        return nrows.value, nnz.value

    def get_csr_rows(self, which: int, row_lo: int, row_hi: int):
        """Rows row_lo..row_hi (1-based, inclusive) of a resident matrix:
        (rowptr from 0, 1-based col, val as double)."""
        n = row_hi - row_lo + 1
        rowptr = np.zeros(n + 1, np.int64)
        self._check(self.L.pci_gpu_get_csr_rows(self.h, which, row_lo, row_hi, _p(rowptr), None, None))
        col = np.zeros(rowptr[-1], np.int32)
        val = np.zeros(rowptr[-1], np.float64)
        self._check(self.L.pci_gpu_get_csr_rows(self.h, which, row_lo, row_hi, _p(rowptr), _p(col), _p(val)))
        return rowptr, col, val

    def set_csr(self, which, rowptr, col, val, hmin=0.0):
        rowptr = np.ascontiguousarray(rowptr, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        self._check(self.L.pci_gpu_set_csr(self.h, which, rowptr.size - 1, col.size, _p(rowptr), _p(col),
                                           _p(val), float(hmin)))

    # --- Diag4 ----------------------------------------------------------
    def davidson(self, nd: int, Nlv: int, N_it: int = 200, Crt4: float = 1e-8, Kl4: int = 1, Kv: int = 4,
                 Nc4: int = 0, MaxNd0: int = 3000, mode: int = PCI_DVD_FP64, XJ_av: float = 0.0,
                 admix_crit: float = 1e-6, X0=None, want_vectors: bool = True):
        p = DvdParams(Nlv, N_it, Kl4, Kv, Nc4, MaxNd0, mode, 0, Crt4, XJ_av, admix_crit)
        Tk = np.zeros(Nlv)
        Tj = np.zeros(Nlv)
        ic = np.zeros(Nlv, np.int32)
        res = np.zeros(Nlv)
        X = np.zeros((Nlv, nd)) if want_vectors else None   # column-major Nd x Nlv == row-major Nlv x Nd
        x0 = None if X0 is None else np.ascontiguousarray(np.asarray(X0).T, np.float64)
        iters = C.c_int32()
        self._check(self.L.pci_gpu_davidson(self.h, C.byref(p), _p(x0), _p(Tk), _p(Tj), _p(ic), _p(X),
                                            C.byref(iters), _p(res)))
        return dict(Tk=Tk, Tj=Tj, Iconverge=ic, X=None if X is None else X.T, iterations=iters.value, resid=res)

    def j_av(self, X, nlim=None):
        """J of each column of X (Nd x nv) from <x|J^2|x> over rows/columns <= nlim."""
        X = np.asarray(X, np.float64)
        if X.ndim == 1:
            X = X[:, None]
        nd, nv = X.shape
        xc = np.ascontiguousarray(X.T)        # column-major Nd x nv
        out = np.zeros(nv)
        self._check(self.L.pci_gpu_j_av(self.h, _p(xc), nv, nd if nlim is None else nlim, _p(out)))
        return out

    def lsj(self, X):
        """(J, L, S) of each column of X (Nd x nv), as pconf's kLSJ = 1 step
        computes them (pci_gpu_lsj)."""
        X = np.asarray(X, np.float64)
        if X.ndim == 1:
            X = X[:, None]
        nd, nv = X.shape
        xc = np.ascontiguousarray(X.T)        # column-major Nd x nv
        xj, xl, xs = np.zeros(nv), np.zeros(nv), np.zeros(nv)
        self._check(self.L.pci_gpu_lsj(self.h, _p(xc), nv, _p(xj), _p(xl), _p(xs)))
        return xj, xl, xs

    def density(self, X, trd=1e-10):
        """FormDM's one-particle density matrix of each column of X: [nv, Nst, Nst]
        with entry [v, i, j] = Ro(i+1, j+1)."""
        X = np.asarray(X, np.float64)
        if X.ndim == 1:
            X = X[:, None]
        nd, nv = X.shape
        xc = np.ascontiguousarray(X.T)
        nst = self._nst
        ro = np.zeros((nv, nst, nst))
        self._check(self.L.pci_gpu_density(self.h, _p(xc), nv, float(trd), _p(ro)))
        return np.transpose(ro, (0, 2, 1))             # column-major per vector -> [v, i, j]

    def transition_density(self, initial, b_initial, b_final, trd=1e-10):
        """FormTM's transition density from a level of `initial` (another
        Engine holding the initial basis) to a level of this engine's basis:
        [Nst, Nst] with entry [i, j] = Ro(i+1, j+1), i the initial m-state."""
        bi = np.ascontiguousarray(b_initial, np.float64)
        bf = np.ascontiguousarray(b_final, np.float64)
        ro = np.zeros(self._nst * self._nst)
        self._check(self.L.pci_gpu_transition_density(initial.h, self.h, _p(bi), _p(bf), float(trd), _p(ro)))
        return ro.reshape(self._nst, self._nst).T

    def form_csf(self):
        """jbasis + formh_sym on the device: the CSF Hamiltonian replaces the
        determinant one (needs form_h(64) and form_j first); (ncsf, stored
        elements)."""
        n, nnz = C.c_int64(), C.c_int64()
        self._check(self.L.pci_gpu_form_csf(self.h, C.byref(n), C.byref(nnz)))
        self._ncsf = n.value
        return n.value, nnz.value

    def csf_counts(self, nc):
        out = np.zeros(nc, np.int32)
        self._check(self.L.pci_gpu_csf_counts(self.h, _p(out)))
        return out

    def csf_to_det(self, Y):
        """unsym: determinant vectors (Nd x nv) from CSF vectors (Ncsf x nv)."""
        Y = np.asarray(Y, np.float64)
        if Y.ndim == 1:
            Y = Y[:, None]
        nv = Y.shape[1]
        yc = np.ascontiguousarray(Y.T)
        out = np.zeros((nv, self._nd))
        self._check(self.L.pci_gpu_csf_to_det(self.h, _p(yc), nv, _p(out)))
        return out.T

    def form_h_pt(self, nd1: int, nd0: int, value_prec: int = 64, rows=None) -> int:
        """conf_pt's PT block (rows beyond nd1, or the PT rows rows[0] to
        rows[1]-1, against the first nd0 columns) in place of H; returns the
        stored element count."""
        n = C.c_int64()
        if rows is None:
            self._check(self.L.pci_gpu_form_h_pt(self.h, nd1, nd0, value_prec, C.byref(n)))
        else:
            self._check(self.L.pci_gpu_form_h_pt_rows(self.h, nd1, nd0, int(rows[0]), int(rows[1]), value_prec,
                                                      C.byref(n)))
        return n.value

    def pt2_groups(self, nd1, X0, E, groups, avg_diag=False):
        """pt2 with PTE's sums per group of PT rows (groups: ascending
        determinant offsets, e.g. pci_b200.system.nr_configurations): returns
        dE [nv], dEg and dVg [ngroups, nv]."""
        X0 = np.asarray(X0, np.float64)
        if X0.ndim == 1:
            X0 = X0[:, None]
        nd0, nv = X0.shape
        xc = np.ascontiguousarray(X0.T)
        e = np.ascontiguousarray(E, np.float64)
        g = np.ascontiguousarray(groups, np.int64)
        ng = g.size - 1
        de = np.zeros(nv)
        deg = np.zeros((max(ng, 1), nv))
        dvg = np.zeros((max(ng, 1), nv))
        self._check(self.L.pci_gpu_pt2_groups(self.h, nd1, nd0, _p(xc), nv, _p(e), 1 if avg_diag else 0, _p(g), ng,
                                              _p(de), _p(deg), _p(dvg), None))
        return de, deg[:ng], dvg[:ng]

    def pt2_ranges(self, nd1, X0, E, ranges, avg_diag=False, want_vectors=False):
        """pt2 over the PT space in row ranges (pci_b200.system.pt_row_ranges),
        one PT block at a time: the sums of the ranges' dE (and first-order
        coefficients) are the whole PT space's."""
        nd0 = np.asarray(X0).reshape(np.asarray(X0).shape[0], -1).shape[0]
        de, c = None, None
        for lo, hi in ranges:
            self.form_h_pt(nd1, nd0, 64, rows=(lo, hi))
            r = self.pt2(nd1, X0, E, avg_diag=avg_diag, want_vectors=want_vectors)
            d_r, c_r = r if want_vectors else (r, None)
            de = d_r if de is None else de + d_r
            if want_vectors:
                c = c_r if c is None else c + c_r
        return (de, c) if want_vectors else de

    def pt2(self, nd1, X0, E, avg_diag=False, want_vectors=False):
        """Second-order CI+PT (conf_pt's PTE) on the resident H: X0 (nd0 x nv)
        the CI vectors over the first nd0 determinants, E their energies;
        returns dE (and the first-order coefficients, Nd x nv)."""
        X0 = np.asarray(X0, np.float64)
        if X0.ndim == 1:
            X0 = X0[:, None]
        nd0, nv = X0.shape
        xc = np.ascontiguousarray(X0.T)
        e = np.ascontiguousarray(E, np.float64)
        de = np.zeros(nv)
        xpt = np.zeros((nv, self._nd)) if want_vectors else None
        self._check(self.L.pci_gpu_pt2(self.h, nd1, nd0, _p(xc), nv, _p(e), 1 if avg_diag else 0, _p(de),
                                       _p(xpt) if xpt is not None else None))
        return (de, xpt.T) if want_vectors else de

    def set_correction_model(self, mlp):
        """Attach a trained Mlp for mode=PCI_DVD_LEARNED (None detaches)."""
        self._check(self.L.pci_gpu_set_correction_model(self.h, None if mlp is None else mlp.m))
        self._model = mlp

    def davidson_harvest(self, nd, nsu, Nlv, N_it=30, MaxNd0=3000, Xref=None, cap=None, Crt4=1e-8):
        """FP64 Davidson recording samples for the correction model: returns
        (features [n, Nsu+2], targets [n], result dict)."""
        p = DvdParams(Nlv, N_it, 1, 4, 0, MaxNd0, PCI_DVD_FP64, 0, Crt4, 0.0, 0.0)
        cap = cap if cap is not None else N_it * Nlv * nd
        nin = nsu + 2
        feat = np.zeros((cap, nin), np.float32)
        targ = np.zeros(cap, np.float32)
        xr = None if Xref is None else np.ascontiguousarray(np.asarray(Xref, np.float64).T)
        cnt = C.c_int64()
        Tk = np.zeros(Nlv)
        ic = np.zeros(Nlv, np.int32)
        iters = C.c_int32()
        self._check(self.L.pci_gpu_davidson_harvest(self.h, C.byref(p), _p(xr), _p(feat), _p(targ), cap,
                                                    C.byref(cnt), _p(Tk), _p(ic), C.byref(iters)))
        n = min(cnt.value, cap)
        return feat[:n], targ[:n], dict(Tk=Tk, Iconverge=ic, iterations=iters.value, count=cnt.value)

    def jterms(self):
        """Jt(1:Njd) of the current basis (sorted 2J of the terms present)."""
        n = self.L.pci_gpu_jterms(self.h, None, 0)
        if n < 0:
            raise PciError(7, "jterms before set_basis")
        out = np.zeros(max(n, 1), np.int32)
        self.L.pci_gpu_jterms(self.h, _p(out), n)
        return out[:n].tolist()

    def stats(self):
        out = np.zeros(15)
        n = self.L.pci_gpu_stats(self.h, _p(out), 15)
        keys = ["formh_ms", "formh_count_ms", "formh_fill_ms", "formj_ms", "davidson_ms", "spmm_ms",
                "spmm_calls", "init_ms", "adjacency_ms", "pairs", "scanned", "formh_launches",
                "formh_compact_ms", "formh_single_eval", "formh_slots"]
        return dict(zip(keys[:n], out[:n].tolist()))


class Mlp:
    """The learned-correction network on one device (pci_mlp_* of the C ABI)."""

    def __init__(self, nin: int, device: int = 0, seed: int = 0):
        self.L = load()
        self.m = C.c_void_p()
        rc = self.L.pci_mlp_create(device, nin, seed, C.byref(self.m))
        if rc != PCI_OK:
            raise PciError(rc, "pci_mlp_create failed")
        self.nin = nin
        self.nparam = int(self.L.pci_mlp_num_params(self.m))

    def _check(self, rc):
        if rc != PCI_OK:
            raise PciError(rc, self.L.pci_mlp_last_error(self.m).decode())

    def params(self):
        p = np.zeros(self.nparam, np.float32)
        self._check(self.L.pci_mlp_get_params(self.m, _p(p), self.nparam))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.L.pci_mlp_set_params(self.m, _p(p), p.size))

    def forward(self, X):
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(X.shape[0], np.float32)
        self._check(self.L.pci_mlp_forward(self.m, _p(X), X.shape[0], _p(y)))
        return y

    def forward_occ(self, orbs, f):
        """Tensor-core forward from compact inputs: orbs [n, 8] uint8 (0xff empty), f [n, 3]."""
        orbs = np.ascontiguousarray(orbs, np.uint8)
        f = np.ascontiguousarray(f, np.float32)
        y = np.zeros(orbs.shape[0], np.float32)
        self._check(self.L.pci_mlp_forward_occ(self.m, _p(orbs), _p(f), orbs.shape[0], _p(y)))
        return y

    def loss_grad(self, X, T):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = C.c_float()
        g = np.zeros(self.nparam, np.float32)
        self._check(self.L.pci_mlp_loss_grad(self.m, _p(X), _p(T), X.shape[0], C.byref(loss), _p(g)))
        return float(loss.value), g

    def train(self, X, T, epochs=10, batch=4096, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = C.c_float()
        self._check(self.L.pci_mlp_train(self.m, _p(X), _p(T), X.shape[0], epochs, batch, lr, seed,
                                         C.byref(loss)))
        return float(loss.value)

    def close(self):
        if self.m:
            self.L.pci_mlp_destroy(self.m)
            self.m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_reduction(device, rows, nv):
    """Measured GB/s of random FP64 reductions in the SpMM's transpose-part pattern."""
    L = load()
    g = C.c_double()
    rc = L.pci_batch_probe_reduction(device, rows, nv, C.byref(g))
    if rc != PCI_OK:
        raise PciError(rc, "pci_batch_probe_reduction failed")
    return g.value


def batch_variants():
    """(lanes per row, thread blocks per SM) of every SpMM variant of the batched form."""
    L = load()
    out, v = [], 0
    a, b = C.c_int32(), C.c_int32()
    while L.pci_batch_variant(v, C.byref(a), C.byref(b)) == PCI_OK:
        out.append((a.value, b.value))
        v += 1
    return out


class Batch:
    """Many independent CI blocks solved together (pci_batch_* of include/pci_batch.h)."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.b = C.c_void_p()
        self.device = device
        rc = self.L.pci_batch_create(device, C.byref(self.b))
        if rc != PCI_OK:
            msg = self.L.pci_batch_last_error(self.b).decode() if self.b else "pci_batch_create failed"
            raise PciError(rc, msg)
        self.sizes = []

    def _check(self, rc):
        if rc != PCI_OK:
            raise PciError(rc, self.L.pci_batch_last_error(self.b).decode())

    def add_engine(self, eng):
        """Take over the Hamiltonian resident in an Engine as the next block."""
        nd = C.c_int64()
        nnz = C.c_int64()
        self.L.pci_gpu_csr_info(eng.h, PCI_MAT_H, C.byref(nd), C.byref(nnz))
        idx = C.c_int32()
        self._check(self.L.pci_batch_add_block(self.b, eng.h, C.byref(idx)))
        self.sizes.append(int(nd.value))
        return idx.value

    def add_system(self, sysm, value_prec: int = 32):
        """Build a system's H on the device (FormH) and add it as the next block."""
        with Engine(self.device) as e:
            e.load_system(sysm)
            e.form_h(value_prec)
            return self.add_engine(e)

    def add_csr(self, rowptr, col, val):
        """Add a lower-triangle CSR held on the host (0-based rowptr, 1-based col)."""
        with Engine(self.device) as e:
            e.set_csr(PCI_MAT_H, rowptr, col, val)
            return self.add_engine(e)

    def set_value_prec(self, value_prec: int):
        """32: blocks rounded to FP32 when added (default); 64: kept as built;
        48: split into FP32 hi + lo pairs (for the mixed-precision form)."""
        self._check(self.L.pci_batch_set_value_prec(self.b, value_prec))

    def set_storage(self, mode: int):
        """0: lower triangles only (default), 1: full symmetric copies where memory allows."""
        self._check(self.L.pci_batch_set_storage(self.b, mode))

    def info(self):
        n, r, z = C.c_int32(), C.c_int64(), C.c_int64()
        self._check(self.L.pci_batch_info(self.b, C.byref(n), C.byref(r), C.byref(z)))
        return n.value, r.value, z.value

    def tune(self, nv: int, cache=None):
        v, ms, fc = C.c_int32(), C.c_double(), C.c_int32()
        self._check(self.L.pci_batch_tune(self.b, nv, cache.encode() if cache else None, C.byref(v),
                                          C.byref(ms), C.byref(fc)))
        return v.value, ms.value, bool(fc.value)

    def davidson(self, nlv=6, max_sub=48, keep=None, max_it=300, tol=1e-8, it_per_graph=4, spmm_variant=-1,
                 precision=PCI_BATCH_FP64, switch_tol=1e-5, stall_max=0, correction=PCI_BATCH_CORR_DIAG):
        nblk = len(self.sizes)
        p = BatchParams(nlv, max_sub, keep if keep is not None else 2 * nlv, max_it, tol, it_per_graph,
                        spmm_variant, precision, stall_max, switch_tol, correction, 0)
        E = np.zeros((nblk, nlv))
        rn = np.zeros((nblk, nlv))
        it = np.zeros(nblk, np.int32)
        st = np.zeros(nblk, np.int32)
        gl = C.c_int32()
        self._check(self.L.pci_batch_davidson(self.b, C.byref(p), _p(E), _p(rn), _p(it), _p(st), C.byref(gl)))
        self.nlv = nlv
        return dict(E=E, rnorm=rn, iters=it, status=st, graph_launches=gl.value)

    def vectors(self, blk):
        X = np.zeros((self.nlv, self.sizes[blk]))
        self._check(self.L.pci_batch_vectors(self.b, blk, _p(X)))
        return X.T

    def stats(self):
        out = np.zeros(10)
        self._check(self.L.pci_batch_stats(self.b, _p(out), 10))
        keys = ["total_ms", "iterations", "spmm_ms", "spmm_variant", "setup_ms", "launches_per_iteration",
                "full_share", "spmm32_ms", "fp32_iterations", "switched_blocks"]
        return dict(zip(keys, out.tolist()))

    def set_correction_model(self, mlp):
        """Attach a trained Mlp for correction=PCI_BATCH_CORR_LEARNED (None detaches)."""
        self._check(self.L.pci_batch_set_correction_model(self.b, mlp.m if mlp is not None else None))
        self._model = mlp

    def set_harvest(self, rows_per_block, capacity, seed=0):
        """Record training samples in the next solves (0 rows: off)."""
        self._check(self.L.pci_batch_set_harvest(self.b, rows_per_block, capacity, seed))
        self._hv_cap = int(capacity) if rows_per_block > 0 else 0

    def harvest(self):
        """Samples of the last solve as a structured array (SAMPLE_DTYPE), and the
        number the solve produced (above the capacity given to set_harvest, the
        samples past the capacity were dropped and are not in the array)."""
        cnt = C.c_int64()
        self._check(self.L.pci_batch_harvest(self.b, None, 0, C.byref(cnt)))
        n = min(cnt.value, getattr(self, "_hv_cap", 0))
        out = np.zeros(n, SAMPLE_DTYPE)
        if n:
            self._check(self.L.pci_batch_harvest(self.b, out.ctypes.data_as(C.c_void_p), n, C.byref(cnt)))
        return out, int(cnt.value)

    def close(self):
        if self.b:
            self.L.pci_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
