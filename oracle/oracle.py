"""Python side of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (built from ``pci_oracle.c`` by ``build()``)
and restates pconf's Davidson driver ``Diag4`` and the ``davidson`` module in
numpy (npes = 1).  Only tests, the smoke check and the CPU-baseline leg of the
benchmark use this module; the product path never imports it.

Parity status: unpinned against the reference itself (a Fortran code with no
compiler here and no golden outputs); see the header of pci_oracle.c for the
independent checks that stand in.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "pci_oracle.c")


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc (OpenMP, no FP contraction)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC):
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-fno-fast-math", "-o", LIB_PATH, SRC, "-lm"]
        subprocess.check_call(cmd)
    return LIB_PATH


class OrcSys(C.Structure):
    _fields_ = [
        ("ne", C.c_int), ("nst", C.c_int), ("ns", C.c_int), ("nso", C.c_int),
        ("nx", C.c_int), ("mj", C.c_int), ("nlx", C.c_int), ("kbrt", C.c_int),
        ("nd", C.c_int64), ("nc", C.c_int),
        ("iarr", C.c_void_p), ("nh", C.c_void_p), ("jz", C.c_void_p),
        ("nn", C.c_void_p), ("kk", C.c_void_p), ("ll", C.c_void_p), ("jj", C.c_void_p),
        ("ndc", C.c_void_p), ("hint_lut", C.c_void_p), ("gaunt_lut", C.c_void_p),
        ("n_gaunt_lut", C.c_int64), ("ngint", C.c_int64), ("r2_is_f64", C.c_int),
        ("rint2", C.c_void_p), ("iint2", C.c_void_p), ("iint3", C.c_void_p),
        ("gj", C.c_double),
        ("cap", C.c_int64), ("hiac", C.c_void_p), ("hibd", C.c_void_p), ("hpos", C.c_void_p),
        ("err", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_build_hash.argtypes = [C.POINTER(OrcSys)]
        L.orc_free_hash.argtypes = [C.POINTER(OrcSys)]
        L.orc_form_h.argtypes = [C.POINTER(OrcSys), C.c_int64, C.c_int64, P, P, P, P, P, P, P, C.c_int]
        L.orc_form_h.restype = C.c_int64
        L.orc_form_j.argtypes = [C.POINTER(OrcSys), P, P, P, P]
        L.orc_form_j.restype = C.c_int64
        L.orc_mxmpy.argtypes = [C.c_int64, P, P, P, C.c_double, P, P, P]
        L.orc_mxmpy_block.argtypes = [C.c_int64, P, P, P, C.c_double, C.c_int, P, P, C.c_int]
        L.orc_j_av.argtypes = [C.c_int64, P, P, P, P, C.c_int64]
        L.orc_j_av.restype = C.c_double
        L.orc_h_element.argtypes = [C.POINTER(OrcSys), C.c_int64, C.c_int64, C.POINTER(C.c_int)]
        L.orc_h_element.restype = C.c_double
        L.orc_rspq.argtypes = [P, P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), P, P]
        L.orc_bit_compare.argtypes = [P, P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), P, P]
        L.orc_gaunt.argtypes = [C.POINTER(OrcSys), C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_gaunt.restype = C.c_double
        L.orc_gint.argtypes = [C.POINTER(OrcSys), C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_gint.restype = C.c_double
        L.orc_hint.argtypes = [C.POINTER(OrcSys), C.c_int, C.c_int]
        L.orc_hint.restype = C.c_double
        L.orc_lsj.argtypes = [C.POINTER(OrcSys), P, C.c_int, C.c_int, C.c_int, P]
        L.orc_density.argtypes = [C.POINTER(OrcSys), P, C.c_double, P]
        L.orc_transition_density.argtypes = [C.POINTER(OrcSys), C.POINTER(OrcSys), P, P, C.c_double, P]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Oracle:
    """Holds one system's arrays in the layout the C restatement expects."""

    def __init__(self, sysm):
        self.sys = sysm
        L = lib()
        b = sysm.basis
        self._keep = dict(
            iarr=np.ascontiguousarray(sysm.iarr, np.int32),
            nh=np.ascontiguousarray(sysm.nh, np.int32), jz=np.ascontiguousarray(sysm.jz, np.int32),
            nn=np.ascontiguousarray(b.nn, np.int32), kk=np.ascontiguousarray(b.kk, np.int32),
            ll=np.ascontiguousarray(b.ll, np.int32), jj=np.ascontiguousarray(b.jj, np.int32),
            ndc=np.ascontiguousarray(sysm.ndc, np.int32),
            hint=np.ascontiguousarray(sysm.hint_lut, np.float64),
            glut=np.ascontiguousarray(sysm.gaunt_lut, np.float64),
            rint2=np.ascontiguousarray(sysm.rint2),
            iint2=np.ascontiguousarray(sysm.iint2, np.int32),
            iint3=np.ascontiguousarray(sysm.iint3, np.int32),
        )
        k = self._keep
        s = OrcSys()
        s.ne, s.nst, s.ns, s.nso = sysm.ne, sysm.nst, b.ns, b.nso
        s.nx, s.mj, s.nlx, s.kbrt = sysm.nx, sysm.mj, sysm.nlx, sysm.kbrt
        s.nd, s.nc = sysm.nd, sysm.nc
        for name in ("iarr", "nh", "jz", "nn", "kk", "ll", "jj", "ndc"):
            setattr(s, name, _ptr(k[name]))
        s.hint_lut = _ptr(k["hint"])
        s.gaunt_lut = _ptr(k["glut"])
        s.n_gaunt_lut = k["glut"].size
        s.ngint = sysm.ngint
        s.r2_is_f64 = 1 if k["rint2"].dtype == np.float64 else 0
        s.rint2 = _ptr(k["rint2"])
        s.iint2 = _ptr(k["iint2"])
        s.iint3 = _ptr(k["iint3"])
        s.gj = sysm.gj
        self.s = s
        if L.orc_build_hash(C.byref(s)) != 0:
            raise MemoryError("oracle hash allocation failed")

    def __del__(self):
        try:
            lib().orc_free_hash(C.byref(self.s))
        except Exception:
            pass

    # -- single elements ------------------------------------------------
    def h_element(self, n, k):
        nf = C.c_int()
        v = lib().orc_h_element(C.byref(self.s), n, k, C.byref(nf))
        return v, nf.value

    def gaunt(self, k, j1, m1, j2, m2):
        return lib().orc_gaunt(C.byref(self.s), k, j1, m1, j2, m2)

    def gint(self, i1, i2, i3, i4):
        return lib().orc_gint(C.byref(self.s), i1, i2, i3, i4)

    def hint(self, ia, ib):
        return lib().orc_hint(C.byref(self.s), ia, ib)

    # -- FormH / FormJ ----------------------------------------------------
    def form_h(self, row_lo=1, row_hi=None, threads=0):
        """CSR of rows [row_lo, row_hi] (1-based): (rowptr int64, col int32 1-based, val f64,
        numzero, hmin, pairs).  Two passes (count, fill), as the reference's
        comparison/calculation stages."""
        L = lib()
        if row_hi is None:
            row_hi = self.sys.nd
        nrows = row_hi - row_lo + 1
        cnt = np.zeros(nrows, np.int64)
        nz = C.c_int64(0)
        hmin = C.c_double(np.inf)
        pairs = C.c_int64(0)
        L.orc_form_h(C.byref(self.s), row_lo, row_hi, _ptr(cnt), None, None, None,
                     C.byref(nz), C.byref(hmin), C.byref(pairs), threads)
        self._check()
        rowptr = np.zeros(nrows + 1, np.int64)
        np.cumsum(cnt, out=rowptr[1:])
        col = np.zeros(int(rowptr[-1]), np.int32)
        val = np.zeros(int(rowptr[-1]), np.float64)
        nz2 = C.c_int64(0)
        hmin2 = C.c_double(np.inf)
        L.orc_form_h(C.byref(self.s), row_lo, row_hi, None, _ptr(rowptr), _ptr(col), _ptr(val),
                     C.byref(nz2), C.byref(hmin2), None, threads)
        self._check()
        return rowptr, col, val, nz.value, hmin.value, pairs.value

    def form_h_timed_sample(self, rows, threads=0):
        """Count-pass work of FormH (values evaluated, zeros dropped) over the given
        1-based rows; returns (seconds, nnz, pairs).  Used by the CPU baseline."""
        L = lib()
        t0 = time.perf_counter()
        nnz = 0
        pairs = C.c_int64(0)
        nz = C.c_int64(0)
        hmin = C.c_double(np.inf)
        for lo, hi in rows:
            cnt = np.zeros(hi - lo + 1, np.int64)
            nnz += L.orc_form_h(C.byref(self.s), lo, hi, _ptr(cnt), None, None, None,
                                C.byref(nz), C.byref(hmin), C.byref(pairs), threads)
        return time.perf_counter() - t0, nnz, pairs.value

    def lsj_sums(self, X, ic_lo=1, ic_hi=None):
        """calcLSJ (src/pconf.F90:2805-2863) over configurations ic_lo..ic_hi
        (1-based): the sums of c_n c_k t for J, L, S, shape [3, nv]."""
        X = np.asarray(X, np.float64)
        if X.ndim == 1:
            X = X[:, None]
        nv = X.shape[1]
        xc = np.ascontiguousarray(X.T)
        out = np.zeros(3 * nv)
        lib().orc_lsj(C.byref(self.s), _ptr(xc), nv, ic_lo, self.sys.nc if ic_hi is None else ic_hi, _ptr(out))
        return out.reshape(3, nv)

    def lsj(self, X):
        """(J, L, S) of each column of X, lsj's final step
        (src/pconf.F90:2798-2800): x = (sqrt(<X^2> + 1) - 1) / 2."""
        t = self.lsj_sums(X)
        x = 0.5 * (np.sqrt(t + 1) - 1)
        return x[0], x[1], x[2]

    def density(self, b, trd=1e-10):
        """FormDM's density matrix (src/pdtm.f90:1254-1310) of vector b:
        [Nst, Nst] with entry [i, j] = Ro(i+1, j+1)."""
        b = np.ascontiguousarray(b, np.float64)
        nst = self.sys.nst
        ro = np.zeros(nst * nst)
        lib().orc_density(C.byref(self.s), _ptr(b), float(trd), _ptr(ro))
        return ro.reshape(nst, nst).T

    def transition_density(self, initial, b_initial, b_final, trd=1e-10):
        """FormTM's transition density (src/pdtm.f90:1538-1605) from a level of
        `initial` (another Oracle) to a level of this system: [Nst, Nst] with
        entry [i, j] = Ro(i+1, j+1), i the initial m-state."""
        bi = np.ascontiguousarray(b_initial, np.float64)
        bf = np.ascontiguousarray(b_final, np.float64)
        nst = self.sys.nst
        ro = np.zeros(nst * nst)
        lib().orc_transition_density(C.byref(initial.s), C.byref(self.s), _ptr(bi), _ptr(bf), float(trd), _ptr(ro))
        return ro.reshape(nst, nst).T

    def form_j(self):
        L = lib()
        nd = self.sys.nd
        cnt = np.zeros(nd, np.int64)
        L.orc_form_j(C.byref(self.s), _ptr(cnt), None, None, None)
        rowptr = np.zeros(nd + 1, np.int64)
        np.cumsum(cnt, out=rowptr[1:])
        col = np.zeros(int(rowptr[-1]), np.int32)
        val = np.zeros(int(rowptr[-1]), np.float64)
        L.orc_form_j(C.byref(self.s), None, _ptr(rowptr), _ptr(col), _ptr(val))
        return rowptr, col, val

    def _check(self):
        if self.s.err == 1:
            raise KeyError("Gint: integral is absent")
        if self.s.err == 2:
            raise ValueError("Gint error: ma+mb /= mc+md")


def csr_to_dense(nd, rowptr, col, val):
    """Symmetric dense matrix from a lower-triangle CSR with 1-based columns."""
    a = np.zeros((nd, nd))
    rows = np.repeat(np.arange(nd), np.diff(rowptr))
    a[rows, col - 1] = val
    a[col - 1, rows] = val
    return a


def j_av(rowptr, col, val, x, nx):
    x = np.ascontiguousarray(x, np.float64)
    return lib().orc_j_av(rowptr.size - 1, _ptr(rowptr), _ptr(col), _ptr(val), _ptr(x), nx)


def j_terms(basis, configs, mj):
    """Jt(1:Njd), the sorted 2J values of the terms present, as Dinit finds
    them (src/determinants.f90:227-325): for every configuration that has
    determinants with 2M = mj, count its determinants nmj(im) with
    2M = mj + 2(im-1) >= mj, peel terms off from the largest im down, and keep
    each new 2J = mj + 2(im-1) once.  ``configs`` as in
    pci_b200.system.enumerate_determinants; determinants are enumerated
    explicitly (small systems only)."""
    import itertools
    jt = []
    for conf in configs:
        shells = [(ni, nq) for ni, nq in conf if nq > 0]
        per_shell = []
        for ni, nq in shells:
            j2 = int(basis.jj[ni - 1])
            ms = list(range(-j2, j2 + 1, 2))
            per_shell.append([sum(c) for c in itertools.combinations(ms, nq)])
        nmj = {}
        ndi = 0
        for combo in itertools.product(*per_shell):
            m = sum(combo)
            if m == mj:
                ndi += 1
            if m >= mj:
                im = (m - mj) // 2 + 1
                nmj[im] = nmj.get(im, 0) + 1
        if ndi == 0:
            continue
        imax = max(nmj)
        cnt = [0] * (imax + 1)
        for im, c in nmj.items():
            cnt[im] = c
        for im in range(imax, 0, -1):
            n = cnt[im]
            if n != 0:
                mt = (im - 1) * 2 + mj
                for j in range(1, im + 1):
                    cnt[j] -= n
                if mt not in jt:
                    jt.append(mt)
    return sorted(jt)


def calc_nd0(ndc, nc4, max_nd0):
    """calcNd0, src/determinants.f90:22-45 (kCSF = 0)."""
    ic1, n2, n1, n0 = 0, 0, 0, max_nd0 + 1
    for ic in range(1, nc4 + 1):
        if ic > ndc.size:
            break
        n1 += int(ndc[ic - 1])
        if n1 < n0:
            n2 = n1
            ic1 = ic
    return ic1, n2


class DavidsonResult(dict):
    pass


def diag4(nd, H, hmin, J, params, ndc, mxmpy_threads=1, log=None, timing=None, jt=None):
    """Restatement of Diag4 (src/pconf.F90:1993-2264) with Init4, DiagInitApprox,
    FormB0, Ortn, Mxmpy, FormP, Dvdsn, FormB/FormBskip and WriteFinalXIJ from
    src/davidson.f90 (npes = 1).  Kv = 3 (K_prj = 1) adds the J selection of
    FormB0, AvgDiag in the first iteration and Prj_J on the new vectors, which
    needs the term list ``jt`` (j_terms).  H and J are (rowptr, col, val) lower-triangle CSR with 1-based
    columns.  Returns energies Tk (binding-energy convention, -(E+Hmin)),
    Tj, eigenvectors X[nd, Nlv], iterations and the residual norms."""
    rowptr, col, val = H
    jrow, jcol, jval = J
    Nlv = int(params["Nlv"])
    N_it = int(params.get("N_it", 200))
    Crt4 = float(params.get("Crt4", 1e-8))
    Kl4 = int(params.get("Kl4", 1))
    Kv = int(params.get("Kv", 4))
    K_prj = 1 if Kv == 3 else 0
    XJ_av = float(params.get("XJ_av", 0.0))
    admix_crit = float(params.get("admix_crit", 1e-6))
    nc4 = int(params.get("Nc4", ndc.size))
    _, Nd0 = calc_nd0(ndc, nc4, int(params.get("MaxNd0", 3000)))
    L = lib()
    t_start = time.perf_counter()

    # Init4 (src/davidson.f90:20-73)
    Z1 = np.zeros((Nd0, Nd0))
    for n in range(1, Nd0 + 1):
        for l in range(rowptr[n - 1], rowptr[n]):
            k = int(col[l])
            t = val[l]
            if n == k:
                t = t - hmin
            if k <= Nd0:
                Z1[n - 1, k - 1] = t
                Z1[k - 1, n - 1] = t
    # DiagInitApprox: DSYEVD
    E1, Z1 = np.linalg.eigh(Z1)
    # FormB0 (src/davidson.f90:75-193), Kl4 /= 2
    ArrB = np.zeros((nd, 3 * Nlv), order="F")
    E = np.zeros(2 * Nlv)
    Tj = np.zeros(Nlv)
    num = 0
    for j in range(Nd0):
        b1 = Z1[:, j]
        xj = j_av(jrow, jcol, jval, b1, Nd0)
        ierr = 1 if (K_prj == 1 and abs(xj - XJ_av) > 0.1) else 0
        if ierr == 0:
            E[num] = -(E1[j] + hmin)
            Tj[num] = xj
            ArrB[:Nd0, num] = b1
            num += 1
            if num >= Nlv:
                break
    Nlv = num
    ArrB = ArrB[:, :3 * Nlv].copy(order="F") if ArrB.shape[1] != 3 * Nlv else ArrB
    P = np.zeros((2 * Nlv, 2 * Nlv))
    Tk = np.zeros(Nlv)
    Iconverge = np.zeros(Nlv, np.int32)
    diag = np.zeros(nd)
    diag_init = [False]
    crit, ax, cnx, vmax = 1e-6 if admix_crit is None else admix_crit, 1.0, 1.0, 0.0
    n01 = 1 if abs(Kl4) == 2 else Nlv + 1
    Z1s = Z1[:, n01 - 1:]
    E1s = E1[n01 - 1:]
    cnorms = np.zeros(Nlv)
    it_done = 0
    x_tmp = np.zeros(nd)
    y_tmp = np.zeros(nd)

    def ortn(j):  # src/davidson.f90:649-741, j 1-based
        jm = j - 1
        smax2 = 1e10
        it = 0
        while True:
            it += 1
            smax1 = 0.0
            if jm > 0:
                s_arr = ArrB[:, :jm].T @ ArrB[:, j - 1]
                for l in range(1, jm + 1):
                    if l > Nlv and Iconverge[l - Nlv - 1] == 1:
                        s_arr[l - 1] = 0.0
                    elif abs(s_arr[l - 1]) > smax1:
                        smax1 = abs(s_arr[l - 1])
                ArrB[:, j - 1] -= ArrB[:, :jm] @ s_arr
            if smax1 < 1e-6:
                break
            if smax1 > smax2 or it > 3:
                raise RuntimeError(f"Fail of orthogonalization of vector {j}")
            smax2 = smax1
        s = float(ArrB[:, j - 1] @ ArrB[:, j - 1])
        if s < 1e-9:
            raise RuntimeError(f"Fail of normalization of vector {j}")
        ArrB[:, j - 1] *= 1.0 / np.sqrt(s)

    def mxmpy(ip):  # src/davidson.f90:572-647
        i2min = 1 + ip * Nlv
        i1min = i2min - Nlv
        kd = not diag_init[0]
        for iv in range(Nlv):
            x_tmp[:] = ArrB[:, i1min - 1 + iv]
            d = diag if (kd and iv == 0) else None
            L.orc_mxmpy(nd, _ptr(rowptr), _ptr(col), _ptr(val), hmin, _ptr(x_tmp), _ptr(y_tmp),
                        _ptr(d) if d is not None else None)
            ArrB[:, i2min - 1 + iv] = y_tmp
        diag_init[0] = True

    def formp(kp):  # src/davidson.f90:300-369
        if kp == 1:
            Pt = ArrB[:, :Nlv].T @ ArrB[:, Nlv:2 * Nlv]
            for i in range(Nlv):
                for k in range(i + 1):
                    P[i, k] = Pt[i, k]
                    P[k, i] = Pt[i, k]
        else:
            Pt = ArrB[:, :2 * Nlv].T @ ArrB[:, 2 * Nlv:3 * Nlv]
            for i in range(Nlv):
                for k in range(Nlv, 2 * Nlv):
                    P[i, k] = Pt[i, k - Nlv]
                    P[k, i] = Pt[i, k - Nlv]
            for i in range(Nlv, 2 * Nlv):
                for k in range(Nlv, i + 1):
                    P[i, k] = Pt[i, k - Nlv]
                    P[k, i] = Pt[i, k - Nlv]
            for i in range(Nlv):
                if Iconverge[i] == 1:
                    i1 = i + Nlv
                    P[i1, :] = 0.0
                    P[:, i1] = 0.0
                    P[i1, i1] = 2 * vmax - P[i, i] + 1.0

    def dvdsn(j):  # src/davidson.f90:436-570, j 1-based
        nonlocal cnx
        j1 = j + Nlv
        v = P[j - 1, j - 1]
        t = ArrB[:, j1 - 1] - v * ArrB[:, j - 1]
        cn = np.sqrt(abs(float(t @ t)))
        cnorms[j - 1] = cn
        Iconverge[j - 1] = 1 if cn < Crt4 else 0
        if cn > cnx:
            cnx = cn
        if Iconverge[j - 1] == 1:
            ArrB[:, j1 - 1] = 0.0
            return
        b1 = np.zeros(Nd0)
        if Z1s.shape[1] > 0:
            s_vec = Z1s.T @ t[:Nd0]
            den = v - E1s
            small = np.abs(den) < 1e-6
            s_vec = np.where(small, 0.0, s_vec / np.where(small, 1.0, den))
            b1 = Z1s @ s_vec
        b_loc = t[Nd0:] / (v - diag[Nd0:])
        s = 1.0 / np.sqrt(float(b1 @ b1) + float(b_loc @ b_loc))
        ArrB[:Nd0, j1 - 1] = b1 * s
        ArrB[Nd0:, j1 - 1] = b_loc * s

    def avg_diag():  # src/davidson.f90:371-434
        id0 = 0
        for c in ndc:
            c = int(c)
            if c > 0:
                s = 0.0
                for i in range(id0, id0 + c):
                    s += diag[i]
                diag[id0:id0 + c] = s / c
                id0 += c

    if K_prj == 1:
        if jt is None:
            raise ValueError("Kv = 3 needs the term list jt")
        if 0 in jt and int(2 * XJ_av + 0.1) != 0:
            # the filter factor 1/(jx(jx+2)) of src/davidson.f90:808 is 1/0 for
            # a J = 0 term, which the reference applies when XJ_av /= 0
            raise ValueError("Prj_J: a J = 0 term with XJ_av /= 0 divides by zero")

    def prj_j(lin, num, lout, trsd):  # src/davidson.f90:743-884, lin/lout 1-based
        jav = int(2 * XJ_av + 0.1)
        col_in = np.array(ArrB[:, lin - 1:lin - 1 + num])
        col_out = np.zeros_like(col_in)
        go = [Iconverge[i] == 0 for i in range(num)]
        njd = len(jt)
        jx, f = 0, 0.0
        for itr in range(1, njd + 2):
            itj = njd + 1 - itr
            if itj != 0:
                jx = int(jt[itj - 1])
                f = 1.0 / (jx * (jx + 2)) if jx != 0 else float("inf")   # IEEE 1/0 of the reference
            if jx != jav or itj == 0:
                col_out[:] = 0.0
                for i in range(num):
                    if go[i]:
                        x = np.ascontiguousarray(col_in[:, i])
                        L.orc_mxmpy(nd, _ptr(jrow), _ptr(jcol), _ptr(jval), 0.0, _ptr(x), _ptr(y_tmp), None)
                        col_out[:, i] = y_tmp
                ArrB[:, lout - 1:lout - 1 + num] = col_out
                err1 = 0.0
                for i in range(num):
                    if go[i]:
                        sj = float(col_in[:, i] @ col_out[:, i])
                        err1 = max(err1, abs(np.sqrt(1 + sj) - 1 - jav))
                if err1 < trsd:
                    return
                if itj != 0:
                    for i in range(num):
                        if go[i]:
                            a = col_in[:, i] - f * col_out[:, i]
                            col_in[:, i] = a / np.sqrt(float(a @ a))
                            ArrB[:, lin - 1 + i] = col_in[:, i]

    hist = []
    for it in range(1, N_it + 1):
        if not (ax > crit):
            continue
        it_done = it
        for i in range(1, Nlv + 1):
            ortn(i)
        mxmpy(1)
        formp(1)
        if it == 1 and K_prj == 1:
            avg_diag()
        cnx = 0.0
        for i in range(1, Nlv + 1):
            dvdsn(i)
            if Iconverge[i - 1] == 0:
                ortn(i + Nlv)
        if K_prj == 1:
            prj_j(Nlv + 1, Nlv, 2 * Nlv + 1, 1e-5)
            for i in range(Nlv + 1, 2 * Nlv + 1):
                if Iconverge[i - Nlv - 1] == 0:
                    ortn(i)
        hist.append(cnorms.copy())
        if cnx > Crt4:
            mxmpy(2)
            pmax = max(P[i, i] for i in range(Nlv))
            if pmax > vmax:
                vmax = pmax
            formp(2)
            Evals, Pv = np.linalg.eigh(P)
            P[:, :] = Pv
            E[:] = Evals
            ax = 0.0
            vmax = -1e10
            for i in range(Nlv):
                xx = np.max(np.abs(P[Nlv:2 * Nlv, i]))
                ax = max(ax, xx)
                vmax = max(vmax, E[i])
            ArrB[:, 2 * Nlv:3 * Nlv] = ArrB[:, :2 * Nlv] @ P[:, :Nlv]
            Tk[:] = -(E[:Nlv] + hmin)
            ArrB[:, :Nlv] = ArrB[:, 2 * Nlv:3 * Nlv]
            if log:
                log(it, Tk.copy(), cnorms.copy())
        else:
            if it == 1:
                Tk[:] = E[:Nlv]
            break
    X = np.array(ArrB[:, :Nlv])
    for n in range(Nlv):
        Tj[n] = j_av(jrow, jcol, jval, X[:, n], nd)
    res = DavidsonResult(Tk=Tk.copy(), Tj=Tj.copy(), X=X, iterations=it_done,
                         cnorm=cnorms.copy(), converged=bool(np.all(Iconverge == 1)),
                         Nd0=Nd0, seconds=time.perf_counter() - t_start, history=hist)
    return res


def csf_basis(sysm, J):
    """jbasis (src/csf.f90:17-407) for every configuration, densely: the J^2
    block of the configuration's determinants (build_j2, 409-452, from the
    FormJ CSR J = (rowptr, col 1-based, val) lower triangle), its
    eigenvectors (DSYEVD), and the ones with 2J = Mj kept, J from
    (sqrt(1 + eigenvalue) - 1) / 2.  Returns (per-configuration CSF counts,
    the block-diagonal Nd x Ncsf coefficient matrix C)."""
    jr, jc, jv = J
    nd = sysm.nd
    starts = np.concatenate([[0], np.cumsum(sysm.ndc)])
    counts, cols = [], []
    for c in range(len(sysm.ndc)):
        a, b = int(starts[c]), int(starts[c + 1])
        m = b - a
        Z = np.zeros((m, m))
        for n in range(a, b):
            for l in range(jr[n], jr[n + 1]):
                k = jc[l] - 1
                if a <= k <= n:
                    Z[n - a, k - a] = Z[k - a, n - a] = jv[l]
        de, zz = np.linalg.eigh(Z)
        tj = 0.5 * (np.sqrt(1.0 + de) - 1.0)
        jtt = np.floor(2 * tj + 0.0001).astype(int)
        if np.any(np.abs(2 * tj - jtt) > 1e-7):
            raise ValueError(f"jbasis: J not integer or half-integer in configuration {c + 1}")
        sel = np.flatnonzero(jtt == sysm.mj)
        counts.append(sel.size)
        for s in sel:
            v = np.zeros(nd)
            v[a:b] = zz[:, s]
            cols.append(v)
    C = np.stack(cols, axis=1) if cols else np.zeros((nd, 0))
    return np.asarray(counts), C


def csf_hamiltonian(H_dense, C):
    """formh_sym (src/csf.f90:538-964): the CSF-basis H = C^T H C."""
    return C.T @ H_dense @ C


def pt2_groups(H_dense, nd1, nd0, X0, E, groups, conf_sizes=None, avg_diag=False):
    """PTE's contributions per group of PT rows (src/conf_pt.f90:825-875,
    dE(n,ic) and dV(n,ic) over the determinants of NR configuration ic), in
    the engine's convention: rows groups[g]..groups[g+1]-1."""
    nd = H_dense.shape[0]
    X0 = np.asarray(X0, np.float64).reshape(nd0, -1)
    E = np.asarray(E, np.float64)
    diag = np.diag(H_dense).copy()
    if avg_diag:
        starts = np.concatenate([[0], np.cumsum(conf_sizes)])
        for a, b in zip(starts[:-1], starts[1:]):
            if a >= nd1 and b > a:
                diag[b - 1] = diag[a:b].mean()
    ng = len(groups) - 1
    dEg = np.zeros((ng, len(E)))
    dVg = np.zeros((ng, len(E)))
    for g in range(ng):
        for i in range(int(groups[g]), int(groups[g + 1])):
            x = H_dense[i, :nd0] @ X0
            dl = E - diag[i]
            dEg[g] += x * x / dl
            dVg[g] += (x / dl) ** 2
    return dEg, dVg


def pt2(H_dense, nd1, nd0, X0, E, conf_sizes=None, avg_diag=False):
    """PTE (src/conf_pt.f90:751-952) densely, in the engine's convention: for
    every determinant i beyond nd1, x = sum_(k < nd0) H_ik X0_kn, dE_n +=
    x^2 / (E_n - e_i) and c_in = x / (E_n - e_i), e_i = H_ii; average_diag
    (conf_pt.f90:710-724) puts each PT configuration's mean on its last
    determinant (the position the reference writes).  conf_sizes: the
    determinants of each configuration (needed for avg_diag)."""
    nd = H_dense.shape[0]
    X0 = np.asarray(X0, np.float64).reshape(nd0, -1)
    E = np.asarray(E, np.float64)
    diag = np.diag(H_dense).copy()
    if avg_diag:
        starts = np.concatenate([[0], np.cumsum(conf_sizes)])
        for a, b in zip(starts[:-1], starts[1:]):
            if a >= nd1 and b > a:
                diag[b - 1] = diag[a:b].mean()
    dE = np.zeros(len(E))
    C = np.zeros((nd, len(E)))
    for i in range(nd1, nd):
        x = H_dense[i, :nd0] @ X0
        dl = E - diag[i]
        dE += x * x / dl
        C[i] = x / dl
    return dE, C
