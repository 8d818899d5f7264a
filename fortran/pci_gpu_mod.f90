! ISO_C_BINDING interface to libpci_gpu.so (include/pci_gpu.h) for pconf.
! Use it under #ifdef PCI_GPU in place of the FormH / FormJ / Diag4 calls at
! pconf.F90:217-238 (FormH + RedistributeHamCSR, FormJ, Diag4).  Indices and
! arrays are passed exactly as pconf holds them (1-based, column-major).
module pci_gpu_mod
  use, intrinsic :: iso_c_binding
  implicit none
  type, bind(C) :: pci_dvd_params
     integer(c_int32_t) :: Nlv, N_it, Kl4, Kv, Nc4, MaxNd0, mode, KXIJ
     real(c_double)     :: Crt4, XJ_av, admix_crit
  end type
  interface
     integer(c_int) function pci_gpu_create(device, h) bind(C)
       import; integer(c_int32_t), value :: device; type(c_ptr) :: h
     end function
     integer(c_int) function pci_gpu_set_basis(h, Ne, Nd, Nst, Nsu, Nso, Nx, Mj, Iarr, Nh, Jz, &
                                               Nn, Kk, Ll, Jj, Nc, Ndc, Gj) bind(C)
       import; type(c_ptr), value :: h
       integer(c_int32_t), value :: Ne, Nst, Nsu, Nso, Nx, Mj, Nc
       integer(c_int64_t), value :: Nd
       integer(c_int32_t) :: Iarr(*), Nh(*), Jz(*), Nn(*), Kk(*), Ll(*), Jj(*), Ndc(*)
       real(c_double), value :: Gj
     end function
     integer(c_int) function pci_gpu_set_integrals(h, HintLUT, Nlx, nGauntLUT, GauntLUT, Ngint, kbrt, &
                                                   r2_is_f64, Rint2, Iint2, Iint3) bind(C)
       import; type(c_ptr), value :: h
       real(c_double) :: HintLUT(*), GauntLUT(*)
       integer(c_int32_t), value :: Nlx, kbrt, r2_is_f64
       integer(c_int64_t), value :: nGauntLUT, Ngint
       type(c_ptr), value :: Rint2
       integer(c_int32_t) :: Iint2(*), Iint3(*)
     end function
     integer(c_int) function pci_gpu_form_h(h, value_prec, NumH, numzero, Hmin) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t), value :: value_prec
       integer(c_int64_t) :: NumH, numzero; real(c_double) :: Hmin
     end function
     integer(c_int) function pci_gpu_form_j(h, NumJ) bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t) :: NumJ
     end function
     integer(c_int) function pci_gpu_davidson(h, p, X0, Tk, Tj, Iconverge, X, iters, resid) bind(C)
       import; type(c_ptr), value :: h; type(pci_dvd_params) :: p
       type(c_ptr), value :: X0
       real(c_double) :: Tk(*), Tj(*), X(*), resid(*)
       integer(c_int32_t) :: Iconverge(*), iters
     end function
     integer(c_int) function pci_gpu_j_av(h, X, nv, nlim, Tj) bind(C)
       import; type(c_ptr), value :: h; real(c_double) :: X(*), Tj(*)
       integer(c_int32_t), value :: nv; integer(c_int64_t), value :: nlim
     end function
     integer(c_int) function pci_gpu_csr_info(h, which, nrows, nnz) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t), value :: which
       integer(c_int64_t) :: nrows, nnz
     end function
     ! WriteMatrixCSR's arrays (matrix_io.f90:689-799): the whole resident CSR of H or J^2
     integer(c_int) function pci_gpu_get_csr(h, which, rowptr, col, val) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t), value :: which
       integer(c_int64_t) :: rowptr(*); integer(c_int32_t) :: col(*); real(c_double) :: val(*)
     end function
     ! ReadMatrixCSR (matrix_io.f90:801-939), Kl = 1: a stored CSR and its Hmin made resident
     integer(c_int) function pci_gpu_set_csr(h, which, Nd, nnz, rowptr, col, val, Hmin) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t), value :: which
       integer(c_int64_t), value :: Nd, nnz
       integer(c_int64_t) :: rowptr(*); integer(c_int32_t) :: col(*); real(c_double) :: val(*)
       real(c_double), value :: Hmin
     end function
     ! one rank's row range of H (which 0) or J^2 (which 1), as RedistributeHamCSR leaves it
     integer(c_int) function pci_gpu_get_csr_rows(h, which, row_lo, row_hi, rowptr, col, val) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t), value :: which
       integer(c_int64_t), value :: row_lo, row_hi
       integer(c_int64_t) :: rowptr(*)
       type(c_ptr), value :: col, val
     end function
     ! Jterm's table (determinants.f90:227-325): returns Njd, up to cap 2J values in out
     integer(c_int32_t) function pci_gpu_jterms(h, out, cap) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t) :: out(*); integer(c_int32_t), value :: cap
     end function
     ! timings and counters of the last calls (the list in pci_gpu.h); returns the number written
     integer(c_int32_t) function pci_gpu_stats(h, out, n) bind(C)
       import; type(c_ptr), value :: h; real(c_double) :: out(*); integer(c_int32_t), value :: n
     end function
     ! kLSJ = 1 (lsj, pconf.F90:2672-2962): J, L, S of nv vectors X(Nd, nv)
     integer(c_int) function pci_gpu_lsj(h, X, nv, xj, xl, xs) bind(C)
       import; type(c_ptr), value :: h; real(c_double) :: X(*), xj(*), xl(*), xs(*)
       integer(c_int32_t), value :: nv
     end function
     ! kCSF = 1: jbasis + formh_sym (csf.f90); the CSF H replaces H on the handle
     integer(c_int) function pci_gpu_form_csf(h, ncsf, numh) bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t) :: ncsf, numh
     end function
     ! CSFs of each configuration (jbasis's per-configuration counts): per_conf(Nc)
     integer(c_int) function pci_gpu_csf_counts(h, per_conf) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t) :: per_conf(*)
     end function
     ! unsym (csf.f90:1088-1134): Y(Ncsf, nv) -> X(Nd, nv)
     integer(c_int) function pci_gpu_csf_to_det(h, Y, nv, X) bind(C)
       import; type(c_ptr), value :: h; real(c_double) :: Y(*), X(*)
       integer(c_int32_t), value :: nv
     end function
     ! conf_pt PTE (conf_pt.f90:751-952): second-order energies dE(nv), Xpt(Nd, nv) or c_null_ptr
     integer(c_int) function pci_gpu_pt2(h, nd1, nd0, X0, nv, E, avg_diag, dE, Xpt) bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t), value :: nd1, nd0
       real(c_double) :: X0(*), E(*), dE(*); integer(c_int32_t), value :: nv, avg_diag
       type(c_ptr), value :: Xpt
     end function
     ! PTE with dE(n,ic), dV(n,ic) of row groups (conf_pt.f90:871-872): dEg(nv, ngrp), dVg(nv, ngrp)
     integer(c_int) function pci_gpu_pt2_groups(h, nd1, nd0, X0, nv, E, avg_diag, grp, ngrp, dE, dEg, dVg, Xpt) &
         bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t), value :: nd1, nd0
       real(c_double) :: X0(*), E(*), dE(*), dEg(*), dVg(*); integer(c_int32_t), value :: nv, avg_diag, ngrp
       integer(c_int64_t) :: grp(*); type(c_ptr), value :: Xpt
     end function
     ! conf_pt FormH (conf_pt.f90:1319-1351): the PT block (rows > nd1, columns <= nd0) in place of H
     integer(c_int) function pci_gpu_form_h_pt(h, nd1, nd0, value_prec, NumH) bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t), value :: nd1, nd0
       integer(c_int32_t), value :: value_prec; integer(c_int64_t) :: NumH
     end function
     ! the PT block for the PT rows row_lo+1..row_hi only (one share of the PT space)
     integer(c_int) function pci_gpu_form_h_pt_rows(h, nd1, nd0, row_lo, row_hi, value_prec, NumH) bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t), value :: nd1, nd0, row_lo, row_hi
       integer(c_int32_t), value :: value_prec; integer(c_int64_t) :: NumH
     end function
     ! pdtm FormDM density pass: Ro(Nst, Nst, nv) of X(Nd, nv)
     integer(c_int) function pci_gpu_density(h, X, nv, trd, Ro) bind(C)
       import; type(c_ptr), value :: h; real(c_double) :: X(*), Ro(*)
       integer(c_int32_t), value :: nv; real(c_double), value :: trd
     end function
     ! pdtm FormTM transition density: initial level B1 (handle hi), final level B2 (handle hf)
     integer(c_int) function pci_gpu_transition_density(hi, hf, B1, B2, trd, Ro) bind(C)
       import; type(c_ptr), value :: hi, hf; real(c_double) :: B1(*), B2(*), Ro(*)
       real(c_double), value :: trd
     end function
     ! FormBarr: Barr(nint, Nd) of the basis (barr may be c_null_ptr)
     integer(c_int) function pci_gpu_form_barr(h, nint, barr) bind(C)
       import; type(c_ptr), value :: h; integer(c_int32_t) :: nint
       type(c_ptr), value :: barr
     end function
     ! compare_bit_dets + get_det_indexes for n pairs (pairs(2, n), 1-based)
     integer(c_int) function pci_gpu_bit_compare(h, n, pairs, ndiffs, is, idx1, idx2) bind(C)
       import; type(c_ptr), value :: h; integer(c_int64_t), value :: n
       integer(c_int64_t) :: pairs(*)
       integer(c_int32_t) :: ndiffs(*), is(*), idx1(*), idx2(*)
     end function
     ! CONF.HIJ / CONF.JJJ record stream (sort.f90), written in row ranges
     integer(c_int) function pci_io_append_hij(path, row0, nrows, rowptr, col, val, errbuf, errlen) bind(C)
       import; character(kind=c_char) :: path(*), errbuf(*)
       integer(c_int64_t), value :: row0, nrows
       integer(c_int64_t) :: rowptr(*); integer(c_int32_t) :: col(*); real(c_double) :: val(*)
       integer(c_int32_t), value :: errlen
     end function
     type(c_ptr) function pci_gpu_last_error(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     subroutine pci_gpu_destroy(h) bind(C)
       import; type(c_ptr), value :: h
     end subroutine
  end interface
end module
