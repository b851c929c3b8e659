! cholesky_gammcor_gpu.f90 -- the module Cholesky_Gammcor with the interface of
! src/gammcor-interface/Cholesky_Gammcor.f90 (module name, TCholeskyVecsOTF,
! CHOL_ACCURACY_*, chol_gammcor_Rkpq and chol_gammcor_Rkab unchanged), whose
! decomposition and AO->MO transformation run in libgci.so on the GPU through
! the C ABI of include/gci.h.
!
! Build: compile this file in place of Cholesky_Gammcor.f90 into the
! cholesky.a archive, and link libgci.so (with -lcudart).
! The modules it uses (arithmetic, display, TwoStepCholesky_definitions,
! basis_definitions, Auto2eInterface) are the reference's own.
!
! Differences a caller can observe:
!  * TCholeskyVecsOTF keeps the library handle in a private component; the
!    device memory it owns is released by the type's finalizer or by
!    chol_gammcor_free.
!  * chol_gammcor_Rkpq fills Rkpq(NVecs, MaxSubsetDim, NSubsets) only when
!    chol_gammcor_store_rkpq is .true. (the default, as the reference);
!    with .false. Rkpq is allocated with a zero-size last dimension and
!    chol_gammcor_Rkab builds Rkab directly from the integrals.
module gci_capi
      use iso_c_binding
      implicit none

      integer(c_int), parameter :: GCI_OK = 0
      integer(c_int), parameter :: GCI_FLAG_MATERIALIZE_RKPQ = 1
      integer(c_int), parameter :: GCI_PREC_FP64 = 0

      type, bind(C) :: gci_basis
            integer(c_int64_t) :: natoms, nshells, nshellparams, ldprim, ldnorm
            type(c_ptr) :: atom_coords, shell_centers, shell_params_idx, shell_momentum
            type(c_ptr) :: nprimitives, cntr_coeffs, exponents, norm_factors
            integer(c_int32_t) :: spher_ao
      end type gci_basis

      interface
            integer(c_int) function gci_init() bind(C, name="gci_init")
                  import :: c_int
            end function gci_init

            integer(c_int) function gci_rkpq(basis, accuracy, omega, flags, handle) bind(C, name="gci_rkpq")
                  import :: c_int, c_double, c_ptr, gci_basis
                  type(gci_basis), intent(in) :: basis
                  integer(c_int), value :: accuracy, flags
                  real(c_double), value :: omega
                  type(c_ptr), intent(out) :: handle
            end function gci_rkpq

            integer(c_int) function gci_query(h, nvecs, msd, nsub, npq, nsp, npsp) bind(C, name="gci_query")
                  import :: c_int, c_int64_t, c_ptr
                  type(c_ptr), value :: h
                  integer(c_int64_t), intent(out) :: nvecs, msd, nsub, npq, nsp, npsp
            end function gci_query

            integer(c_int) function gci_copy_rkpq(h, dst) bind(C, name="gci_copy_rkpq")
                  import :: c_int, c_ptr, c_double
                  type(c_ptr), value :: h
                  real(c_double), intent(out) :: dst(*)
            end function gci_copy_rkpq

            integer(c_int) function gci_copy_chol2data(h, sp, spl, spd, sd, sb, piv, psp, pspl, pspd, porb, invl) &
                  bind(C, name="gci_copy_chol2data")
                  import :: c_int, c_ptr, c_int64_t, c_double
                  type(c_ptr), value :: h
                  integer(c_int64_t), intent(out) :: sp(*), spl(*), spd(*), sd(*), sb(*), piv(*)
                  integer(c_int64_t), intent(out) :: psp(*), pspl(*), pspd(*), porb(*)
                  real(c_double), intent(out) :: invl(*)
            end function gci_copy_chol2data

            integer(c_int) function gci_rkab(h, ca, ldca, a0, a1, cb, ldcb, b0, b1, mb, prec, rkab) &
                  bind(C, name="gci_rkab")
                  import :: c_int, c_ptr, c_int64_t, c_double
                  type(c_ptr), value :: h
                  real(c_double), intent(in) :: ca(*), cb(*)
                  integer(c_int64_t), value :: ldca, a0, a1, ldcb, b0, b1, mb
                  integer(c_int), value :: prec
                  real(c_double), intent(out) :: rkab(*)
            end function gci_rkab

            subroutine gci_free(h) bind(C, name="gci_free")
                  import :: c_ptr
                  type(c_ptr), value :: h
            end subroutine gci_free

            type(c_ptr) function gci_last_error() bind(C, name="gci_last_error")
                  import :: c_ptr
            end function gci_last_error

            integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
                  import :: c_size_t, c_ptr
                  type(c_ptr), value :: s
            end function c_strlen
      end interface

contains

      function gci_error_text() result(text)
            ! gci_last_error() of the calling thread as a Fortran string
            character(:), allocatable :: text
            type(c_ptr) :: p
            character(kind=c_char), dimension(:), pointer :: chars
            integer :: n, i
            p = gci_last_error()
            n = int(c_strlen(p))
            call c_f_pointer(p, chars, [n])
            allocate(character(n) :: text)
            do i = 1, n
                  text(i:i) = chars(i)
            end do
      end function gci_error_text
end module gci_capi


module Cholesky_Gammcor
      use iso_c_binding
      use arithmetic
      use display
      use TwoStepCholesky_definitions
      use basis_definitions
      use Auto2eInterface
      use gci_capi

      implicit none

      integer, parameter :: CHOL_ACCURACY_DEFAULT = 1
      integer, parameter :: CHOL_ACCURACY_TIGHT = 2
      integer, parameter :: CHOL_ACCURACY_LUDICROUS = 3
      integer, parameter :: CHOL_ACCURACY_DEBUG = 4
      !
      ! .false.: keep Rkpq on the device only (zero-size host Rkpq); chol_gammcor_Rkab
      ! then forms Rkab directly from the integrals
      !
      logical :: chol_gammcor_store_rkpq = .true.

      type TCholeskyVecsOTF
            real(F64), dimension(:, :, :), allocatable :: Rkpq
            type(TChol2Vecs) :: Chol2Data
            type(c_ptr), private :: Handle = c_null_ptr
      contains
            final :: chol_gammcor_finalize
      end type TCholeskyVecsOTF

contains

      subroutine gci_check(status)
            ! The reference reports errors with msg + error stop; so does the shim.
            integer(c_int), intent(in) :: status
            if (status /= GCI_OK) then
                  call msg(gci_error_text())
                  error stop
            end if
      end subroutine gci_check


      subroutine chol_gammcor_finalize(this)
            type(TCholeskyVecsOTF), intent(inout) :: this
            if (c_associated(this%Handle)) call gci_free(this%Handle)
            this%Handle = c_null_ptr
      end subroutine chol_gammcor_finalize


      subroutine chol_gammcor_free(CholeskyVecsOTF)
            ! Release the device memory of a decomposition before the variable goes
            ! out of scope.
            type(TCholeskyVecsOTF), intent(inout) :: CholeskyVecsOTF
            call chol_gammcor_finalize(CholeskyVecsOTF)
      end subroutine chol_gammcor_free


      subroutine chol_gammcor_Rkpq(CholeskyVecsOTF, AOBasis, Accuracy, Omega)
            !
            ! Cholesky vectors in AO basis (two-step decomposition on the GPU).
            !
            type(TCholeskyVecsOTF), intent(out)                     :: CholeskyVecsOTF
            type(TAOBasis), intent(in)                              :: AOBasis
            integer, intent(in)                                     :: Accuracy
            real(F64), optional, intent(in)                         :: Omega

            type(gci_basis) :: b
            real(c_double), dimension(:, :), allocatable, target :: coords, coefs, exps, norms
            integer(c_int64_t), dimension(:), allocatable, target :: centers, params, lmom, nprim
            integer(c_int64_t) :: nvecs, msd, nsub, npq, nsp, npsp
            real(c_double) :: om
            integer(c_int) :: flags
            integer(c_int64_t), dimension(:, :), allocatable :: sp, spl, sb
            integer(c_int64_t), dimension(:), allocatable :: spd, sd, piv, psp, pspl, pspd, porb
            type(c_ptr) :: h

            call gci_check(gci_init())
            !
            ! TAOBasis arrays as the C ABI reads them (64-bit integers, contiguous copies)
            !
            coords = AOBasis%AtomCoords
            coefs = AOBasis%CntrCoeffs
            exps = AOBasis%Exponents
            if (AOBasis%SpherAO) then
                  norms = AOBasis%NormFactorsSpher
            else
                  norms = AOBasis%NormFactorsCart
            end if
            centers = int(AOBasis%ShellCenters, c_int64_t)
            params = int(AOBasis%ShellParamsIdx, c_int64_t)
            lmom = int(AOBasis%ShellMomentum, c_int64_t)
            nprim = int(AOBasis%NPrimitives, c_int64_t)
            b%natoms = AOBasis%NAtoms
            b%nshells = AOBasis%NShells
            b%nshellparams = AOBasis%NShellParams
            b%ldprim = size(coefs, dim=1)
            b%ldnorm = size(norms, dim=1)
            b%atom_coords = c_loc(coords)
            b%shell_centers = c_loc(centers)
            b%shell_params_idx = c_loc(params)
            b%shell_momentum = c_loc(lmom)
            b%nprimitives = c_loc(nprim)
            b%cntr_coeffs = c_loc(coefs)
            b%exponents = c_loc(exps)
            b%norm_factors = c_loc(norms)
            b%spher_ao = merge(1_c_int32_t, 0_c_int32_t, AOBasis%SpherAO)
            om = 0.0_c_double
            if (present(Omega)) om = Omega
            flags = 0
            if (chol_gammcor_store_rkpq) flags = GCI_FLAG_MATERIALIZE_RKPQ
            call gci_check(gci_rkpq(b, int(Accuracy, c_int), om, flags, h))
            CholeskyVecsOTF%Handle = h
            call gci_check(gci_query(h, nvecs, msd, nsub, npq, nsp, npsp))
            !
            ! TChol2Vecs (TwoStepCholesky_definitions.f90:56-74)
            !
            associate (C2 => CholeskyVecsOTF%Chol2Data)
                  C2%NVecs = int(nvecs)
                  C2%MaxSubsetDim = int(msd)
                  C2%NSubsets = int(nsub)
                  C2%NOrbPairs = int(npq)
                  C2%NShellPairs = int(nsp)
                  C2%NPivotShellPairs = int(npsp)
                  allocate(sp(2, nsp), spl(3, nsp), spd(nsp), sd(nsub), sb(2, nsub), piv(npq))
                  allocate(psp(npsp), pspl(npsp), pspd(npsp), porb(nvecs))
                  allocate(C2%Inv_L(nvecs, nvecs))
                  call gci_check(gci_copy_chol2data(h, sp, spl, spd, sd, sb, piv, psp, pspl, pspd, porb, C2%Inv_L))
                  C2%ShellPairs = int(sp)
                  C2%ShellPairLoc = int(spl)
                  C2%ShellPairDim = int(spd)
                  C2%SubsetDim = int(sd)
                  C2%SubsetBounds = int(sb)
                  C2%Pivots = int(piv)
                  C2%PivotShellPairs = int(psp)
                  C2%PivotShellPairLoc = int(pspl)
                  C2%PivotShellPairDim = int(pspd)
                  C2%PivotOrbPairs = int(porb)
            end associate
            if (chol_gammcor_store_rkpq) then
                  allocate(CholeskyVecsOTF%Rkpq(nvecs, msd, nsub))
                  call gci_check(gci_copy_rkpq(h, CholeskyVecsOTF%Rkpq))
            else
                  allocate(CholeskyVecsOTF%Rkpq(nvecs, msd, 0))
            end if
      end subroutine chol_gammcor_Rkpq


      subroutine chol_gammcor_Rkab(Rkab, CA, a0, a1, CB, b0, b1, MaxBufferDimMB, CholeskyVecsOTF, &
            AOBasis, ExternalOrdering)
            !
            ! Transformation of the Cholesky vectors to the MO basis: Rkab(k, ab), k fastest.
            !
            real(F64), dimension(:, :), intent(out)    :: Rkab
            real(F64), dimension(:, :), intent(in)     :: CA
            integer, intent(in)                        :: a0, a1
            real(F64), dimension(:, :), intent(in)     :: CB
            integer, intent(in)                        :: b0, b1
            integer, intent(in)                        :: MaxBufferDimMB
            type(TCholeskyVecsOTF), intent(in)         :: CholeskyVecsOTF
            type(TAOBasis), intent(in)                 :: AOBasis
            integer, intent(in)                        :: ExternalOrdering

            integer :: NCholesky, NA, NB, NAO
            real(F64), dimension(:, :), allocatable :: CA_ao, CB_ao
            logical :: TwoIndexTransf, FromExternalAO

            NA = a1 - a0 + 1
            NB = b1 - b0 + 1
            NCholesky = CholeskyVecsOTF%Chol2Data%NVecs
            if (AOBasis%SpherAO) then
                  NAO = AOBasis%NAOSpher
            else
                  NAO = AOBasis%NAOCart
            end if
            if (size(CA, dim=1) /= NAO .or. size(CB, dim=1) /= NAO) then
                  call msg("Invalid number of atomic orbitals in CA/CB")
                  error stop
            end if
            if (size(Rkab, dim=1) /= NCholesky .or. size(Rkab, dim=2) /= NA*NB) then
                  call msg("Invalid dimension of Rkab")
                  error stop
            end if
            !
            ! External AO order -> Auto2e order (and ORCA phases), as the reference does
            !
            allocate(CA_ao, mold=CA)
            allocate(CB_ao, mold=CB)
            FromExternalAO = .true.
            TwoIndexTransf = .false.
            call auto2e_interface_AngFuncTransf(CA_ao, CA, FromExternalAO, TwoIndexTransf, AOBasis, ExternalOrdering)
            call auto2e_interface_AngFuncTransf(CB_ao, CB, FromExternalAO, TwoIndexTransf, AOBasis, ExternalOrdering)
            if (ExternalOrdering == ORBITAL_ORDERING_ORCA) then
                  call auto2e_interface_ApplyOrcaPhases_Matrix(CA_ao, AOBasis, TwoIndexTransf)
                  call auto2e_interface_ApplyOrcaPhases_Matrix(CB_ao, AOBasis, TwoIndexTransf)
            end if
            call gci_check(gci_rkab(CholeskyVecsOTF%Handle, CA_ao, int(size(CA_ao, dim=1), c_int64_t), &
                  int(a0, c_int64_t), int(a1, c_int64_t), CB_ao, int(size(CB_ao, dim=1), c_int64_t), &
                  int(b0, c_int64_t), int(b1, c_int64_t), int(MaxBufferDimMB, c_int64_t), GCI_PREC_FP64, Rkab))
      end subroutine chol_gammcor_Rkab
end module Cholesky_Gammcor
