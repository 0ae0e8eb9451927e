!========================================================================================!
! fem25gpu_mod.f90 -- ISO_C_BINDING interface of libfem25gpu (include/fem25gpu.h)    !
! for the fem25 Fortran drivers.                                                         !
!                                                                                        !
! The interfaces mirror the C prototypes one to one (VALUE scalars, C_PTR for opaque    !
! handles and device buffers, assumed-size arrays for host buffers).  The wrappers in   !
! CONTAINS keep the argument lists of the reference routines they stand in for, so a    !
! driver swaps one call:                                                                 !
!   ASMBLE_DRIVER(NZLOC,CFTYPE,FREQ,PY,MSH,CDIST,IERR)       asmble.f90:1-2             !
!       -> ASMBLE_DRIVER_GPU (same arguments)   bielak25.f90:434, funcgradh.f90:191     !
!   ASMB_PEFF(MASTER,MYCOMM,NDOF,NDOFL,NZLOC,CNP,MYDOFS,IRPTR_LOC,JCPTR_LOC,             !
!             CDIST,UE,PEFF)                                 asmble.f90:318-319         !
!       -> ASMB_PEFF_GPU (same arguments)       bielak25.f90:536, funcgradh.f90:233     !
!   CFMAT_DIST + ADJGRAD's ADJFLAM_DIST/SAXPY on GRADL       hessloc.f90:1,             !
!       adjgrad.f90:63-76 -> CFMAT_ADJGRAD_GPU  funcgradh.f90:279-295                    !
!   UPDMOD's model update (gengmask.f90:657) -> FEM25_UPDATE_MODEL                       !
! Single-process use (NPARTS = 1): NZLOC = NZERO, MYDOFS = 1..NDOF.                      !
! Build: compile with the drivers (it INCLUDEs 'fwd_struc.h' for MESH_INFO) and link    !
! libfem25gpu.so.                                                                        !
!========================================================================================!
MODULE FEM25GPU
  USE ISO_C_BINDING
  IMPLICIT NONE
  PRIVATE :: FILL_MESH
  INTEGER, PARAMETER :: FEM25_OK = 0, FEM25_PREC_FP64 = 0, FEM25_PREC_TF32X3 = 1, &
                        FEM25_PREC_TF32X3_POINTWISE = 2
  ! fem25_mesh of fem25gpu.h: the MESH_INFO fields the library reads
  TYPE, BIND(C) :: FEM25_MESH
     INTEGER(C_INT) :: NELEM, NNPG, NORD, LDISP
     TYPE(C_PTR)    :: IENG, CDOMAIN, CNNPG, XLOCS, ZLOCS, XD, ZD, ECOEFF, DENS
     REAL(C_DOUBLE) :: XWIDTH, ZWIDTH
     REAL(C_DOUBLE) :: RCOEFF_SRF, DMAX_SRF, KAPPA_SRF, FCENT_SRF
     REAL(C_DOUBLE) :: RCOEFF_BDY, DMAX_BDY, KAPPA_BDY, FCENT_BDY
     TYPE(C_PTR)    :: QP, QS
     REAL(C_DOUBLE) :: FREQ0
  END TYPE
  ! the device context of the run (created by the first wrapper call)
  TYPE(C_PTR), SAVE :: FEM25_CTX = C_NULL_PTR

  INTERFACE
     INTEGER(C_INT) FUNCTION FEM25_CREATE(M, NDOF, NZERO, LM, IRPTR, JCPTR, CNP, DEVICE, OUT) &
                    BIND(C, NAME='fem25_create')
       IMPORT :: C_INT, C_LONG_LONG, C_PTR, C_CHAR, FEM25_MESH
       TYPE(FEM25_MESH), INTENT(IN) :: M
       INTEGER(C_INT), VALUE :: NDOF, DEVICE
       INTEGER(C_LONG_LONG), VALUE :: NZERO
       INTEGER(C_INT), INTENT(IN) :: LM(*), IRPTR(*), JCPTR(*)
       CHARACTER(KIND=C_CHAR), INTENT(IN) :: CNP(*)
       TYPE(C_PTR), INTENT(OUT) :: OUT
     END FUNCTION
     SUBROUTINE FEM25_DESTROY(CTX) BIND(C, NAME='fem25_destroy')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: CTX
     END SUBROUTINE
     INTEGER(C_INT) FUNCTION FEM25_LAST_ERROR(CTX, BUF, N) BIND(C, NAME='fem25_last_error')
       IMPORT :: C_INT, C_PTR, C_CHAR
       TYPE(C_PTR), VALUE :: CTX
       CHARACTER(KIND=C_CHAR), INTENT(OUT) :: BUF(*)
       INTEGER(C_INT), VALUE :: N
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_UPDATE_MODEL(CTX, ECOEFF, DENS) &
                    BIND(C, NAME='fem25_update_model')
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: CTX
       REAL(C_DOUBLE), INTENT(IN) :: ECOEFF(*), DENS(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_ASMBLE_DRIVER(CTX, NZLOC, CFTYPE, FREQ, PY, CDIST) &
                    BIND(C, NAME='fem25_asmble_driver')
       IMPORT :: C_INT, C_PTR, C_CHAR, C_DOUBLE, C_FLOAT_COMPLEX
       TYPE(C_PTR), VALUE :: CTX
       INTEGER(C_INT), VALUE :: NZLOC
       CHARACTER(KIND=C_CHAR), VALUE :: CFTYPE
       REAL(C_DOUBLE), VALUE :: FREQ, PY
       COMPLEX(C_FLOAT_COMPLEX), INTENT(OUT) :: CDIST(*)
     END FUNCTION
     ! CDIST may be C_NULL_PTR: the last ASMBLE_DRIVER system, kept on the device
     INTEGER(C_INT) FUNCTION FEM25_ASMB_PEFF(CTX, NDOF, CDIST, UE, PEFF) &
                    BIND(C, NAME='fem25_asmb_peff')
       IMPORT :: C_INT, C_PTR, C_FLOAT_COMPLEX
       TYPE(C_PTR), VALUE :: CTX, CDIST
       INTEGER(C_INT), VALUE :: NDOF
       COMPLEX(C_FLOAT_COMPLEX), INTENT(IN) :: UE(*)
       COMPLEX(C_FLOAT_COMPLEX), INTENT(OUT) :: PEFF(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_CFMAT_ADJGRAD(CTX, CINVTYPE, VPVS, FREQ, PY, WAVE, ADJLAM, &
                    ACCUMULATE, GRADL) BIND(C, NAME='fem25_cfmat_adjgrad')
       IMPORT :: C_INT, C_PTR, C_CHAR, C_DOUBLE, C_FLOAT, C_FLOAT_COMPLEX
       TYPE(C_PTR), VALUE :: CTX
       CHARACTER(KIND=C_CHAR), INTENT(IN) :: CINVTYPE(2)
       REAL(C_DOUBLE), VALUE :: VPVS, FREQ, PY
       COMPLEX(C_FLOAT_COMPLEX), INTENT(IN) :: WAVE(*), ADJLAM(*)
       INTEGER(C_INT), VALUE :: ACCUMULATE
       REAL(C_FLOAT), INTENT(INOUT) :: GRADL(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_REF_GRADIENT_INFO(CTX, NNPINV, NZ_FDIST, MASKG) &
                    BIND(C, NAME='fem25_ref_gradient_info')
       IMPORT :: C_INT, C_PTR, C_LONG_LONG
       TYPE(C_PTR), VALUE :: CTX
       INTEGER(C_INT), INTENT(OUT) :: NNPINV
       INTEGER(C_LONG_LONG), INTENT(OUT) :: NZ_FDIST
       INTEGER(C_INT), INTENT(OUT) :: MASKG(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_MISFIT_OPTIONS(CTX, NORM, IRESTP, IBPHASE, EPS, THRESH, &
                    DTMAX, DTMAX_OBJ) BIND(C, NAME='fem25_misfit_options')
       IMPORT :: C_INT, C_PTR, C_FLOAT
       TYPE(C_PTR), VALUE :: CTX
       INTEGER(C_INT), VALUE :: NORM, IRESTP, IBPHASE
       REAL(C_FLOAT), VALUE :: EPS, THRESH, DTMAX, DTMAX_OBJ
     END FUNCTION
     ! device-buffer entry points: arrays are device addresses (C_PTR), e.g. from
     ! cudaMalloc or CUDA Fortran; STREAM is a cudaStream_t (C_NULL_PTR = default)
     INTEGER(C_INT) FUNCTION FEM25_MISFIT_DEV(CTX, NSRC, NREC, MRDOF, YREC, FREQ, PY, AZMOD, &
                    RECV, SOL, OBS, WGHTS, EST, RHS, MISFIT, STREAM) &
                    BIND(C, NAME='fem25_misfit_dev')
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_FLOAT, C_FLOAT_COMPLEX
       TYPE(C_PTR), VALUE :: CTX, SOL, RHS, STREAM
       INTEGER(C_INT), VALUE :: NSRC, NREC
       INTEGER(C_INT), INTENT(IN) :: MRDOF(*)
       REAL(C_DOUBLE), INTENT(IN) :: YREC(*)
       REAL(C_DOUBLE), VALUE :: FREQ, PY, AZMOD
       COMPLEX(C_FLOAT_COMPLEX), INTENT(IN) :: RECV(*), OBS(*)
       REAL(C_FLOAT), INTENT(IN) :: WGHTS(*)
       COMPLEX(C_FLOAT_COMPLEX), INTENT(OUT) :: EST(*)
       REAL(C_FLOAT), INTENT(OUT) :: MISFIT(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_GRADIENT_ACCUMULATE_DEV(CTX, NPAIRS, FREQ, PY, NSRC, U, LAM, &
                    STREAM) BIND(C, NAME='fem25_gradient_accumulate_dev')
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: CTX, U, LAM, STREAM
       INTEGER(C_INT), VALUE :: NPAIRS, NSRC
       REAL(C_DOUBLE), INTENT(IN) :: FREQ(*), PY(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_GRADIENT_FINALIZE_DEV(CTX, GRAD, STREAM) &
                    BIND(C, NAME='fem25_gradient_finalize_dev')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: CTX, GRAD, STREAM
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_SYNC_STATUS(CTX, STREAM) BIND(C, NAME='fem25_sync_status')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: CTX, STREAM
     END FUNCTION
     ! sparse direct solve on the GPU in place of CMUMPS (bielak25.f90:334-335,
     ! 443-446, 545-551; adjgrad.f90:327-341); CSR128 and RHS are device buffers
     INTEGER(C_INT) FUNCTION FEM25_SPARSE_FACTOR_DEV(CTX, CSR128, STREAM) &
                    BIND(C, NAME='fem25_sparse_factor_dev')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: CTX, CSR128, STREAM
     END FUNCTION
     INTEGER(C_INT) FUNCTION FEM25_SPARSE_SOLVE_DEV(CTX, NRHS, TRANS, RHS, STREAM) &
                    BIND(C, NAME='fem25_sparse_solve_dev')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: CTX, RHS, STREAM
       INTEGER(C_INT), VALUE :: NRHS, TRANS
     END FUNCTION
  END INTERFACE

CONTAINS

  ! fem25_mesh view of MESH_INFO (fwd_struc.h:10-141); the pointer arrays are
  ! contiguous, so C_LOC of their first element is the array
  SUBROUTINE FILL_MESH(MSH, M)
    INCLUDE 'fwd_struc.h'
    TYPE (MESH_INFO), TARGET, INTENT(IN) :: MSH
    TYPE(FEM25_MESH), INTENT(OUT) :: M
    M%NELEM = MSH%NELEM
    M%NNPG  = MSH%NNPG
    M%NORD  = MSH%NORD
    M%LDISP = 0
    IF (MSH%LDISP) M%LDISP = 1
    M%IENG    = C_LOC(MSH%IENG(1,1))
    M%CDOMAIN = C_LOC(MSH%CDOMAIN(1))
    M%CNNPG   = C_LOC(MSH%CNNPG(1))
    M%XLOCS   = C_LOC(MSH%XLOCS(1))
    M%ZLOCS   = C_LOC(MSH%ZLOCS(1))
    M%XD      = C_LOC(MSH%XD(1))
    M%ZD      = C_LOC(MSH%ZD(1))
    M%ECOEFF  = C_LOC(MSH%ECOEFF(1,1))
    M%DENS    = C_LOC(MSH%DENS(1))
    M%XWIDTH = MSH%XWIDTH
    M%ZWIDTH = MSH%ZWIDTH
    M%RCOEFF_SRF = MSH%RCOEFF_SRF
    M%DMAX_SRF   = MSH%DMAX_SRF
    M%KAPPA_SRF  = MSH%KAPPA_SRF
    M%FCENT_SRF  = MSH%FCENT_SRF
    M%RCOEFF_BDY = MSH%RCOEFF_BDY
    M%DMAX_BDY   = MSH%DMAX_BDY
    M%KAPPA_BDY  = MSH%KAPPA_BDY
    M%FCENT_BDY  = MSH%FCENT_BDY
    M%QP = C_NULL_PTR
    M%QS = C_NULL_PTR
    IF (MSH%LDISP) THEN
       M%QP = C_LOC(MSH%QP(1))
       M%QS = C_LOC(MSH%QS(1))
    ENDIF
    M%FREQ0 = MSH%FREQ0
  END SUBROUTINE

  ! the run's context: mesh, model and graph (LM, IRPTR, JCPTR, CNP of
  ! GEN_GRAPH25) copied to GPU 0 on first use
  SUBROUTINE FEM25_ENSURE(MSH, IERR)
    INCLUDE 'fwd_struc.h'
    TYPE (MESH_INFO), TARGET, INTENT(IN) :: MSH
    INTEGER*4, INTENT(OUT) :: IERR
    TYPE(FEM25_MESH) :: M
    IERR = 0
    IF (C_ASSOCIATED(FEM25_CTX)) RETURN
    CALL FILL_MESH(MSH, M)
    IERR = FEM25_CREATE(M, MSH%NDOF, INT(MSH%NZERO, C_LONG_LONG), MSH%LM, MSH%IRPTR, &
                        MSH%JCPTR, MSH%CNP, 0, FEM25_CTX)
    IF (IERR /= 0) WRITE(*,*) 'fem25_ensure: fem25_create failed, IERR =', IERR
  END SUBROUTINE

  ! drop-in for ASMBLE_DRIVER (asmble.f90:1-2): the host COMPLEX*8 CDIST
  SUBROUTINE ASMBLE_DRIVER_GPU(NZLOC, CFTYPE, FREQ, PY, MSH, CDIST, IERR)
    INCLUDE 'fwd_struc.h'
    TYPE (MESH_INFO), TARGET :: MSH
    CHARACTER(1), INTENT(IN) :: CFTYPE
    REAL*8, INTENT(IN) :: FREQ, PY
    INTEGER*4, INTENT(IN) :: NZLOC
    COMPLEX*8, INTENT(OUT) :: CDIST(NZLOC)
    INTEGER*4, INTENT(OUT) :: IERR
    CALL FEM25_ENSURE(MSH, IERR)
    IF (IERR /= 0) RETURN
    IERR = FEM25_ASMBLE_DRIVER(FEM25_CTX, NZLOC, CFTYPE, FREQ, PY, CDIST)
  END SUBROUTINE

  ! drop-in for ASMB_PEFF (asmble.f90:318-377), single process: the CDIST the
  ! library assembled last is still on the GPU, so it is not uploaded again
  ! (pass it through FEM25_ASMB_PEFF with C_LOC(CDIST) to force an upload)
  SUBROUTINE ASMB_PEFF_GPU(MASTER, MYCOMM, NDOF, NDOFL, NZLOC, CNP, MYDOFS, IRPTR_LOC, &
                           JCPTR_LOC, CDIST, UE, PEFF)
    CHARACTER(1), INTENT(IN) :: CNP(NDOF)
    COMPLEX*8, INTENT(IN) :: UE(NDOF), CDIST(NZLOC)
    INTEGER*4, INTENT(IN) :: MYDOFS(NDOFL), IRPTR_LOC(NDOFL+1), JCPTR_LOC(NZLOC), &
                             NDOF, NDOFL, NZLOC, MASTER, MYCOMM
    COMPLEX*8, INTENT(OUT) :: PEFF(*)
    INTEGER*4 IERR
    IERR = FEM25_ASMB_PEFF(FEM25_CTX, NDOF, C_NULL_PTR, UE, PEFF)
    IF (IERR /= 0) WRITE(*,*) 'asmb_peff_gpu: Error', IERR
  END SUBROUTINE

  ! CFMAT_DIST (hessloc.f90:1-133) + ADJFLAM_DIST and SAXPY into GRADL
  ! (adjgrad.f90:63-76) for one source, host arrays; INV%CINVTYPE 'PP' or 'SS'
  SUBROUTINE CFMAT_ADJGRAD_GPU(CINVTYPE, VPVS, FREQ, PY, WAVE, ADJLAM, GRADL, IERR)
    CHARACTER(2), INTENT(IN) :: CINVTYPE
    REAL*8, INTENT(IN) :: VPVS, FREQ, PY
    COMPLEX*8, INTENT(IN) :: WAVE(*), ADJLAM(*)
    REAL*4, INTENT(INOUT) :: GRADL(*)
    INTEGER*4, INTENT(OUT) :: IERR
    CHARACTER(KIND=C_CHAR) :: CT(2)
    CT(1) = CINVTYPE(1:1)
    CT(2) = CINVTYPE(2:2)
    IERR = FEM25_CFMAT_ADJGRAD(FEM25_CTX, CT, VPVS, FREQ, PY, WAVE, ADJLAM, 0, GRADL)
  END SUBROUTINE

  ! frees the context (end of the run)
  SUBROUTINE FEM25_FINISH()
    IF (C_ASSOCIATED(FEM25_CTX)) CALL FEM25_DESTROY(FEM25_CTX)
    FEM25_CTX = C_NULL_PTR
  END SUBROUTINE
END MODULE FEM25GPU
