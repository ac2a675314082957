!==============================================================================!
! fvg_bind.f90 - ISO_C_BINDING interface to the B200 mode-split step (fvg.h).
!
! Drop-in for FVCOM's SUBROUTINE INTERNAL_STEP (FVCOM_source/internal_step.F:29) and
! SUBROUTINE EXTERNAL_STEP (FVCOM_source/external_step.F:30).  FVG_SETUP is called once
! after GRID_METRICS and STARTUP (fvcom.F:629, 753); FVG_INTERNAL_STEP replaces the call
! at fvcom.F:852; FVG_PULL copies the prognostic fields back before ARCHIVE (fvcom.F:874).
!
! Arrays FVCOM allocates without a ghost row (NBSN, NBVE, NBVT, DLTXTRIE.., IEC, IENODE,
! NIEC, NTRG, DLTXE, DLTYE, DLTXNCVE, DLTYNCVE) are copied into ghost-rowed buffers here;
! everything else is passed by address.  Compiled with the FVCOM build (serial, DOUBLE_PRECISION,
! GCN, LIMITED_NO, WET_DRY); no Fortran compiler exists on the build machine of this library.
!==============================================================================!
MODULE FVG_BIND
  USE ISO_C_BINDING
  IMPLICIT NONE

  TYPE, BIND(C) :: FVG_MESH_T
    INTEGER(C_INT32_T) :: M, N, KB, NE, NCV, NCV_I, NBSN_COLS, NBVE_COLS, TRIE_COLS
    TYPE(C_PTR) :: VX, VY, H, ART1, ART2, GRAV_N, NN_HVC, SITA_GD, PHPN
    TYPE(C_PTR) :: ISONB, NTSN, NTVE, NBSN, NBVE, NBVT
    TYPE(C_PTR) :: DLTXTRIE, DLTYTRIE, DLTXECEC, DLTYECEC, DLTXNEC, DLTYNEC
    TYPE(C_PTR) :: Z, ZZ, DZ, DZZ
    TYPE(C_PTR) :: XC, YC, ART, H1, COR, GRAV_E, CC_HVC, CC_SPONGE, CC_Z0B, EPOR, IUCP, ALPHA
    TYPE(C_PTR) :: NV, NBE, ISBCE, A1U, A2U, AWX, AWY, Z1, ZZ1, DZ1, DZZ1
    TYPE(C_PTR) :: IEC, IENODE, ISBC, XIJC, YIJC, DLTXC, DLTYC
    TYPE(C_PTR) :: NIEC, NTRG, DLTXE, DLTYE, DLTXNCVE, DLTYNCVE
    INTEGER(C_INT32_T) :: IOBCN
    TYPE(C_PTR) :: I_OBC_N, TYPE_OBC, NEXT_OBC, NADJC_OBC, ADJC_OBC, FLUXF_OBC, DLTN_OBC
    INTEGER(C_INT32_T) :: NUMQBC
    TYPE(C_PTR) :: INODEQ, ICELLQ, N_ICELLQ, RDISQ, QAREA, ANGLEQ, VQDIST
  END TYPE FVG_MESH_T

  TYPE, BIND(C) :: FVG_PARAMS_T
    REAL(C_DOUBLE) :: DTE
    INTEGER(C_INT32_T) :: ISPLIT, IRAMP
    REAL(C_DOUBLE) :: MIN_DEPTH, STATIC_SSH_ADJ
    INTEGER(C_INT32_T) :: HORIZONTAL_MIXING
    REAL(C_DOUBLE) :: HPRNU, UMOL, VPRNU, CBCMIN
    INTEGER(C_INT32_T) :: VERTICAL_MIXING, WETTING_DRYING_ON, SCALAR_POSITIVITY_CONTROL
    INTEGER(C_INT32_T) :: BAROTROPIC, TEMPERATURE_ACTIVE, SALINITY_ACTIVE
    INTEGER(C_INT32_T) :: OBC_ELEVATION_FORCING_ON, OBC_TS_TYPE, RIVER_TS_SETTING, RIVER_LOCATION
    REAL(C_DOUBLE) :: TIDE_REF_TIME
    INTEGER(C_INT32_T) :: HEATING_ON
    REAL(C_DOUBLE) :: RHEAT, ZETA1, ZETA2
    INTEGER(C_INT32_T) :: LIMITER        ! 0 LIMITED_NO, 1 LIMITED_1, 2 slope limiter alone
    INTEGER(C_INT32_T) :: BAROPG_Z       ! 1: BAROCLINIC_PRESSURE_GRADIENT = 'z coordinates'
    INTEGER(C_INT32_T) :: GHOST_CELLS    ! 0: GCN build, 1: GCY1 or GCY2 build
  END TYPE FVG_PARAMS_T

  TYPE, BIND(C) :: FVG_FORCING_T
    INTEGER(C_INT32_T) :: NTIDE
    TYPE(C_PTR) :: PERIOD, APT, PHAI, EMEAN, QDIS, TDIS, SDIS, WSTRESS_X, WSTRESS_Y
    TYPE(C_PTR) :: SWRAD, WTSURF
  END TYPE FVG_FORCING_T

  INTERFACE
    INTEGER(C_INT) FUNCTION fvg_create(mesh, params, forcing, handle) BIND(C, NAME="fvg_create")
      IMPORT :: C_INT, C_PTR, FVG_MESH_T, FVG_PARAMS_T, FVG_FORCING_T
      TYPE(FVG_MESH_T), INTENT(IN) :: mesh
      TYPE(FVG_PARAMS_T), INTENT(IN) :: params
      TYPE(FVG_FORCING_T), INTENT(IN) :: forcing
      TYPE(C_PTR), INTENT(OUT) :: handle
    END FUNCTION
    SUBROUTINE fvg_destroy(handle) BIND(C, NAME="fvg_destroy")
      IMPORT :: C_PTR
      TYPE(C_PTR), VALUE :: handle
    END SUBROUTINE
    INTEGER(C_INT) FUNCTION fvg_set_field(handle, name, src, cnt) BIND(C, NAME="fvg_set_field")
      IMPORT :: C_INT, C_PTR, C_CHAR, C_INT64_T
      TYPE(C_PTR), VALUE :: handle
      CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: name
      TYPE(C_PTR), VALUE :: src
      INTEGER(C_INT64_T), VALUE :: cnt
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_get_field(handle, name, dst, cnt) BIND(C, NAME="fvg_get_field")
      IMPORT :: C_INT, C_PTR, C_CHAR, C_INT64_T
      TYPE(C_PTR), VALUE :: handle
      CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: name
      TYPE(C_PTR), VALUE :: dst
      INTEGER(C_INT64_T), VALUE :: cnt
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_set_ifield(handle, name, src, cnt) BIND(C, NAME="fvg_set_ifield")
      IMPORT :: C_INT, C_PTR, C_CHAR, C_INT64_T
      TYPE(C_PTR), VALUE :: handle
      CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: name
      TYPE(C_PTR), VALUE :: src
      INTEGER(C_INT64_T), VALUE :: cnt
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_set_clock(handle, iint, ext_time) BIND(C, NAME="fvg_set_clock")
      IMPORT :: C_INT, C_PTR, C_INT32_T, C_DOUBLE
      TYPE(C_PTR), VALUE :: handle
      INTEGER(C_INT32_T), VALUE :: iint
      REAL(C_DOUBLE), VALUE :: ext_time
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_internal_step(handle) BIND(C, NAME="fvg_internal_step")
      IMPORT :: C_INT, C_PTR
      TYPE(C_PTR), VALUE :: handle
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_shutdown_check(handle) BIND(C, NAME="fvg_shutdown_check")
      IMPORT :: C_INT, C_PTR
      TYPE(C_PTR), VALUE :: handle
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_get_ifield(handle, name, dst, cnt) BIND(C, NAME="fvg_get_ifield")
      IMPORT :: C_INT, C_PTR, C_CHAR, C_INT64_T
      TYPE(C_PTR), VALUE :: handle
      CHARACTER(KIND=C_CHAR), DIMENSION(*), INTENT(IN) :: name
      TYPE(C_PTR), VALUE :: dst
      INTEGER(C_INT64_T), VALUE :: cnt
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_set_forcing(handle, forcing) BIND(C, NAME="fvg_set_forcing")
      IMPORT :: C_INT, C_PTR, FVG_FORCING_T
      TYPE(C_PTR), VALUE :: handle
      TYPE(FVG_FORCING_T), INTENT(IN) :: forcing
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_run(handle, nsteps) BIND(C, NAME="fvg_run")
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE :: handle
      INTEGER(C_INT32_T), VALUE :: nsteps
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_set_precision(handle, mode) BIND(C, NAME="fvg_set_precision")
      IMPORT :: C_INT, C_PTR, C_INT32_T
      TYPE(C_PTR), VALUE :: handle
      INTEGER(C_INT32_T), VALUE :: mode
    END FUNCTION
    INTEGER(C_INT) FUNCTION fvg_budget(handle, out) BIND(C, NAME="fvg_budget")
      IMPORT :: C_INT, C_PTR, C_DOUBLE
      TYPE(C_PTR), VALUE :: handle
      REAL(C_DOUBLE), DIMENSION(3), INTENT(OUT) :: out
    END FUNCTION
    FUNCTION fvg_last_error(handle) BIND(C, NAME="fvg_last_error")
      IMPORT :: C_PTR
      TYPE(C_PTR), VALUE :: handle
      TYPE(C_PTR) :: fvg_last_error
    END FUNCTION
  END INTERFACE

  TYPE(C_PTR), SAVE :: FVG_HANDLE = C_NULL_PTR

CONTAINS

  ! Copy of an (1:L, 1:C) array with a zero ghost row 0, as fvg.h expects.
  FUNCTION GHOSTED_I(A, L, NC) RESULT(B)
    INTEGER, INTENT(IN) :: L, NC, A(L, NC)
    INTEGER, ALLOCATABLE :: B(:,:)
    ALLOCATE(B(0:L, NC)); B = 0; B(1:L, :) = A
  END FUNCTION GHOSTED_I

  SUBROUTINE PUSH(NAME, A)
    CHARACTER(LEN=*), INTENT(IN) :: NAME
    REAL(C_DOUBLE), TARGET, INTENT(IN) :: A(:,:)
    INTEGER(C_INT) :: RC
    RC = fvg_set_field(FVG_HANDLE, TRIM(NAME)//C_NULL_CHAR, C_LOC(A), INT(SIZE(A), C_INT64_T))
    IF (RC /= 0) CALL FATAL_ERROR("fvg_set_field failed for "//TRIM(NAME))
  END SUBROUTINE PUSH

  SUBROUTINE PULL(NAME, A)
    CHARACTER(LEN=*), INTENT(IN) :: NAME
    REAL(C_DOUBLE), TARGET, INTENT(INOUT) :: A(:,:)
    INTEGER(C_INT) :: RC
    RC = fvg_get_field(FVG_HANDLE, TRIM(NAME)//C_NULL_CHAR, C_LOC(A), INT(SIZE(A), C_INT64_T))
    IF (RC /= 0) CALL FATAL_ERROR("fvg_get_field failed for "//TRIM(NAME))
  END SUBROUTINE PULL

  ! Forcing of the coming internal step (the river, wind and heating arrays BCOND_GCN(8)
  ! updated on the host, UPDATE_RIVERS / UPDATE_WIND / UPDATE_HEAT), handed over before
  ! FVG_INTERNAL_STEP; FRC's pointers are C_LOC of FVCOM's arrays, as for FVG_CREATE.
  SUBROUTINE FVG_FORCE(FRC)
    TYPE(FVG_FORCING_T), INTENT(IN) :: FRC
    INTEGER(C_INT) :: RC
    RC = fvg_set_forcing(FVG_HANDLE, FRC)
    IF (RC /= 0) CALL FATAL_ERROR("fvg_set_forcing failed")
  END SUBROUTINE FVG_FORCE

  ! Replacement for CALL INTERNAL_STEP at fvcom.F:852.  IntTime was advanced by the caller;
  ! the library advances IINT and ExtTime (ISPLIT*DTE) itself.
  SUBROUTINE FVG_INTERNAL_STEP
    USE ALL_VARS, ONLY: IINT
    USE MOD_TIME, ONLY: ExtTime
    INTEGER(C_INT) :: RC
    RC = fvg_set_clock(FVG_HANDLE, INT(IINT - 1, C_INT32_T), REAL(SECONDS(ExtTime), C_DOUBLE))
    RC = fvg_internal_step(FVG_HANDLE)
    IF (RC /= 0) CALL FATAL_ERROR("fvg_internal_step failed")
  END SUBROUTINE FVG_INTERNAL_STEP

END MODULE FVG_BIND
