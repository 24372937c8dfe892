!--------------------------------------------------------------------------------------
! nemoh_b200_irf: drop-in for the post-processor's Compute_IRF
! (postProcessor/IRF.f90:100-127) on the GPU through libnemoh_b200.so.
!
! postProcessor/Main.f90:75-78 calls
!     CALL Compute_IRF(IRF,Results)
! which COMPUTE_IRF_B200(IRF,Results) replaces: the impulse response functions
! IRF%K and the infinite-frequency added mass IRF%AddedMass from
! Results%RadiationDamping and Results%AddedMass, for the times IRF%Time set by
! Initialize_IRF. Kept apart from nemoh_b200_iface.f90 because it uses the
! post-processor's own modules (MIRF, MResults).
!--------------------------------------------------------------------------------------
MODULE NEMOH_B200_IRF

    USE ISO_C_BINDING
    USE MIRF
    USE MResults
    IMPLICIT NONE

    INTERFACE
        INTEGER(C_INT) FUNCTION nemoh_b200_create(ctx, device, mode) BIND(C, NAME='nemoh_b200_create')
            IMPORT :: C_PTR, C_INT
            TYPE(C_PTR) :: ctx
            INTEGER(C_INT), VALUE :: device, mode
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_destroy(ctx) BIND(C, NAME='nemoh_b200_destroy')
            IMPORT :: C_PTR, C_INT
            TYPE(C_PTR), VALUE :: ctx
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_irf(ctx, nw, w, nrad, nint, damping, added_mass, ntime, dt, K, ainf) &
                BIND(C, NAME='nemoh_b200_irf')
            IMPORT :: C_PTR, C_INT, C_DOUBLE
            TYPE(C_PTR), VALUE :: ctx
            INTEGER(C_INT), VALUE :: nw, nrad, nint, ntime
            REAL(C_DOUBLE), VALUE :: dt
            REAL(C_DOUBLE), DIMENSION(*) :: w, damping, added_mass, K, ainf
        END FUNCTION
    END INTERFACE

CONTAINS

    SUBROUTINE COMPUTE_IRF_B200(IRF, Results)
        TYPE(TIRF) :: IRF
        TYPE(TResults) :: Results
        TYPE(C_PTR) :: CTX
        REAL(C_DOUBLE), ALLOCATABLE :: W(:), B(:,:,:), A(:,:,:), K(:,:,:), AINF(:,:)
        REAL(C_DOUBLE) :: DT
        INTEGER(C_INT) :: ST
        INTEGER :: NW, NR, NI, NT
        NW = Results%Nw
        NR = Results%Nradiation
        NI = Results%Nintegration
        NT = IRF%Ntime
        ALLOCATE(W(NW), B(NW, NR, NI), A(NW, NR, NI), K(0:NT-1, NR, NI), AINF(NR, NI))
        W = REAL(Results%w(1:NW), C_DOUBLE)
        B = REAL(Results%RadiationDamping(1:NW, 1:NR, 1:NI), C_DOUBLE)
        A = REAL(Results%AddedMass(1:NW, 1:NR, 1:NI), C_DOUBLE)
        DT = 0.
        IF (NT .GT. 1) DT = REAL(IRF%Time(1) - IRF%Time(0), C_DOUBLE)
        IF (NT .LE. 1) DT = 1.
        CTX = C_NULL_PTR
        ST = nemoh_b200_create(CTX, 0_C_INT, 0_C_INT)
        IF (ST .EQ. 0) ST = nemoh_b200_irf(CTX, INT(NW, C_INT), W, INT(NR, C_INT), INT(NI, C_INT), B, A, &
                                           INT(NT, C_INT), DT, K, AINF)
        IF (C_ASSOCIATED(CTX)) ST = MAX(ST, nemoh_b200_destroy(CTX))
        IF (ST .NE. 0) THEN
            WRITE(*,*) ' Error: nemoh_b200_irf failed, status ', ST
            STOP
        END IF
        IRF%K(0:NT-1, 1:NR, 1:NI) = K
        IRF%AddedMass(1:NR, 1:NI) = AINF
        DEALLOCATE(W, B, A, K, AINF)
    END SUBROUTINE

END MODULE NEMOH_B200_IRF
