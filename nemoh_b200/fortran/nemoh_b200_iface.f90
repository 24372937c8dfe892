!--------------------------------------------------------------------------------------
! nemoh_b200_iface: ISO_C_BINDING interface to libnemoh_b200.so, and a drop-in
! replacement for the Solver's direct BEM solve.
!
! The reference Solver calls, once per problem (Solver/Core/SOLVE_BEM.f90:71,83),
!     CALL SOLVE_POTENTIAL_INFD_DIRECT(NVEL)
!     CALL SOLVE_POTENTIAL_FD_DIRECT(NVEL,AMH,NEXP)
! which read the mesh and environment from COM_VAR and leave ZIGB, ZIGS, ZPB,
! ZPS in COM_VAR. SOLVE_POTENTIAL_B200 below does the same job on the GPU for
! both depth regimes (the infinite/finite choice is made inside the library by
! the rule of SOLVE_BEM.f90:66), so SOLVE_BVP replaces its two calls by
!     CALL SOLVE_POTENTIAL_B200(NVEL,NEXP)
! The first call creates the GPU context and uploads the mesh; the factor cache
! follows the reference's w_previous (SOLVE_BEM_INFD_DIRECT.f90:82).
! Reals cross the boundary as C_DOUBLE: with default REAL kind 4 they are
! converted, with -fdefault-real-8 they pass unchanged.
!--------------------------------------------------------------------------------------
MODULE NEMOH_B200_IFACE

    USE ISO_C_BINDING
    IMPLICIT NONE

    INTEGER(C_INT), PARAMETER :: NEMOH_B200_FP64 = 0, NEMOH_B200_MIXED = 1

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
        TYPE(C_PTR) FUNCTION nemoh_b200_last_error(ctx) BIND(C, NAME='nemoh_b200_last_error')
            IMPORT :: C_PTR
            TYPE(C_PTR), VALUE :: ctx
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_set_mesh(ctx, np, nfa, nsymy, xyz, m1234, rho, g, depth) &
                BIND(C, NAME='nemoh_b200_set_mesh')
            IMPORT :: C_PTR, C_INT, C_DOUBLE
            TYPE(C_PTR), VALUE :: ctx
            INTEGER(C_INT), VALUE :: np, nfa, nsymy
            REAL(C_DOUBLE), DIMENSION(3,*) :: xyz
            INTEGER(C_INT), DIMENSION(4,*) :: m1234
            REAL(C_DOUBLE), VALUE :: rho, g, depth
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_solve_problem(ctx, period, nvel, zigb, zigs, zpb, zps, nexp) &
                BIND(C, NAME='nemoh_b200_solve_problem')
            IMPORT :: C_PTR, C_INT, C_DOUBLE, C_DOUBLE_COMPLEX
            TYPE(C_PTR), VALUE :: ctx
            REAL(C_DOUBLE), VALUE :: period
            COMPLEX(C_DOUBLE_COMPLEX), DIMENSION(*) :: nvel, zigb, zigs, zpb, zps
            INTEGER(C_INT) :: nexp
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_solve_frequencies(ctx, nomega, omegas, nrhs, nvel, nint, nds, force) &
                BIND(C, NAME='nemoh_b200_solve_frequencies')
            IMPORT :: C_PTR, C_INT, C_DOUBLE, C_DOUBLE_COMPLEX
            TYPE(C_PTR), VALUE :: ctx
            INTEGER(C_INT), VALUE :: nomega, nrhs, nint
            REAL(C_DOUBLE), DIMENSION(*) :: omegas
            COMPLEX(C_DOUBLE_COMPLEX), DIMENSION(*) :: nvel, force
            REAL(C_DOUBLE), DIMENSION(*) :: nds
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_kochin(ctx, period, xeff, yeff, ntheta, theta, nprob, zigb, zigs, &
                hkochin) BIND(C, NAME='nemoh_b200_kochin')
            IMPORT :: C_PTR, C_INT, C_DOUBLE, C_DOUBLE_COMPLEX
            TYPE(C_PTR), VALUE :: ctx
            REAL(C_DOUBLE), VALUE :: period, xeff, yeff
            INTEGER(C_INT), VALUE :: ntheta, nprob
            REAL(C_DOUBLE), DIMENSION(*) :: theta
            COMPLEX(C_DOUBLE_COMPLEX), DIMENSION(*) :: zigb, zigs, hkochin
        END FUNCTION
        INTEGER(C_INT) FUNCTION nemoh_b200_free_surface(ctx, period, npts, xy, nprob, zigb, zigs, eta) &
                BIND(C, NAME='nemoh_b200_free_surface')
            IMPORT :: C_PTR, C_INT, C_DOUBLE, C_DOUBLE_COMPLEX
            TYPE(C_PTR), VALUE :: ctx
            REAL(C_DOUBLE), VALUE :: period
            INTEGER(C_INT), VALUE :: npts, nprob
            REAL(C_DOUBLE), DIMENSION(*) :: xy
            COMPLEX(C_DOUBLE_COMPLEX), DIMENSION(*) :: zigb, zigs, eta
        END FUNCTION
    END INTERFACE

    TYPE(C_PTR), SAVE :: B200_CTX = C_NULL_PTR
    INTEGER, SAVE :: B200_MODE = 0

CONTAINS

    ! Stop with the library's message, as the reference stops on its errors
    SUBROUTINE B200_CHECK(ST, WHAT)
        INTEGER(C_INT) :: ST
        CHARACTER(*) :: WHAT
        CHARACTER(KIND=C_CHAR), POINTER :: MSG(:)
        INTEGER :: L
        IF (ST .NE. 0) THEN
            CALL C_F_POINTER(nemoh_b200_last_error(B200_CTX), MSG, [512])
            L = 0
            DO WHILE (L .LT. 512)
                IF (MSG(L+1) .EQ. C_NULL_CHAR) EXIT
                L = L + 1
            END DO
            WRITE(*,*) 'nemoh_b200 ', WHAT, ' status ', ST, ': ', MSG(1:L)
            STOP
        END IF
    END SUBROUTINE

    ! First use: context and mesh from COM_VAR (INITIALIZE has run)
    SUBROUTINE B200_INIT
        USE COM_VAR
        REAL(C_DOUBLE), ALLOCATABLE :: XYZ(:,:)
        INTEGER(C_INT), ALLOCATABLE :: MM(:,:)
        INTEGER :: I
        IF (C_ASSOCIATED(B200_CTX)) RETURN
        CALL B200_CHECK(nemoh_b200_create(B200_CTX, 0_C_INT, INT(B200_MODE, C_INT)), 'create')
        ALLOCATE(XYZ(3,NP), MM(4,NFA))
        DO I = 1, NP
            XYZ(1,I) = X(I)
            XYZ(2,I) = Y(I)
            XYZ(3,I) = Z(I)
        END DO
        DO I = 1, NFA
            MM(1,I) = M1(I)
            MM(2,I) = M2(I)
            MM(3,I) = M3(I)
            MM(4,I) = M4(I)
        END DO
        CALL B200_CHECK(nemoh_b200_set_mesh(B200_CTX, INT(NP, C_INT), INT(NFA, C_INT), INT(NSYMY, C_INT), XYZ, MM, &
                        REAL(RHO, C_DOUBLE), REAL(G, C_DOUBLE), REAL(Depth, C_DOUBLE)), 'set_mesh')
        DEALLOCATE(XYZ, MM)
    END SUBROUTINE

    ! Drop-in for SOLVE_POTENTIAL_INFD_DIRECT / SOLVE_POTENTIAL_FD_DIRECT
    SUBROUTINE SOLVE_POTENTIAL_B200(NVEL, NEXP)
        USE COM_VAR
        COMPLEX, DIMENSION(*) :: NVEL
        INTEGER :: NEXP
        COMPLEX(C_DOUBLE_COMPLEX), ALLOCATABLE :: V(:), ZB(:), ZS(:), PB(:), PS(:)
        INTEGER(C_INT) :: NE
        INTEGER :: I, NC
        CALL B200_INIT
        NC = NFA * 2**NSYMY
        ALLOCATE(V(NC), ZB(NFA), ZS(NFA), PB(NFA), PS(NFA))
        DO I = 1, NC
            V(I) = CMPLX(NVEL(I), KIND=C_DOUBLE_COMPLEX)
        END DO
        CALL B200_CHECK(nemoh_b200_solve_problem(B200_CTX, REAL(T, C_DOUBLE), V, ZB, ZS, PB, PS, NE), 'solve_problem')
        DO I = 1, NFA
            ZIGB(I) = ZB(I)
            ZIGS(I) = ZS(I)
            ZPB(I) = PB(I)
            ZPS(I) = PS(I)
        END DO
        NEXP = NE
        DEALLOCATE(V, ZB, ZS, PB, PS)
    END SUBROUTINE

    ! Drop-in for COMPUTE_KOCHIN(kwave,Theta,HKochin) (SOLVE_BEM.f90:98-102): the
    ! library derives kwave from the period T as SOLVE_BVP does and uses the
    ! source strengths ZIGB, ZIGS of the last SOLVE_POTENTIAL_B200 call.
    SUBROUTINE COMPUTE_KOCHIN_B200(Theta, HKochin)
        USE COM_VAR
        REAL :: Theta
        COMPLEX :: HKochin
        REAL(C_DOUBLE) :: TH(1)
        COMPLEX(C_DOUBLE_COMPLEX), ALLOCATABLE :: ZB(:), ZS(:)
        COMPLEX(C_DOUBLE_COMPLEX) :: H(1)
        INTEGER :: I
        ALLOCATE(ZB(NFA), ZS(NFA))
        DO I = 1, NFA
            ZB(I) = CMPLX(ZIGB(I), KIND=C_DOUBLE_COMPLEX)
            ZS(I) = CMPLX(ZIGS(I), KIND=C_DOUBLE_COMPLEX)
        END DO
        TH(1) = REAL(Theta, C_DOUBLE)
        CALL B200_CHECK(nemoh_b200_kochin(B200_CTX, REAL(T, C_DOUBLE), REAL(XEFF, C_DOUBLE), REAL(YEFF, C_DOUBLE), &
                        1_C_INT, TH, 1_C_INT, ZB, ZS, H), 'kochin')
        HKochin = H(1)
        DEALLOCATE(ZB, ZS)
    END SUBROUTINE

    ! Drop-in for the free-surface loop of SOLVE_BVP (SOLVE_BEM.f90:104-109):
    ! ETA(j) = II*W/G*PHI(j) at the points MeshFS%X(1:2, j), from the source
    ! strengths ZIGB, ZIGS of the last SOLVE_POTENTIAL_B200 call.
    SUBROUTINE COMPUTE_FS_B200(NPOINTS, XFS, ETA)
        USE COM_VAR
        INTEGER :: NPOINTS
        REAL, DIMENSION(3, *) :: XFS
        COMPLEX, DIMENSION(*) :: ETA
        REAL(C_DOUBLE), ALLOCATABLE :: XY(:)
        COMPLEX(C_DOUBLE_COMPLEX), ALLOCATABLE :: ZB(:), ZS(:), E(:)
        INTEGER :: I
        IF (NPOINTS .LE. 0) RETURN
        ALLOCATE(XY(2 * NPOINTS), E(NPOINTS), ZB(NFA), ZS(NFA))
        DO I = 1, NPOINTS
            XY(2 * I - 1) = REAL(XFS(1, I), C_DOUBLE)
            XY(2 * I) = REAL(XFS(2, I), C_DOUBLE)
        END DO
        DO I = 1, NFA
            ZB(I) = CMPLX(ZIGB(I), KIND=C_DOUBLE_COMPLEX)
            ZS(I) = CMPLX(ZIGS(I), KIND=C_DOUBLE_COMPLEX)
        END DO
        CALL B200_CHECK(nemoh_b200_free_surface(B200_CTX, REAL(T, C_DOUBLE), INT(NPOINTS, C_INT), XY, 1_C_INT, &
                        ZB, ZS, E), 'free_surface')
        DO I = 1, NPOINTS
            ETA(I) = CMPLX(E(I))
        END DO
        DEALLOCATE(XY, E, ZB, ZS)
    END SUBROUTINE

    SUBROUTINE B200_FINALIZE
        INTEGER(C_INT) :: ST
        IF (C_ASSOCIATED(B200_CTX)) ST = nemoh_b200_destroy(B200_CTX)
        B200_CTX = C_NULL_PTR
    END SUBROUTINE

END MODULE NEMOH_B200_IFACE
