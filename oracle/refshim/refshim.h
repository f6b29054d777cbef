/*
 * refshim.h -- single-process stand-in for the PETSc / SLEPc / MPI / LAPACK
 * interfaces that the reference PolyStokes sources call, so that those sources
 * compile unmodified into the oracle build (oracle/_ref/).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this.
 *
 * What is restated here is library arithmetic, from published descriptions:
 *   - KSPMINRES: preconditioned MINRES (Paige & Saunders, SIAM J. Numer. Anal.
 *     12 (1975) 617), with PETSc's default convergence test (preconditioned
 *     residual norm <= max(rtol * ||B r0||, abstol), ||B b|| for a nonzero
 *     initial guess), divergence on an indefinite preconditioner, maxit 10000.
 *   - PCJACOBI with the fix-diagonal option: zero diagonal entries become 1.
 *     The diagonal is taken afresh at every KSPSolve.
 *   - dense MatMult / MatMultTranspose / MatMatTransposeMult / MatAXPY and
 *     the AIJ (sparse rows) and shell matrix kinds.
 *   - LAPACK dsyev: cyclic Jacobi eigenvalue method (Golub & Van Loan,
 *     Matrix Computations, 4th ed., sec. 8.5), eigenvalues ascending,
 *     eigenvectors in the columns.
 *   - SLEPc MFN with FNSQRT: sqrt(M) b by symmetric Lanczos with full
 *     reorthogonalisation, sqrt taken on the projected tridiagonal (implicit QL,
 *     Golub & Van Loan sec. 8.3) every 5 vectors, stopped when the estimate
 *     changes by less than 1e-13 relative; a negative projected eigenvalue (M
 *     indefinite: no real square root) stops it with a negative converged reason.
 *   - MPI: one rank; collectives copy.
 * Everything the reference computes in its own code (geometry, tensors,
 * assembly, forces, drift, integrator, Schur floor, output) stays the
 * reference's.
 *
 * Hooks for parity fixtures (environment variables, read by this shim only):
 *   ORACLE_KSP_RTOL   overrides the rtol that KSPSetTolerances sets;
 *   ORACLE_REF_DUMP   file to which every KSPSolve appends (n, warm, reason,
 *                     iterations, rhs, solution) and every MFNSolve appends
 *                     (n, reason, input, output), as little-endian binary;
 *   ORACLE_REF_DUMP_MAT  if set, every KSPSolve on a dense operator also
 *                     appends the operator (column-major n*n doubles).
 */
#ifndef REFSHIM_H
#define REFSHIM_H

/* standard headers that the PETSc headers bring in for C++ translation units */
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

typedef int PetscInt;
typedef int PetscMPIInt;
typedef int PetscBLASInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscErrorCode;
typedef int PetscLogEvent;
typedef int PetscClassId;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define PETSC_COMM_WORLD ((MPI_Comm)1)
#define PETSC_COMM_SELF ((MPI_Comm)2)
#define MPIU_SCALAR ((MPI_Datatype)1)
#define MPIU_SUM ((MPI_Op)1)

#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_ERR_SUP 56
#define PETSC_ERR_ARG_WRONG 62

typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { MAT_INITIAL_MATRIX, MAT_REUSE_MATRIX, MAT_IGNORE_MATRIX, MAT_INPLACE_MATRIX } MatReuse;
typedef enum { MAT_DO_NOT_COPY_VALUES, MAT_COPY_VALUES, MAT_SHARE_NONZERO_PATTERN } MatDuplicateOption;
typedef enum { DIFFERENT_NONZERO_PATTERN, SUBSET_NONZERO_PATTERN, SAME_NONZERO_PATTERN, UNKNOWN_NONZERO_PATTERN } MatStructure;
typedef enum { MATOP_MULT, MATOP_GET_DIAGONAL, MATOP_DESTROY } MatOperation;
typedef enum { NORM_1, NORM_2, NORM_FROBENIUS, NORM_INFINITY } NormType;
typedef enum { SCATTER_FORWARD = 0, SCATTER_REVERSE = 1 } ScatterMode;
typedef int KSPConvergedReason;
typedef int MFNConvergedReason;
typedef const char *MatType;
typedef const char *KSPType;
typedef const char *PCType;
typedef const char *FNType;
#define MATDENSE "dense"
#define MATSEQAIJ "seqaij"
#define KSPMINRES "minres"
#define PCJACOBI "jacobi"
#define FNSQRT "sqrt"

struct _p_Vec;
struct _p_Mat;
struct _p_KSP;
struct _p_PC;
struct _p_IS;
struct _p_VecScatter;
struct _p_MFN;
struct _p_FN;
struct _p_Viewer;
typedef struct _p_Vec *Vec;
typedef struct _p_Mat *Mat;
typedef struct _p_KSP *KSP;
typedef struct _p_PC *PC;
typedef struct _p_IS *IS;
typedef struct _p_VecScatter *VecScatter;
typedef struct _p_MFN *MFN;
typedef struct _p_FN *FN;
typedef struct _p_Viewer *PetscViewer;
#define PETSC_VIEWER_STDOUT_WORLD ((PetscViewer)0)

typedef PetscErrorCode (*PetscErrorHandlerFn)(MPI_Comm, int, const char *, const char *, PetscErrorCode, int,
                                              const char *, void *);

/* errors: the reference installs PetscAbortErrorHandler, so any error aborts */
void refshim_error(const char *file, int line, PetscErrorCode ierr);
#define CHKERRQ(e) do { PetscErrorCode _e = (e); if (_e) { refshim_error(__FILE__, __LINE__, _e); return _e; } } while (0)
#define CHKERRV(e) do { PetscErrorCode _e = (e); if (_e) { refshim_error(__FILE__, __LINE__, _e); return; } } while (0)

/* system */
PetscErrorCode SlepcInitialize(int *argc, char ***args, const char *file, const char *help);
PetscErrorCode SlepcFinalize(void);
PetscErrorCode PetscAbortErrorHandler(MPI_Comm, int, const char *, const char *, PetscErrorCode, int, const char *,
                                      void *);
PetscErrorCode PetscPushErrorHandler(PetscErrorHandlerFn h, void *ctx);
PetscErrorCode PetscInitialized(PetscBool *flg);
PetscErrorCode PetscFinalized(PetscBool *flg);
PetscErrorCode PetscPrintf(MPI_Comm comm, const char *fmt, ...);
PetscErrorCode PetscLogDefaultBegin(void);
PetscErrorCode PetscLogView(PetscViewer v);
PetscErrorCode PetscLogEventRegister(const char *name, PetscClassId cls, PetscLogEvent *ev);
/* the first event of a run is check_dist() of step 1 (run.cpp:72-73): its time marks the end of
 * init() and fill_self(); refshim_first_event_time() returns it (CLOCK_MONOTONIC seconds) */
void refshim_event_begin(PetscLogEvent ev);
inline PetscErrorCode PetscLogEventBegin(PetscLogEvent ev, int, int, int, int) { refshim_event_begin(ev); return 0; }
inline PetscErrorCode PetscLogEventEnd(PetscLogEvent, int, int, int, int) { return 0; }
inline PetscReal PetscRealPart(PetscScalar a) { return a; }
inline PetscReal PetscAbsScalar(PetscScalar a) { return std::fabs(a); }
inline PetscReal PetscSqrtReal(PetscReal a) { return std::sqrt(a); }
inline PetscErrorCode PetscBLASIntCast(PetscInt a, PetscBLASInt *b) { *b = (PetscBLASInt)a; return 0; }

/* MPI, one rank */
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Allgatherv(const void *send, int scount, MPI_Datatype st, void *recv, const int *rcounts, const int *displs,
                   MPI_Datatype rt, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);

/* Vec */
PetscErrorCode VecCreate(MPI_Comm comm, Vec *v);
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N);
PetscErrorCode VecSetFromOptions(Vec v);
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec *v);
PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec *v);
PetscErrorCode VecDuplicate(Vec v, Vec *w);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecSet(Vec v, PetscScalar a);
PetscErrorCode VecZeroEntries(Vec v);
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a);
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecScale(Vec x, PetscScalar a);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar *d);
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *n);
PetscErrorCode VecSetValues(Vec x, PetscInt ni, const PetscInt *ix, const PetscScalar *y, InsertMode mode);
PetscErrorCode VecGetSize(Vec x, PetscInt *n);
PetscErrorCode VecGetLocalSize(Vec x, PetscInt *n);
PetscErrorCode VecMAXPY(Vec y, PetscInt nv, const PetscScalar *alpha, Vec *x);

/* IS / VecScatter */
PetscErrorCode ISCreateStride(MPI_Comm comm, PetscInt n, PetscInt first, PetscInt step, IS *is);
PetscErrorCode ISDestroy(IS *is);
PetscErrorCode VecScatterCreate(Vec x, IS ix, Vec y, IS iy, VecScatter *sc);
PetscErrorCode VecScatterBegin(VecScatter sc, Vec x, Vec y, InsertMode mode, ScatterMode smode);
PetscErrorCode VecScatterEnd(VecScatter sc, Vec x, Vec y, InsertMode mode, ScatterMode smode);
PetscErrorCode VecScatterDestroy(VecScatter *sc);

/* Mat */
PetscErrorCode MatCreate(MPI_Comm comm, Mat *A);
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N);
PetscErrorCode MatSetType(Mat A, MatType t);
PetscErrorCode MatSetUp(Mat A);
PetscErrorCode MatCreateSeqAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt nz, const PetscInt *nnz, Mat *A);
PetscErrorCode MatCreateShell(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, void *ctx, Mat *A);
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void));
PetscErrorCode MatShellGetContext(Mat A, void *ctx);
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt *im, PetscInt n, const PetscInt *in,
                            const PetscScalar *v, InsertMode mode);
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode);
PetscErrorCode MatGetValues(Mat A, PetscInt m, const PetscInt *im, PetscInt n, const PetscInt *in, PetscScalar *v);
PetscErrorCode MatAssemblyBegin(Mat A, MatAssemblyType t);
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType t);
PetscErrorCode MatZeroEntries(Mat A);
PetscErrorCode MatDestroy(Mat *A);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z);
PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y);
PetscErrorCode MatGetDiagonal(Mat A, Vec d);
PetscErrorCode MatCopy(Mat A, Mat B, MatStructure s);
PetscErrorCode MatAXPY(Mat Y, PetscScalar a, Mat X, MatStructure s);
PetscErrorCode MatScale(Mat A, PetscScalar a);
PetscErrorCode MatNorm(Mat A, NormType t, PetscReal *n);
PetscErrorCode MatDuplicate(Mat A, MatDuplicateOption op, Mat *B);
PetscErrorCode MatGetSize(Mat A, PetscInt *m, PetscInt *n);
PetscErrorCode MatMatTransposeMult(Mat A, Mat B, MatReuse r, PetscReal fill, Mat *C);
PetscErrorCode MatDenseGetArray(Mat A, PetscScalar **a);
PetscErrorCode MatDenseRestoreArray(Mat A, PetscScalar **a);
PetscErrorCode MatDenseGetArrayRead(Mat A, const PetscScalar **a);
PetscErrorCode MatDenseRestoreArrayRead(Mat A, const PetscScalar **a);
PetscErrorCode MatDenseGetSubMatrix(Mat A, PetscInt rbegin, PetscInt rend, PetscInt cbegin, PetscInt cend, Mat *v);
PetscErrorCode MatDenseRestoreSubMatrix(Mat A, Mat *v);

/* KSP / PC */
PetscErrorCode KSPCreate(MPI_Comm comm, KSP *ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat P);
PetscErrorCode KSPSetType(KSP ksp, KSPType t);
PetscErrorCode KSPGetPC(KSP ksp, PC *pc);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits);
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool flg);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *r);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its);
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal *rn);
PetscErrorCode KSPDestroy(KSP *ksp);
PetscErrorCode PCSetType(PC pc, PCType t);
PetscErrorCode PCJacobiSetFixDiagonal(PC pc, PetscBool flg);

/* SLEPc */
PetscErrorCode FNCreate(MPI_Comm comm, FN *fn);
PetscErrorCode FNSetType(FN fn, FNType t);
PetscErrorCode MFNCreate(MPI_Comm comm, MFN *mfn);
PetscErrorCode MFNSetFN(MFN mfn, FN fn);
PetscErrorCode MFNSetFromOptions(MFN mfn);
PetscErrorCode MFNSetOperator(MFN mfn, Mat A);
PetscErrorCode MFNSolve(MFN mfn, Vec b, Vec x);
PetscErrorCode MFNGetConvergedReason(MFN mfn, MFNConvergedReason *r);

/* LAPACK */
extern "C" void LAPACKsyev_(const char *jobz, const char *uplo, const PetscBLASInt *n, PetscScalar *a,
                            const PetscBLASInt *lda, PetscReal *w, PetscScalar *work, const PetscBLASInt *lwork,
                            PetscBLASInt *info);

#endif
