/*
 * refshim.cpp -- implementation of refshim.h (see there for scope and the
 * published algorithms restated).  TEST INFRASTRUCTURE ONLY.
 */
#include "refshim.h"

#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <ctime>
#include <string>
#include <unordered_map>
#include <vector>

/* ------------------------------------------------------------------------- */
/* objects                                                                    */
/* ------------------------------------------------------------------------- */
struct _p_Vec {
    PetscInt n = -1;
    std::vector<PetscScalar> a;
};

enum MatKind { MK_NONE, MK_DENSE, MK_AIJ, MK_SHELL };

struct _p_Mat {
    MatKind kind = MK_NONE;
    PetscInt m = 0, n = 0;
    /* dense: column-major, element (i,j) at a[i + j*lda]; a points into store or a parent's store */
    std::vector<PetscScalar> store;
    PetscScalar *a = nullptr;
    PetscInt lda = 0;
    /* aij: per-row column -> value */
    std::vector<std::unordered_map<PetscInt, PetscScalar>> rows;
    /* shell */
    void *ctx = nullptr;
    PetscErrorCode (*mult)(Mat, Vec, Vec) = nullptr;
    PetscErrorCode (*getdiag)(Mat, Vec) = nullptr;
    PetscErrorCode (*destroy)(Mat) = nullptr;
};

struct _p_PC {
    bool jacobi = false;
    bool fixdiag = false;
};

struct _p_KSP {
    Mat A = nullptr;
    PC pc = nullptr;
    PetscReal rtol = 1e-5, abstol = 1e-50, dtol = 1e5;
    PetscInt maxit = 10000;
    bool nonzero_guess = false;
    PetscInt its = 0;
    PetscReal rnorm = 0;
    KSPConvergedReason reason = 0;
};

struct _p_IS {
    std::vector<PetscInt> idx;
};

struct _p_VecScatter {
    std::vector<PetscInt> to;   /* y[to[i]] (+)= x[i] */
};

struct _p_FN {
    bool sqrt = false;
};

struct _p_MFN {
    FN fn = nullptr;
    Mat A = nullptr;
    MFNConvergedReason reason = 0;
};

/* ------------------------------------------------------------------------- */
/* system                                                                     */
/* ------------------------------------------------------------------------- */
void refshim_error(const char *file, int line, PetscErrorCode ierr)
{
    std::fprintf(stderr, "[refshim] PETSc-style error %d at %s:%d; the reference's PetscAbortErrorHandler aborts\n",
                 (int)ierr, file, line);
    std::fflush(stderr);
    std::abort();
}

static bool g_init = false, g_final = false;
PetscErrorCode SlepcInitialize(int *, char ***, const char *, const char *) { g_init = true; return 0; }
PetscErrorCode SlepcFinalize(void) { g_final = true; return 0; }
PetscErrorCode PetscAbortErrorHandler(MPI_Comm, int line, const char *, const char *file, PetscErrorCode e, int,
                                      const char *, void *)
{
    refshim_error(file ? file : "?", line, e);
    return e;
}
PetscErrorCode PetscPushErrorHandler(PetscErrorHandlerFn, void *) { return 0; }
PetscErrorCode PetscInitialized(PetscBool *f) { *f = g_init ? PETSC_TRUE : PETSC_FALSE; return 0; }
PetscErrorCode PetscFinalized(PetscBool *f) { *f = g_final ? PETSC_TRUE : PETSC_FALSE; return 0; }
PetscErrorCode PetscLogDefaultBegin(void) { return 0; }
PetscErrorCode PetscLogView(PetscViewer) { return 0; }
static double g_first_event = -1.0;
void refshim_event_begin(PetscLogEvent)
{
    if (g_first_event < 0) {
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        g_first_event = (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
    }
}
extern "C" __attribute__((visibility("default"))) double refshim_first_event_time(void) { return g_first_event; }

PetscErrorCode PetscLogEventRegister(const char *, PetscClassId, PetscLogEvent *ev)
{
    static int next = 1;
    *ev = next++;
    return 0;
}

PetscErrorCode PetscPrintf(MPI_Comm, const char *fmt, ...)
{
    /* PETSc's %D is its PetscInt conversion; PetscInt is int here */
    std::string f(fmt);
    for (size_t p = f.find("%D"); p != std::string::npos; p = f.find("%D", p)) f.replace(p, 2, "%d");
    va_list ap;
    va_start(ap, fmt);
    std::vprintf(f.c_str(), ap);
    va_end(ap);
    std::fflush(stdout);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* MPI, one rank                                                              */
/* ------------------------------------------------------------------------- */
int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype, MPI_Op, MPI_Comm)
{
    if (s != r) std::memmove(r, s, sizeof(PetscScalar) * (size_t)count);
    return 0;
}
int MPI_Allgatherv(const void *s, int scount, MPI_Datatype, void *r, const int *, const int *displs, MPI_Datatype,
                   MPI_Comm)
{
    std::memmove((PetscScalar *)r + displs[0], s, sizeof(PetscScalar) * (size_t)scount);
    return 0;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

/* ------------------------------------------------------------------------- */
/* dumps for parity fixtures                                                  */
/* ------------------------------------------------------------------------- */
static FILE *dump_file()
{
    static FILE *f = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        const char *p = std::getenv("ORACLE_REF_DUMP");
        if (p && *p) f = std::fopen(p, "ab");
    }
    return f;
}
static void dump_header(FILE *f, int tag, int n, int a, int b)
{
    int h[4] = {tag, n, a, b};
    std::fwrite(h, sizeof(int), 4, f);
}

/* ------------------------------------------------------------------------- */
/* Vec                                                                        */
/* ------------------------------------------------------------------------- */
PetscErrorCode VecCreate(MPI_Comm, Vec *v) { *v = new _p_Vec(); return 0; }
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N) { v->n = (N != PETSC_DECIDE) ? N : n; return 0; }
PetscErrorCode VecSetFromOptions(Vec v) { v->a.assign((size_t)std::max(v->n, 0), 0.0); return 0; }
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec *v)
{
    *v = new _p_Vec();
    (*v)->n = n;
    (*v)->a.assign((size_t)n, 0.0);
    return 0;
}
PetscErrorCode VecCreateMPI(MPI_Comm c, PetscInt n, PetscInt N, Vec *v) { return VecCreateSeq(c, N > 0 ? N : n, v); }
PetscErrorCode VecDuplicate(Vec v, Vec *w) { return VecCreateSeq(PETSC_COMM_SELF, v->n, w); }
PetscErrorCode VecDestroy(Vec *v) { delete *v; *v = nullptr; return 0; }
PetscErrorCode VecSet(Vec v, PetscScalar a) { std::fill(v->a.begin(), v->a.end(), a); return 0; }
PetscErrorCode VecZeroEntries(Vec v) { return VecSet(v, 0.0); }
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a.data(); return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar **a) { *a = nullptr; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) { *a = v->a.data(); return 0; }
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **a) { *a = nullptr; return 0; }
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x)
{
    for (PetscInt i = 0; i < y->n; i++) y->a[i] += a * x->a[i];
    return 0;
}
PetscErrorCode VecScale(Vec x, PetscScalar a)
{
    for (auto &e : x->a) e *= a;
    return 0;
}
PetscErrorCode VecCopy(Vec x, Vec y) { y->a = x->a; y->n = x->n; return 0; }
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar *d)
{
    PetscScalar s = 0;
    for (PetscInt i = 0; i < x->n; i++) s += y->a[i] * x->a[i];
    *d = s;
    return 0;
}
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *n)
{
    if (t != NORM_2) return PETSC_ERR_SUP;
    PetscReal s = 0;
    for (PetscInt i = 0; i < x->n; i++) s += x->a[i] * x->a[i];
    *n = std::sqrt(s);
    return 0;
}
PetscErrorCode VecSetValues(Vec x, PetscInt ni, const PetscInt *ix, const PetscScalar *y, InsertMode mode)
{
    for (PetscInt i = 0; i < ni; i++) {
        if (ix[i] < 0) continue;
        if (ix[i] >= x->n) return PETSC_ERR_ARG_WRONG;
        if (mode == ADD_VALUES) x->a[ix[i]] += y[i]; else x->a[ix[i]] = y[i];
    }
    return 0;
}
PetscErrorCode VecGetSize(Vec x, PetscInt *n) { *n = x->n; return 0; }
PetscErrorCode VecGetLocalSize(Vec x, PetscInt *n) { *n = x->n; return 0; }
PetscErrorCode VecMAXPY(Vec y, PetscInt nv, const PetscScalar *alpha, Vec *x)
{
    for (PetscInt k = 0; k < nv; k++) VecAXPY(y, alpha[k], x[k]);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* IS / scatter                                                               */
/* ------------------------------------------------------------------------- */
PetscErrorCode ISCreateStride(MPI_Comm, PetscInt n, PetscInt first, PetscInt step, IS *is)
{
    *is = new _p_IS();
    (*is)->idx.resize((size_t)n);
    for (PetscInt i = 0; i < n; i++) (*is)->idx[i] = first + i * step;
    return 0;
}
PetscErrorCode ISDestroy(IS *is) { delete *is; *is = nullptr; return 0; }
PetscErrorCode VecScatterCreate(Vec x, IS ix, Vec, IS iy, VecScatter *sc)
{
    if (ix) return PETSC_ERR_SUP;
    *sc = new _p_VecScatter();
    if (iy) (*sc)->to = iy->idx;
    else { (*sc)->to.resize((size_t)x->n); for (PetscInt i = 0; i < x->n; i++) (*sc)->to[i] = i; }
    return 0;
}
PetscErrorCode VecScatterBegin(VecScatter sc, Vec x, Vec y, InsertMode mode, ScatterMode smode)
{
    if (smode != SCATTER_FORWARD) return PETSC_ERR_SUP;
    for (size_t i = 0; i < sc->to.size(); i++) {
        if (mode == ADD_VALUES) y->a[sc->to[i]] += x->a[i]; else y->a[sc->to[i]] = x->a[i];
    }
    return 0;
}
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
PetscErrorCode VecScatterDestroy(VecScatter *sc) { delete *sc; *sc = nullptr; return 0; }

/* ------------------------------------------------------------------------- */
/* Mat                                                                        */
/* ------------------------------------------------------------------------- */
static void dense_alloc(Mat A)
{
    A->store.assign((size_t)A->m * (size_t)A->n, 0.0);
    A->a = A->store.data();
    A->lda = A->m;
}
PetscErrorCode MatCreate(MPI_Comm, Mat *A) { *A = new _p_Mat(); return 0; }
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N)
{
    A->m = (M != PETSC_DECIDE) ? M : m;
    A->n = (N != PETSC_DECIDE) ? N : n;
    return 0;
}
PetscErrorCode MatSetType(Mat A, MatType t)
{
    if (!std::strcmp(t, MATDENSE)) A->kind = MK_DENSE;
    else if (!std::strcmp(t, MATSEQAIJ)) A->kind = MK_AIJ;
    else return PETSC_ERR_SUP;
    return 0;
}
PetscErrorCode MatSetUp(Mat A)
{
    if (A->kind == MK_DENSE) dense_alloc(A);
    else if (A->kind == MK_AIJ) A->rows.assign((size_t)A->m, {});
    return 0;
}
PetscErrorCode MatCreateSeqAIJ(MPI_Comm, PetscInt m, PetscInt n, PetscInt, const PetscInt *, Mat *A)
{
    *A = new _p_Mat();
    (*A)->kind = MK_AIJ;
    (*A)->m = m;
    (*A)->n = n;
    (*A)->rows.assign((size_t)m, {});
    return 0;
}
PetscErrorCode MatCreateShell(MPI_Comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, void *ctx, Mat *A)
{
    *A = new _p_Mat();
    (*A)->kind = MK_SHELL;
    (*A)->m = M > 0 ? M : m;
    (*A)->n = N > 0 ? N : n;
    (*A)->ctx = ctx;
    return 0;
}
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void))
{
    if (op == MATOP_MULT) A->mult = (PetscErrorCode(*)(Mat, Vec, Vec))f;
    else if (op == MATOP_GET_DIAGONAL) A->getdiag = (PetscErrorCode(*)(Mat, Vec))f;
    else if (op == MATOP_DESTROY) A->destroy = (PetscErrorCode(*)(Mat))f;
    return 0;
}
PetscErrorCode MatShellGetContext(Mat A, void *ctx) { *(void **)ctx = A->ctx; return 0; }

PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt *im, PetscInt n, const PetscInt *in,
                            const PetscScalar *v, InsertMode mode)
{
    /* values are row-oriented: v[i*n + j] goes to (im[i], in[j]); negative indices are skipped */
    if (A->kind == MK_SHELL) {
        std::fprintf(stderr, "[refshim] MatSetValues on a shell matrix: no MATOP_SET_VALUES\n");
        return PETSC_ERR_SUP;
    }
    for (PetscInt i = 0; i < m; i++) {
        PetscInt r = im[i];
        if (r < 0) continue;
        if (r >= A->m) return PETSC_ERR_ARG_WRONG;
        for (PetscInt j = 0; j < n; j++) {
            PetscInt c = in[j];
            if (c < 0) continue;
            if (c >= A->n) return PETSC_ERR_ARG_WRONG;
            PetscScalar val = v[(size_t)i * n + j];
            if (A->kind == MK_DENSE) {
                PetscScalar &e = A->a[r + (size_t)c * A->lda];
                if (mode == ADD_VALUES) e += val; else e = val;
            } else {
                PetscScalar &e = A->rows[r][c];
                if (mode == ADD_VALUES) e += val; else e = val;
            }
        }
    }
    return 0;
}
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode)
{
    return MatSetValues(A, 1, &i, 1, &j, &v, mode);
}
static PetscScalar mat_get(Mat A, PetscInt r, PetscInt c)
{
    if (A->kind == MK_DENSE) return A->a[r + (size_t)c * A->lda];
    auto it = A->rows[r].find(c);
    return it == A->rows[r].end() ? 0.0 : it->second;
}
PetscErrorCode MatGetValues(Mat A, PetscInt m, const PetscInt *im, PetscInt n, const PetscInt *in, PetscScalar *v)
{
    if (A->kind != MK_DENSE && A->kind != MK_AIJ) return PETSC_ERR_SUP;
    for (PetscInt i = 0; i < m; i++)
        for (PetscInt j = 0; j < n; j++) v[(size_t)i * n + j] = mat_get(A, im[i], in[j]);
    return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatZeroEntries(Mat A)
{
    if (A->kind == MK_DENSE) {
        for (PetscInt j = 0; j < A->n; j++) std::fill(A->a + (size_t)j * A->lda, A->a + (size_t)j * A->lda + A->m, 0.0);
    } else if (A->kind == MK_AIJ) {
        for (auto &r : A->rows) for (auto &kv : r) kv.second = 0.0;
    }
    return 0;
}
PetscErrorCode MatDestroy(Mat *A)
{
    if (*A && (*A)->kind == MK_SHELL && (*A)->destroy) (*A)->destroy(*A);
    delete *A;
    *A = nullptr;
    return 0;
}

/* y = A x; dense columns are accumulated in ascending column order */
static PetscErrorCode mult_into(Mat A, const PetscScalar *x, PetscScalar *y)
{
    if (A->kind == MK_DENSE) {
        /* four columns per sweep of y (a blocked column-oriented gemv) */
        std::fill(y, y + A->m, 0.0);
        PetscInt j = 0;
        for (; j + 4 <= A->n; j += 4) {
            const PetscScalar x0 = x[j], x1 = x[j + 1], x2 = x[j + 2], x3 = x[j + 3];
            const PetscScalar *c0 = A->a + (size_t)j * A->lda, *c1 = c0 + A->lda, *c2 = c1 + A->lda, *c3 = c2 + A->lda;
            for (PetscInt i = 0; i < A->m; i++) y[i] += c0[i] * x0 + c1[i] * x1 + c2[i] * x2 + c3[i] * x3;
        }
        for (; j < A->n; j++) {
            const PetscScalar xj = x[j];
            const PetscScalar *col = A->a + (size_t)j * A->lda;
            for (PetscInt i = 0; i < A->m; i++) y[i] += col[i] * xj;
        }
        return 0;
    }
    if (A->kind == MK_AIJ) {
        for (PetscInt i = 0; i < A->m; i++) {
            PetscScalar s = 0;
            for (auto &kv : A->rows[i]) s += kv.second * x[kv.first];
            y[i] = s;
        }
        return 0;
    }
    return PETSC_ERR_SUP;
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y)
{
    if (A->kind == MK_SHELL) return A->mult ? A->mult(A, x, y) : PETSC_ERR_SUP;
    if (x->n != A->n || y->n != A->m) return PETSC_ERR_ARG_WRONG;
    if (x == y) {
        std::vector<PetscScalar> t((size_t)A->m);
        PetscErrorCode e = mult_into(A, x->a.data(), t.data());
        y->a = t;
        return e;
    }
    return mult_into(A, x->a.data(), y->a.data());
}
PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z)
{
    std::vector<PetscScalar> t((size_t)A->m);
    if (A->kind == MK_SHELL) return PETSC_ERR_SUP;
    PetscErrorCode e = mult_into(A, x->a.data(), t.data());
    for (PetscInt i = 0; i < A->m; i++) z->a[i] = y->a[i] + t[i];
    return e;
}
PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y)
{
    if (x->n != A->m || y->n != A->n) return PETSC_ERR_ARG_WRONG;
    std::vector<PetscScalar> t((size_t)A->n, 0.0);
    if (A->kind == MK_DENSE) {
        for (PetscInt j = 0; j < A->n; j++) {
            const PetscScalar *col = A->a + (size_t)j * A->lda;
            PetscScalar s = 0;
            for (PetscInt i = 0; i < A->m; i++) s += col[i] * x->a[i];
            t[j] = s;
        }
    } else if (A->kind == MK_AIJ) {
        for (PetscInt i = 0; i < A->m; i++)
            for (auto &kv : A->rows[i]) t[kv.first] += kv.second * x->a[i];
    } else {
        return PETSC_ERR_SUP;
    }
    y->a = t;
    return 0;
}
PetscErrorCode MatGetDiagonal(Mat A, Vec d)
{
    if (A->kind == MK_SHELL) return A->getdiag ? A->getdiag(A, d) : PETSC_ERR_SUP;
    for (PetscInt i = 0; i < std::min(A->m, A->n); i++) d->a[i] = mat_get(A, i, i);
    return 0;
}
PetscErrorCode MatCopy(Mat A, Mat B, MatStructure)
{
    if (A->kind != MK_DENSE || B->kind != MK_DENSE || A->m != B->m || A->n != B->n) return PETSC_ERR_SUP;
    for (PetscInt j = 0; j < A->n; j++)
        for (PetscInt i = 0; i < A->m; i++) B->a[i + (size_t)j * B->lda] = A->a[i + (size_t)j * A->lda];
    return 0;
}
PetscErrorCode MatAXPY(Mat Y, PetscScalar a, Mat X, MatStructure)
{
    if (Y->kind != MK_DENSE || X->kind != MK_DENSE || Y->m != X->m || Y->n != X->n) return PETSC_ERR_SUP;
    for (PetscInt j = 0; j < Y->n; j++)
        for (PetscInt i = 0; i < Y->m; i++) Y->a[i + (size_t)j * Y->lda] += a * X->a[i + (size_t)j * X->lda];
    return 0;
}
PetscErrorCode MatScale(Mat A, PetscScalar a)
{
    if (A->kind != MK_DENSE) return PETSC_ERR_SUP;
    for (PetscInt j = 0; j < A->n; j++)
        for (PetscInt i = 0; i < A->m; i++) A->a[i + (size_t)j * A->lda] *= a;
    return 0;
}
PetscErrorCode MatNorm(Mat A, NormType t, PetscReal *n)
{
    if (A->kind != MK_DENSE || t != NORM_FROBENIUS) return PETSC_ERR_SUP;
    PetscReal s = 0;
    for (PetscInt j = 0; j < A->n; j++)
        for (PetscInt i = 0; i < A->m; i++) { PetscScalar v = A->a[i + (size_t)j * A->lda]; s += v * v; }
    *n = std::sqrt(s);
    return 0;
}
PetscErrorCode MatDuplicate(Mat A, MatDuplicateOption op, Mat *B)
{
    if (A->kind != MK_DENSE) return PETSC_ERR_SUP;
    *B = new _p_Mat();
    (*B)->kind = MK_DENSE;
    (*B)->m = A->m;
    (*B)->n = A->n;
    dense_alloc(*B);
    if (op == MAT_COPY_VALUES) return MatCopy(A, *B, SAME_NONZERO_PATTERN);
    return 0;
}
PetscErrorCode MatGetSize(Mat A, PetscInt *m, PetscInt *n)
{
    if (m) *m = A->m;
    if (n) *n = A->n;
    return 0;
}
PetscErrorCode MatMatTransposeMult(Mat A, Mat B, MatReuse, PetscReal, Mat *C)
{
    /* C = A B^T */
    if (A->kind != MK_DENSE || B->kind != MK_DENSE || A->n != B->n) return PETSC_ERR_SUP;
    *C = new _p_Mat();
    (*C)->kind = MK_DENSE;
    (*C)->m = A->m;
    (*C)->n = B->m;
    dense_alloc(*C);
    for (PetscInt j = 0; j < B->m; j++)
        for (PetscInt i = 0; i < A->m; i++) {
            PetscScalar s = 0;
            for (PetscInt k = 0; k < A->n; k++) s += A->a[i + (size_t)k * A->lda] * B->a[j + (size_t)k * B->lda];
            (*C)->a[i + (size_t)j * (*C)->lda] = s;
        }
    return 0;
}
PetscErrorCode MatDenseGetArray(Mat A, PetscScalar **a) { if (A->kind != MK_DENSE) return PETSC_ERR_SUP; *a = A->a; return 0; }
PetscErrorCode MatDenseRestoreArray(Mat, PetscScalar **a) { *a = nullptr; return 0; }
PetscErrorCode MatDenseGetArrayRead(Mat A, const PetscScalar **a) { if (A->kind != MK_DENSE) return PETSC_ERR_SUP; *a = A->a; return 0; }
PetscErrorCode MatDenseRestoreArrayRead(Mat, const PetscScalar **a) { *a = nullptr; return 0; }
PetscErrorCode MatDenseGetSubMatrix(Mat A, PetscInt rbegin, PetscInt rend, PetscInt cbegin, PetscInt cend, Mat *v)
{
    if (A->kind != MK_DENSE) return PETSC_ERR_SUP;
    *v = new _p_Mat();
    (*v)->kind = MK_DENSE;
    (*v)->m = rend - rbegin;
    (*v)->n = cend - cbegin;
    (*v)->lda = A->lda;
    (*v)->a = A->a + rbegin + (size_t)cbegin * A->lda;
    return 0;
}
PetscErrorCode MatDenseRestoreSubMatrix(Mat, Mat *v) { delete *v; *v = nullptr; return 0; }

/* ------------------------------------------------------------------------- */
/* KSP: preconditioned MINRES with Jacobi                                     */
/* ------------------------------------------------------------------------- */
PetscErrorCode KSPCreate(MPI_Comm, KSP *ksp)
{
    *ksp = new _p_KSP();
    (*ksp)->pc = new _p_PC();
    return 0;
}
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat) { ksp->A = A; return 0; }
PetscErrorCode KSPSetType(KSP, KSPType t) { return std::strcmp(t, KSPMINRES) ? PETSC_ERR_SUP : 0; }
PetscErrorCode KSPGetPC(KSP ksp, PC *pc) { *pc = ksp->pc; return 0; }
PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits)
{
    if (rtol != PETSC_DEFAULT) ksp->rtol = rtol;
    if (abstol != PETSC_DEFAULT) ksp->abstol = abstol;
    if (dtol != PETSC_DEFAULT) ksp->dtol = dtol;
    if (maxits != PETSC_DEFAULT) ksp->maxit = maxits;
    const char *e = std::getenv("ORACLE_KSP_RTOL");
    if (e && *e) ksp->rtol = std::atof(e);
    return 0;
}
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool f) { ksp->nonzero_guess = (f == PETSC_TRUE); return 0; }
PetscErrorCode PCSetType(PC pc, PCType t) { pc->jacobi = !std::strcmp(t, PCJACOBI); return pc->jacobi ? 0 : PETSC_ERR_SUP; }
PetscErrorCode PCJacobiSetFixDiagonal(PC pc, PetscBool f) { pc->fixdiag = (f == PETSC_TRUE); return 0; }

static PetscScalar dotv(const std::vector<PetscScalar> &a, const std::vector<PetscScalar> &b)
{
    PetscScalar s = 0;
    for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
    return s;
}

PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x)
{
    Mat A = ksp->A;
    const PetscInt n = b->n;
    PetscErrorCode ierr;
    /* Jacobi: 1/diag(A) with zero entries replaced by 1 (fix-diagonal) */
    Vec d;
    VecCreateSeq(PETSC_COMM_SELF, n, &d);
    if ((ierr = MatGetDiagonal(A, d))) return ierr;
    std::vector<PetscScalar> Dinv((size_t)n);
    for (PetscInt i = 0; i < n; i++) {
        PetscScalar v = d->a[i];
        if (v == 0.0 && ksp->pc->fixdiag) v = 1.0;
        Dinv[i] = 1.0 / v;
    }
    VecDestroy(&d);
    const bool warm = ksp->nonzero_guess;
    Vec R1, R2, Y, V, W, W1, W2;
    VecCreateSeq(PETSC_COMM_SELF, n, &R1); VecCreateSeq(PETSC_COMM_SELF, n, &R2);
    VecCreateSeq(PETSC_COMM_SELF, n, &Y); VecCreateSeq(PETSC_COMM_SELF, n, &V);
    VecCreateSeq(PETSC_COMM_SELF, n, &W); VecCreateSeq(PETSC_COMM_SELF, n, &W1); VecCreateSeq(PETSC_COMM_SELF, n, &W2);
    std::vector<PetscScalar> rhs0 = b->a;
    if (warm) {
        if ((ierr = MatMult(A, x, Y))) return ierr;
        for (PetscInt i = 0; i < n; i++) R1->a[i] = b->a[i] - Y->a[i];
    } else {
        std::fill(x->a.begin(), x->a.end(), 0.0);
        R1->a = b->a;
    }
    for (PetscInt i = 0; i < n; i++) Y->a[i] = R1->a[i] * Dinv[i];
    PetscReal np0 = std::sqrt(dotv(Y->a, Y->a)), ref = np0;
    if (warm) {
        PetscReal acc = 0;
        for (PetscInt i = 0; i < n; i++) { PetscScalar z = b->a[i] * Dinv[i]; acc += z * z; }
        ref = std::sqrt(acc);
    }
    PetscReal ttol = std::max(ksp->rtol * ref, ksp->abstol);
    PetscReal beta1 = dotv(R1->a, Y->a);
    KSPConvergedReason reason = 0;
    PetscInt k = 0;
    PetscReal np = np0;
    if (beta1 < 0) {
        reason = -8; /* KSP_DIVERGED_INDEFINITE_PC */
    } else {
        beta1 = std::sqrt(beta1);
        if (np0 <= ttol || beta1 == 0.0) {
            reason = 2; /* KSP_CONVERGED_RTOL */
        } else {
            R2->a = R1->a;
            PetscReal oldb = 0, beta = beta1, dbar = 0, epsln = 0, phibar = beta1, cs = -1, sn = 0;
            for (k = 1; k <= ksp->maxit; k++) {
                PetscReal sinv = 1.0 / beta;
                for (PetscInt i = 0; i < n; i++) V->a[i] = sinv * Y->a[i];
                if ((ierr = MatMult(A, V, Y))) return ierr;
                if (k >= 2) for (PetscInt i = 0; i < n; i++) Y->a[i] -= (beta / oldb) * R1->a[i];
                PetscReal alfa = dotv(V->a, Y->a);
                for (PetscInt i = 0; i < n; i++) Y->a[i] -= (alfa / beta) * R2->a[i];
                std::swap(R1, R2);
                R2->a = Y->a;
                for (PetscInt i = 0; i < n; i++) Y->a[i] = R2->a[i] * Dinv[i];
                oldb = beta;
                PetscReal bb = dotv(R2->a, Y->a);
                if (bb < 0) { reason = -8; break; }
                beta = std::sqrt(bb);
                PetscReal oldeps = epsln;
                PetscReal delta = cs * dbar + sn * alfa;
                PetscReal gbar = sn * dbar - cs * alfa;
                epsln = sn * beta;
                dbar = -cs * beta;
                PetscReal gamma = std::sqrt(gbar * gbar + beta * beta);
                if (gamma < 2.2250738585072014e-308) gamma = 2.2250738585072014e-308;
                cs = gbar / gamma;
                sn = beta / gamma;
                PetscReal phi = cs * phibar;
                phibar = sn * phibar;
                PetscReal denom = 1.0 / gamma;
                std::swap(W1, W2);   /* W1 <- old W2 */
                std::swap(W2, W);    /* W2 <- old W; W takes old W1's storage, overwritten below */
                for (PetscInt i = 0; i < n; i++) W->a[i] = (V->a[i] - oldeps * W1->a[i] - delta * W2->a[i]) * denom;
                for (PetscInt i = 0; i < n; i++) x->a[i] += phi * W->a[i];
                np = np * std::fabs(sn);
                if (!(np == np)) { reason = -9; break; } /* KSP_DIVERGED_NANORINF */
                if (np <= ttol) { reason = 2; break; }
                if (beta == 0.0) { reason = 3; break; }
            }
            if (k > ksp->maxit) { reason = -3; k = ksp->maxit; } /* KSP_DIVERGED_ITS */
        }
    }
    ksp->its = k;
    ksp->rnorm = np;
    ksp->reason = reason;
    VecDestroy(&R1); VecDestroy(&R2); VecDestroy(&Y); VecDestroy(&V);
    VecDestroy(&W); VecDestroy(&W1); VecDestroy(&W2);
    if (FILE *f = dump_file()) {
        if (std::getenv("ORACLE_REF_DUMP_MAT") && A->kind == MK_DENSE) {
            dump_header(f, 'A', n, 0, 0);
            for (PetscInt j = 0; j < n; j++) std::fwrite(A->a + (size_t)j * A->lda, sizeof(PetscScalar), (size_t)n, f);
        }
        dump_header(f, 'K', n, warm ? 1 : 0, reason);
        int its = (int)k;
        std::fwrite(&its, sizeof(int), 1, f);
        std::fwrite(rhs0.data(), sizeof(PetscScalar), (size_t)n, f);
        std::fwrite(x->a.data(), sizeof(PetscScalar), (size_t)n, f);
        std::fflush(f);
    }
    return 0;
}
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *r) { *r = ksp->reason; return 0; }
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its) { *its = ksp->its; return 0; }
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal *rn) { *rn = ksp->rnorm; return 0; }
PetscErrorCode KSPDestroy(KSP *ksp)
{
    if (*ksp) delete (*ksp)->pc;
    delete *ksp;
    *ksp = nullptr;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* symmetric eigen: cyclic Jacobi                                             */
/* ------------------------------------------------------------------------- */
/* a: n x n symmetric, column-major (lda); on return lam ascending and, if vec,
 * a's columns hold the matching orthonormal eigenvectors. */
static void jacobi_eig(PetscInt n, PetscScalar *a, PetscInt lda, PetscReal *lam, bool vec)
{
    std::vector<double> S((size_t)n * n), Q((size_t)n * n, 0.0);
    for (PetscInt j = 0; j < n; j++)
        for (PetscInt i = 0; i < n; i++) S[i + (size_t)j * n] = a[i + (size_t)j * lda];
    for (PetscInt i = 0; i < n; i++) Q[i + (size_t)i * n] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (PetscInt j = 0; j < n; j++)
            for (PetscInt i = 0; i < n; i++) {
                double v = S[i + (size_t)j * n] * S[i + (size_t)j * n];
                tot += v;
                if (i != j) off += v;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (PetscInt p = 0; p < n - 1; p++)
            for (PetscInt q = p + 1; q < n; q++) {
                double apq = S[p + (size_t)q * n];
                if (apq == 0.0) continue;
                double app = S[p + (size_t)p * n], aqq = S[q + (size_t)q * n];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (PetscInt k = 0; k < n; k++) {   /* columns p, q */
                    double skp = S[k + (size_t)p * n], skq = S[k + (size_t)q * n];
                    S[k + (size_t)p * n] = c * skp - s * skq;
                    S[k + (size_t)q * n] = s * skp + c * skq;
                }
                for (PetscInt k = 0; k < n; k++) {   /* rows p, q */
                    double spk = S[p + (size_t)k * n], sqk = S[q + (size_t)k * n];
                    S[p + (size_t)k * n] = c * spk - s * sqk;
                    S[q + (size_t)k * n] = s * spk + c * sqk;
                }
                for (PetscInt k = 0; k < n; k++) {
                    double qkp = Q[k + (size_t)p * n], qkq = Q[k + (size_t)q * n];
                    Q[k + (size_t)p * n] = c * qkp - s * qkq;
                    Q[k + (size_t)q * n] = s * qkp + c * qkq;
                }
            }
    }
    std::vector<PetscInt> ord((size_t)n);
    for (PetscInt i = 0; i < n; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](PetscInt x, PetscInt y) { return S[x + (size_t)x * n] < S[y + (size_t)y * n]; });
    for (PetscInt j = 0; j < n; j++) {
        lam[j] = S[ord[j] + (size_t)ord[j] * n];
        if (vec)
            for (PetscInt i = 0; i < n; i++) a[i + (size_t)j * lda] = Q[i + (size_t)ord[j] * n];
    }
}

extern "C" void LAPACKsyev_(const char *jobz, const char *, const PetscBLASInt *n, PetscScalar *a,
                            const PetscBLASInt *lda, PetscReal *w, PetscScalar *work, const PetscBLASInt *lwork,
                            PetscBLASInt *info)
{
    *info = 0;
    if (*lwork == -1) { work[0] = (PetscScalar)std::max(1, 3 * *n - 1); return; }
    jacobi_eig(*n, a, *lda, w, *jobz == 'V' || *jobz == 'v');
}

/* ------------------------------------------------------------------------- */
/* SLEPc MFN + FNSQRT                                                         */
/* ------------------------------------------------------------------------- */
PetscErrorCode FNCreate(MPI_Comm, FN *fn) { *fn = new _p_FN(); return 0; }
PetscErrorCode FNSetType(FN fn, FNType t) { fn->sqrt = !std::strcmp(t, FNSQRT); return fn->sqrt ? 0 : PETSC_ERR_SUP; }
PetscErrorCode MFNCreate(MPI_Comm, MFN *mfn) { *mfn = new _p_MFN(); return 0; }
PetscErrorCode MFNSetFN(MFN mfn, FN fn) { mfn->fn = fn; return 0; }
PetscErrorCode MFNSetFromOptions(MFN) { return 0; }
PetscErrorCode MFNSetOperator(MFN mfn, Mat A) { mfn->A = A; return 0; }
PetscErrorCode MFNGetConvergedReason(MFN mfn, MFNConvergedReason *r) { *r = mfn->reason; return 0; }

/* symmetric tridiagonal eigenproblem by implicit QL with Wilkinson shifts (Golub & Van Loan,
 * sec. 8.3): d (diagonal, n) and e (sub-diagonal, n-1; e[n-1] scratch) in, d = eigenvalues and
 * Z (n x n, row-major, Z[i*n + c] = component i of eigenvector c) out */
static void tql(std::vector<double> &d, std::vector<double> &e, std::vector<double> &Z, int n)
{
    Z.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) Z[(size_t)i * n + i] = 1.0;
    e.resize((size_t)n + 1, 0.0);
    for (int l = 0; l < n; l++) {
        for (int iter = 0; iter < 60; iter++) {
            int m;
            for (m = l; m < n - 1; m++) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= 1e-16 * dd) break;
            }
            if (m == l) break;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
            double s = 1, c = 1, p = 0;
            int i;
            bool early = false;
            for (i = m - 1; i >= l; i--) {
                double f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) { d[i + 1] -= p; e[m] = 0.0; early = true; break; }
                s = f / r; c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; k++) {
                    double fz = Z[(size_t)k * n + i + 1];
                    Z[(size_t)k * n + i + 1] = s * Z[(size_t)k * n + i] + c * fz;
                    Z[(size_t)k * n + i] = c * Z[(size_t)k * n + i] - s * fz;
                }
            }
            if (early) continue;
            d[l] -= p; e[l] = g; e[m] = 0.0;
        }
    }
}

PetscErrorCode MFNSolve(MFN mfn, Vec b, Vec x)
{
    Mat A = mfn->A;
    const PetscInt n = b->n;
    std::vector<PetscScalar> in = b->a;
    PetscReal b0 = std::sqrt(dotv(in, in));
    std::vector<PetscScalar> out((size_t)n, 0.0);
    mfn->reason = 1;
    if (b0 > 0) {
        /* Lanczos with full reorthogonalisation; every 5 vectors (and at the end) the estimate
         * b0 Q_m sqrt(T_m) e1 is formed and the run stops when it changed by <= 1e-13
         * relative, or at once if T_m has a negative eigenvalue (no real square root) */
        const PetscInt kmax = std::min<PetscInt>(n, 300);
        std::vector<std::vector<PetscScalar>> Q;
        std::vector<PetscReal> al, be, gprev;
        Q.push_back(in);
        for (auto &e : Q[0]) e /= b0;
        Vec v, w;
        VecCreateSeq(PETSC_COMM_SELF, n, &v);
        VecCreateSeq(PETSC_COMM_SELF, n, &w);
        std::vector<PetscReal> g;
        bool neg = false;
        for (PetscInt j = 0; j < kmax; j++) {
            v->a = Q[j];
            PetscErrorCode ierr = MatMult(A, v, w);
            if (ierr) return ierr;
            if (j > 0) for (PetscInt i = 0; i < n; i++) w->a[i] -= be[j - 1] * Q[j - 1][i];
            PetscReal aj = dotv(Q[j], w->a);
            al.push_back(aj);
            for (PetscInt i = 0; i < n; i++) w->a[i] -= aj * Q[j][i];
            for (int pass = 0; pass < 2; pass++)
                for (PetscInt l = 0; l <= j; l++) {
                    PetscReal h = dotv(Q[l], w->a);
                    for (PetscInt i = 0; i < n; i++) w->a[i] -= h * Q[l][i];
                }
            PetscReal bj = std::sqrt(dotv(w->a, w->a));
            const bool last = bj <= 1e-14 * b0 || j == kmax - 1;
            if ((j + 1) % 5 == 0 || last) {
                const int m = (int)j + 1;
                std::vector<double> d(al.begin(), al.end()), e(be.begin(), be.end()), Z;
                e.resize((size_t)m, 0.0);
                tql(d, e, Z, m);
                neg = false;
                g.assign((size_t)m, 0.0);
                for (int c = 0; c < m; c++) {
                    if (d[c] < 0) { neg = true; continue; }
                    const double wc = std::sqrt(d[c]) * Z[c];   /* sqrt(theta_c) U[0,c] */
                    for (int i = 0; i < m; i++) g[i] += Z[(size_t)i * m + c] * wc;
                }
                for (auto &gi : g) gi *= b0;
                bool conv = false;
                if (!gprev.empty()) {
                    PetscReal dn = 0, gn = 0;
                    for (int i = 0; i < m; i++) {
                        PetscReal gp = i < (int)gprev.size() ? gprev[i] : 0.0;
                        dn += (g[i] - gp) * (g[i] - gp);
                        gn += g[i] * g[i];
                    }
                    conv = dn <= 1e-26 * gn;
                }
                gprev = g;
                if (neg || conv || last) break;
            }
            be.push_back(bj);
            Q.push_back(w->a);
            for (auto &e : Q.back()) e /= bj;
        }
        for (size_t l = 0; l < g.size(); l++)
            for (PetscInt i = 0; i < n; i++) out[i] += g[l] * Q[l][i];
        VecDestroy(&v);
        VecDestroy(&w);
        if (neg) mfn->reason = -1;
    }
    x->a = out;
    if (FILE *f = dump_file()) {
        dump_header(f, 'F', n, mfn->reason, 0);
        std::fwrite(in.data(), sizeof(PetscScalar), (size_t)n, f);
        std::fwrite(out.data(), sizeof(PetscScalar), (size_t)n, f);
        std::fflush(f);
    }
    return 0;
}
