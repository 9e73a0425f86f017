// Project-written minimal stand-ins for the parts of MPI and PETSc that the
// reference's Jacobian assembly touches (form_petsc_jacobian.hpp,
// petsc_interface.hpp), single process only: a Mat is an ordered map of
// (row, col) -> value with ADD/INSERT semantics. Test infrastructure only.
#pragma once
#include <cstddef>
#include <map>
#include <utility>
#include <vector>

typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscErrorCode;
typedef int PetscMPIInt;
#define PETSC_COMM_WORLD 0
#define PETSC_DETERMINE (-1)
#define PETSC_DECIDE (-1)
typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES } InsertMode;

struct _p_Mat {
  PetscInt m = 0, n = 0;
  std::map<std::pair<PetscInt, PetscInt>, double> v;
  // preallocated block storage (set by the timing harness): entry (i, j) goes
  // to block (i / bs, j / bs) of a block-row pattern, found by a scan of the
  // row's few blocks, like MatSetValues into a preallocated PETSc BAIJ matrix
  double* bsr_vals = nullptr;
  const int* bsr_rowptr = nullptr;
  const int* bsr_colidx = nullptr;
  int bs = 0;
};
typedef _p_Mat* Mat;
struct _p_Vec {
  std::vector<double> a;
};
typedef _p_Vec* Vec;

#define PetscCallAbort(comm, expr) do { (void)(comm); (void)(expr); } while (0)
#define PetscCall(expr) do { (void)(expr); } while (0)

inline PetscErrorCode MatCreate(MPI_Comm, Mat* A) { *A = new _p_Mat{}; return 0; }
inline PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt, PetscInt) { A->m = m; A->n = n; return 0; }
inline PetscErrorCode MatDestroy(Mat* A) { delete *A; *A = nullptr; return 0; }
inline PetscErrorCode MatGetOwnershipRange(Mat, PetscInt* b, PetscInt* e) { *b = 0; *e = 0; return 0; }
inline PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt* im, PetscInt n, const PetscInt* in,
                                   const PetscScalar* vals, InsertMode mode) {
  if (A->bsr_vals) {
    const int bs = A->bs;
    for (PetscInt i = 0; i < m; ++i) {
      const int ib = im[i] / bs, ir = im[i] % bs;
      for (PetscInt j = 0; j < n; ++j) {
        const int jb = in[j] / bs;
        int k = A->bsr_rowptr[ib];
        while (k < A->bsr_rowptr[ib + 1] && A->bsr_colidx[k] != jb) ++k;
        if (k == A->bsr_rowptr[ib + 1]) continue;  // outside the preallocated pattern
        double& dst = A->bsr_vals[((std::size_t)k * bs + ir) * bs + in[j] % bs];
        if (mode == ADD_VALUES) dst += vals[i * n + j];
        else dst = vals[i * n + j];
      }
    }
    return 0;
  }
  for (PetscInt i = 0; i < m; ++i)
    for (PetscInt j = 0; j < n; ++j) {
      auto key = std::make_pair(im[i], in[j]);
      if (mode == ADD_VALUES) A->v[key] += vals[i * n + j];
      else A->v[key] = vals[i * n + j];
    }
  return 0;
}
inline PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode) {
  return MatSetValues(A, 1, &i, 1, &j, &v, mode);
}
inline PetscErrorCode VecGetArray(Vec x, PetscScalar** a) { *a = x->a.data(); return 0; }
inline PetscErrorCode VecRestoreArray(Vec, PetscScalar**) { return 0; }
inline PetscErrorCode VecGetLocalSize(Vec x, PetscInt* n) { *n = (PetscInt)x->a.size(); return 0; }

/// dense row-major copy of a shim matrix (n x n, n = declared local size)
inline void petsc_shim_to_dense(Mat A, double* out) {
  std::size_t n = (std::size_t)A->m;
  for (std::size_t i = 0; i < n * (std::size_t)A->n; ++i) out[i] = 0.0;
  for (auto& kv : A->v) out[(std::size_t)kv.first.first * A->n + kv.first.second] = kv.second;
}
