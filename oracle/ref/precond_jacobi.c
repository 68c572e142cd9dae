/*
 * Link-time wrap of the Jacobi build of the reference (frehd_ref_jacobi; test
 * infrastructure, see oracle/ref/Makefile).  solveMatrix (nsfunctions.c:1016)
 * hands SSORPrecond to laspack's CGIter; with `ld --wrap=SSORPrecond` the same
 * call receives laspack's own JacobiPrecond (precond.c:26-46) instead, which is
 * the preconditioner of the device solve.  Nothing else changes: same matrix,
 * same CGIter, same x = 0 start and stopping rule.
 */
#include "laspack/precond.h"

Vector *__wrap_SSORPrecond(QMatrix *A, Vector *y, Vector *c, double Omega) {
  return JacobiPrecond(A, y, c, Omega);
}
