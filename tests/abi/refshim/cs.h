/* Declarations of the CXSparse names that the reference's headers use
 * (common_defs.hpp, sparse_interface.hpp, arpack_interface.hpp), for the
 * compile check of include/chainamps_b200_shim.hpp against those headers.
 * Declarations only: nothing here is linked or run.  The compressed/triplet
 * sparse matrix structure is CXSparse's public interface (Davis, Direct
 * Methods for Sparse Linear Systems, SIAM 2006): nzmax, m, n, column
 * pointers (or column indices), row indices, values, nz (-1 for CSC). */
#ifndef CHAINAMPS_B200_TEST_CS_H
#define CHAINAMPS_B200_TEST_CS_H
#include <complex>
#include <cstdint>
typedef int64_t SuiteSparse_long;
typedef struct cs_cl_sparse {
  SuiteSparse_long nzmax;
  SuiteSparse_long m;
  SuiteSparse_long n;
  SuiteSparse_long *p;
  SuiteSparse_long *i;
  std::complex<double> *x;
  SuiteSparse_long nz;
} cs_cl;
SuiteSparse_long cs_cl_dropzeros(cs_cl *A);
#endif
