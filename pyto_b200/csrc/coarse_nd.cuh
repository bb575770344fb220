// Internal interface of the nested-dissection coarse solver (coarse_nd.cu) for the
// deflated PCG drivers (deflation.cu).
#pragma once
#include "krylov.cuh"

namespace pyto {
// device block-sparse coarse matrix of a bound plan (64-bit fixed point while assembled)
double* nd_matrix(const pyto_coarse_nd* P);
long long nd_matrix_bytes(const pyto_coarse_nd* P);
// conversion, diagonal shift and numeric factorisation (stream-ordered, capturable)
int nd_factor(const pyto_coarse_nd* P, const int32_t* nptr, const int32_t* nlist, const int* gexp, double shift,
              int relative, cudaStream_t st);
// mu = E^-1 v; kernels return at once when S is given and S->done is set
int nd_solve(const pyto_coarse_nd* P, const double* v, double* mu, const KrylovState* S, cudaStream_t st);
}  // namespace pyto
