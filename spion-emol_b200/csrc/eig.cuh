// eig.cuh -- batched symmetric eigenvalues (see eig.cu).
#pragma once

#include "common.cuh"

namespace scatt {

struct EigEntry {
    double* M;      // n x n (ld), lower triangle read, destroyed
    int n, ld;
    double* d;      // n
    double* e;      // n
    double* work;   // 2n
    double* out;    // eigenvalues, ascending (nwant of them)
};

// nwant > 0: the nwant smallest eigenvalues; nwant <= 0: all.
int sym_eigvals_batched(const EigEntry* entries_dev, int count, int nmax, int nwant,
                        cudaStream_t stream);

}  // namespace scatt
