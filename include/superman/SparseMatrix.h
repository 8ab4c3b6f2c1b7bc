// Sparse view of a square matrix with both compressed-column (CSC: cptrs,
// rows, cvals) and compressed-row (CSR: rptrs, cols, rvals) arrays, indices
// ascending — the contract of the reference's SparseMatrix<S>
// (Structures/SparseMatrix.h:31-101).  Like the reference, construction takes
// ownership of the given Matrix: its dense storage moves into this object and
// the Matrix object itself is deleted.
#pragma once

#include <vector>

#include "Matrix.h"

template <class S>
class SparseMatrix : public Matrix<S> {
public:
    SparseMatrix(Matrix<S>* matrix, int nnz_) : Matrix<S>(std::move(*matrix)), nnz(nnz_)
    {
        const int n = this->nov;
        const S* m = this->mat;
        cptrs = new int[n + 1];
        rptrs = new int[n + 1];
        rows = new int[nnz > 0 ? nnz : 1];
        cols = new int[nnz > 0 ? nnz : 1];
        cvals = new S[nnz > 0 ? nnz : 1];
        rvals = new S[nnz > 0 ? nnz : 1];
        int rc = 0, cc = 0;
        for (int r = 0; r < n; ++r) {  // rows, columns ascending
            rptrs[r] = rc;
            for (int j = 0; j < n; ++j)
                if (m[(size_t)r * n + j] != S(0)) { cols[rc] = j; rvals[rc] = m[(size_t)r * n + j]; ++rc; }
        }
        rptrs[n] = rc;
        for (int j = 0; j < n; ++j) {
            cptrs[j] = cc;
            for (int r = 0; r < n; ++r)
                if (m[(size_t)r * n + j] != S(0)) { rows[cc] = r; cvals[cc] = m[(size_t)r * n + j]; ++cc; }
        }
        cptrs[n] = cc;
        delete matrix;
    }

    SparseMatrix(const SparseMatrix&) = delete;
    SparseMatrix& operator=(const SparseMatrix&) = delete;
    SparseMatrix(SparseMatrix&&) = delete;
    SparseMatrix& operator=(SparseMatrix&&) = delete;

    ~SparseMatrix() override
    {
        delete[] cptrs;
        delete[] rptrs;
        delete[] rows;
        delete[] cols;
        delete[] cvals;
        delete[] rvals;
    }

    int* cptrs;  // CSC
    int* rows;
    S* cvals;
    int* rptrs;  // CSR
    int* cols;
    S* rvals;
    int nnz;
};
