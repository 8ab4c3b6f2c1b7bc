// Dense n x n matrix, row-major: the data contract of the reference's
// Matrix<S> (Structures/Matrix.h:32-57) — same members (mat, nov, sparsity),
// deep-copying copy constructor, stealing move constructor, deleted
// assignments, destructor that frees mat.
#pragma once

#include <cstring>
#include <utility>

template <class S>
class Matrix {
public:
    Matrix() : mat(nullptr), nov(0), sparsity(0.0) {}

    explicit Matrix(int n) : mat(new S[(size_t)n * n]()), nov(n), sparsity(0.0) {}

    Matrix(const Matrix& other) : mat(new S[(size_t)other.nov * other.nov]), nov(other.nov),
                                  sparsity(other.sparsity)
    {
        std::copy(other.mat, other.mat + (size_t)nov * nov, mat);
    }

    Matrix(Matrix&& other) noexcept : mat(other.mat), nov(other.nov), sparsity(other.sparsity)
    {
        other.mat = nullptr;
    }

    Matrix& operator=(const Matrix&) = delete;
    Matrix& operator=(Matrix&&) = delete;

    virtual ~Matrix() { delete[] mat; }

    S* mat;          // row-major nov x nov entries
    int nov;         // number of rows (= columns)
    double sparsity; // percentage of nonzero entries
};
