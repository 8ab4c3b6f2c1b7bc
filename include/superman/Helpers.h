// Structural helpers on dense matrices (degree counts, rank deficiency) and
// the scaling record — the reference's CommonFiles/Helpers.h:120-204.  The
// reference's file-mailbox IPC and progress bar (Helpers.h:40-116, 219-242)
// belong to its two-process launcher and are not part of this layer.
#pragma once

#include "Matrix.h"

struct ScalingCompact {
    ScalingCompact() : rowScale(nullptr), colScale(nullptr) {}
    ~ScalingCompact()
    {
        delete[] rowScale;
        delete[] colScale;
    }
    ScalingCompact(const ScalingCompact&) = delete;
    ScalingCompact& operator=(const ScalingCompact&) = delete;
    double* rowScale;
    double* colScale;
};

template <class S>
inline int getRowNNZ(const Matrix<S>* m, int row)
{
    int c = 0;
    for (int j = 0; j < m->nov; ++j) c += m->mat[(size_t)row * m->nov + j] != S(0);
    return c;
}

template <class S>
inline int getColNNZ(const Matrix<S>* m, int col)
{
    int c = 0;
    for (int i = 0; i < m->nov; ++i) c += m->mat[(size_t)i * m->nov + col] != S(0);
    return c;
}

template <class S>
inline int getNNZ(const Matrix<S>* m)
{
    int c = 0;
    for (size_t i = 0; i < (size_t)m->nov * m->nov; ++i) c += m->mat[i] != S(0);
    return c;
}

// Smallest row or column degree.
template <class S>
inline int getMinDegree(const Matrix<S>* m)
{
    int best = m->nov;
    for (int i = 0; i < m->nov; ++i) {
        int r = getRowNNZ(m, i), c = getColNNZ(m, i);
        if (r < best) best = r;
        if (c < best) best = c;
    }
    return best;
}

// True when some row or column is empty (the permanent is then 0).
template <class S>
inline bool isRankDeficient(const Matrix<S>* m)
{
    for (int i = 0; i < m->nov; ++i)
        if (getRowNNZ(m, i) == 0 || getColNNZ(m, i) == 0) return true;
    return false;
}
