// Structural decomposition wrapped around every permanent driver — the
// reference's DecomposePerman<C,S,Permanent> (CommonFiles/DecomposePerman.h:
// 76-557), same rules:
//  * while n > 30: fold a row/column with one nonzero (the permanent is that
//    entry times the minor's, the entry moved into the minor's first row) or
//    with two nonzeros (the two columns, or rows, merge into one weighted
//    combination); stop on an empty row/column (permanent 0);
//  * then, while n > 30 and the smallest degree is below 5: fold degree 1/2
//    again, or split a degree-3/4 line into two matrices whose permanents add;
//  * every remaining piece (n <= 63) is copied into a driver, computed and
//    summed; optional Sinkhorn scaling is undone per piece.
// Result.time is the wall time of the whole decomposition and computation.
#pragma once

#include <chrono>
#include <memory>
#include <stdexcept>
#include <vector>

#include "Helpers.h"
#include "IO.h"
#include "Matrix.h"
#include "Result.h"
#include "Settings.h"

// Pieces computed by the decompositions on this thread (the reference keeps
// these counters in process globals, main.cpp:36-40).
struct DecomposeStats {
    int pieces = 0;
    double sumN = 0;
    double sumNNZ = 0;
};
inline thread_local DecomposeStats g_decomposeStats;

template <class C, class S, class Driver>
class DecomposePerman {
public:
    DecomposePerman(Matrix<S>* matrix, Settings settings) : m_Matrix(matrix), m_Settings(settings) {}
    DecomposePerman(const DecomposePerman&) = delete;
    DecomposePerman& operator=(const DecomposePerman&) = delete;

    Result computePermanentRecursively()
    {
        const auto t0 = std::chrono::steady_clock::now();
        startRecursion(m_Matrix);
        double overall = 0;
        for (size_t p = 0; p < m_Drivers.size(); ++p) {
            Driver* d = m_Drivers[p].get();
            g_decomposeStats.pieces += 1;
            g_decomposeStats.sumN += d->m_Matrix->nov;
            g_decomposeStats.sumNNZ += getNNZ(d->m_Matrix);
            double r = d->computePermanent();
            if (m_Settings.scaling) {
                const ScalingCompact* sc = m_Scaling[p].get();
                for (int i = 0; i < d->m_Matrix->nov; ++i) r = r / sc->rowScale[i] / sc->colScale[i];
            }
            overall += r;
        }
        m_Drivers.clear();
        m_Scaling.clear();
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return Result(t, overall);
    }

    // Pieces the decomposition would compute, without computing them.
    std::vector<Matrix<S>*> pieces()
    {
        startRecursion(m_Matrix);
        std::vector<Matrix<S>*> out;
        for (auto& d : m_Drivers) out.push_back(new Matrix<S>(*d->m_Matrix));
        m_Drivers.clear();
        m_Scaling.clear();
        return out;
    }

private:
    static constexpr int kFoldAbove = 30;  // decompose only while n > 30

    void startRecursion(Matrix<S>* m)
    {
        // The approximation samples the whole matrix as one piece
        // (CommonFiles/DecomposePerman.h:122-126).
        if (m_Settings.algorithm == APPROXIMATION) {
            enqueue(m);
            return;
        }
        bool folded = true;
        while (folded && m->nov > kFoldAbove) {
            folded = fold1(m) || fold2(m);
            if (isRankDeficient(m)) return;
        }
        recurse(m);
    }

    void recurse(Matrix<S>* m)
    {
        const int d = getMinDegree(m);
        if (m->nov > kFoldAbove && d < 5) {
            if (d == 1) {
                fold1(m);
                recurse(m);
            } else if (d == 2) {
                fold2(m);
                recurse(m);
            } else if (d == 3 || d == 4) {
                Matrix<S> other;
                split34(m, &other, d);
                recurse(m);
                recurse(&other);
            }
            // d == 0: an empty line, the piece contributes nothing
            return;
        }
        enqueue(m);
    }

    void enqueue(Matrix<S>* m)
    {
        m->sparsity = m->nov ? 100.0 * getNNZ(m) / ((double)m->nov * m->nov) : 0.0;
        if (m->nov > 63 && m_Settings.algorithm != APPROXIMATION)
            throw std::runtime_error("Permanent is an #P-complete problem. The size of the matrix you want to calculate the permanent for exceeds the limit of what is computationally possible. Try approximation algorithms.\n");
        std::unique_ptr<ScalingCompact> sc;
        if (m_Settings.scaling) {
            sc.reset(new ScalingCompact);
            IO::scale<C, S>(m, m_Settings, sc.get());
        }
        m_Drivers.emplace_back(new Driver(new Matrix<S>(*m), m_Settings));
        m_Scaling.emplace_back(std::move(sc));
    }

    // First line (scanning row i, then column i, for i = 0, 1, ...) with
    // exactly `deg` nonzeros; *isRow tells which.  -1 if none.
    static int findLine(const Matrix<S>* m, int deg, bool* isRow)
    {
        for (int i = 0; i < m->nov; ++i) {
            if (getRowNNZ(m, i) == deg) { *isRow = true; return i; }
            if (getColNNZ(m, i) == deg) { *isRow = false; return i; }
        }
        return -1;
    }

    static S at(const Matrix<S>* m, int r, int c) { return m->mat[(size_t)r * m->nov + c]; }

    // Copy of m without row `dr` and column `dc`.
    static std::vector<S> minor(const Matrix<S>* m, int dr, int dc)
    {
        const int n = m->nov;
        std::vector<S> out;
        out.reserve((size_t)(n - 1) * (n - 1));
        for (int r = 0; r < n; ++r)
            if (r != dr)
                for (int c = 0; c < n; ++c)
                    if (c != dc) out.push_back(at(m, r, c));
        return out;
    }

    static void assign(Matrix<S>* m, const std::vector<S>& v, int n)
    {
        // keep the existing allocation (it is large enough), as the reference does
        std::copy(v.begin(), v.end(), m->mat);
        m->nov = n;
    }

    // Degree-1 fold: perm(A) = a * perm(minor); a multiplies the minor's first row.
    static bool fold1(Matrix<S>* m)
    {
        bool isRow = false;
        const int line = findLine(m, 1, &isRow);
        if (line < 0) return false;
        const int n = m->nov;
        int r = line, c = line;
        for (int k = 0; k < n; ++k) {
            if (isRow && at(m, line, k) != S(0)) { c = k; break; }
            if (!isRow && at(m, k, line) != S(0)) { r = k; break; }
        }
        const S v = at(m, r, c);
        std::vector<S> mm = minor(m, r, c);
        for (int k = 0; k < n - 1; ++k) mm[k] *= v;
        assign(m, mm, n - 1);
        return true;
    }

    // Degree-2 fold of row r with nonzeros at columns c1 < c2: drop row r and
    // column c2, replace column c1 by a_{r,c2}*A[:,c1] + a_{r,c1}*A[:,c2]
    // (transposed for a column).
    static bool fold2(Matrix<S>* m)
    {
        bool isRow = false;
        const int line = findLine(m, 2, &isRow);
        if (line < 0) return false;
        const int n = m->nov;
        int k1 = -1, k2 = -1;
        for (int k = 0; k < n; ++k) {
            const S v = isRow ? at(m, line, k) : at(m, k, line);
            if (v != S(0)) {
                if (k1 < 0) k1 = k;
                else { k2 = k; break; }
            }
        }
        std::vector<S> out;
        out.reserve((size_t)(n - 1) * (n - 1));
        for (int r = 0; r < n; ++r) {
            if (isRow ? r == line : r == k2) continue;
            for (int c = 0; c < n; ++c) {
                if (isRow ? c == k2 : c == line) continue;
                S v = at(m, r, c);
                if (isRow && c == k1) v = at(m, r, k1) * at(m, line, k2) + at(m, r, k2) * at(m, line, k1);
                if (!isRow && r == k1) v = at(m, k1, c) * at(m, k2, line) + at(m, k2, c) * at(m, k1, line);
                out.push_back(v);
            }
        }
        assign(m, out, n - 1);
        return true;
    }

    // Degree-3/4 split: the line's nonzeros c0..c3 (c3 = a zero position for
    // degree 3) pair up as {c0,c1} and {c2,c3}; m keeps the fold of the first
    // pair, other receives the fold of the second.  perm(A) = perm(m) +
    // perm(other).  A low-degree column is handled on the transpose.
    static void split34(Matrix<S>* m, Matrix<S>* other, int deg)
    {
        bool isRow = false;
        const int line = findLine(m, deg, &isRow);
        if (line < 0) return;
        const int n = m->nov;
        std::vector<S> t((size_t)n * n);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) t[(size_t)r * n + c] = isRow ? at(m, r, c) : at(m, c, r);
        auto T = [&](int r, int c) { return t[(size_t)r * n + c]; };
        int nz[4] = {-1, -1, -1, -1}, cnt = 0, zero = -1;
        for (int c = 0; c < n; ++c) {
            if (T(line, c) != S(0)) { if (cnt < 4) nz[cnt++] = c; }
            else zero = c;
        }
        if (nz[3] < 0) nz[3] = zero;
        std::vector<S> a, b;
        a.reserve((size_t)(n - 1) * (n - 1));
        b.reserve((size_t)(n - 1) * (n - 1));
        for (int r = 0; r < n; ++r) {
            if (r == line) continue;
            for (int c = 0; c < n; ++c) {
                if (c != nz[1])
                    a.push_back(c == nz[0] ? T(line, nz[0]) * T(r, nz[1]) + T(line, nz[1]) * T(r, nz[0]) : T(r, c));
                if (c != nz[3])
                    b.push_back(c == nz[2] ? T(line, nz[2]) * T(r, nz[3]) + T(line, nz[3]) * T(r, nz[2]) : T(r, c));
            }
        }
        assign(m, a, n - 1);
        delete[] other->mat;
        other->mat = new S[(size_t)(n - 1) * (n - 1)];
        assign(other, b, n - 1);
    }

    Matrix<S>* m_Matrix;
    Settings m_Settings;
    std::vector<std::unique_ptr<Driver>> m_Drivers;
    std::vector<std::unique_ptr<ScalingCompact>> m_Scaling;
};
