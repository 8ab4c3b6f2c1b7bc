// Structural preprocessing of the reference (IO/dm.h:43-107, IO/dm.cpp:441-501):
//  * findCCs: connected components of the bipartite row/column graph; the
//    permanent of the matrix is the product of the components' permanents,
//    and is zero when a component has unequal row and column counts.
//  * dm_prune: Dulmage-Mendelsohn fine decomposition — keeps exactly the
//    entries that lie on some perfect matching (an entry (i,j) does iff row i
//    and the row matched to column j are in the same strongly connected
//    component of the alternating graph), which leaves the permanent
//    unchanged and can split the matrix into more components.
#pragma once

#include <queue>
#include <vector>

#include "Matrix.h"

// Prunes the row-major pattern given as CSR (rptrs[n+1], cols[nnz]) in place:
// on return rptrs/cols hold only entries on some perfect matching.  Returns
// false (and empties the pattern) when no perfect matching exists, i.e. the
// permanent is structurally zero.  Implemented in superman_b200/csrc/dm.cpp.
bool dm_prune(std::vector<int>& rptrs, std::vector<int>& cols, int n);

template <class S>
inline void findCCs(const Matrix<S>* matrix, std::vector<std::vector<unsigned>>& rowComponents,
                    std::vector<std::vector<unsigned>>& colComponents, unsigned& biggestComponentSize)
{
    const unsigned n = (unsigned)matrix->nov;
    biggestComponentSize = 0;
    std::vector<char> seen(2 * (size_t)n, 0);
    for (unsigned start = 0; start < 2 * n; ++start) {
        if (seen[start]) continue;
        std::vector<unsigned> rv, cv;
        std::queue<unsigned> q;
        seen[start] = 1;
        q.push(start);
        while (!q.empty()) {
            const unsigned v = q.front();
            q.pop();
            if (v < n) {  // row vertex: neighbours are its nonzero columns
                rv.push_back(v);
                for (unsigned c = 0; c < n; ++c)
                    if (matrix->mat[(size_t)v * n + c] != S(0) && !seen[n + c]) { seen[n + c] = 1; q.push(n + c); }
            } else {      // column vertex: neighbours are its nonzero rows
                const unsigned c = v - n;
                cv.push_back(c);
                for (unsigned r = 0; r < n; ++r)
                    if (matrix->mat[(size_t)r * n + c] != S(0) && !seen[r]) { seen[r] = 1; q.push(r); }
            }
        }
        if (rv.size() == cv.size() && rv.size() > biggestComponentSize) biggestComponentSize = (unsigned)rv.size();
        rowComponents.emplace_back(std::move(rv));
        colComponents.emplace_back(std::move(cv));
    }
}
