// Dulmage-Mendelsohn fine pruning of a square sparsity pattern (the role of
// the reference's dm(), IO/dm.cpp:441-501, called from IO/IO.h:477-508).
//
// An entry (i, j) lies on some perfect matching iff, for a fixed perfect
// matching M, row i and the row M matches to column j belong to the same
// strongly connected component of the "alternating" digraph on rows with an
// arc i -> rowOf[j] for every entry (i, j).  Entries on no perfect matching
// contribute nothing to the permanent, so removing them leaves it unchanged
// and exposes a finer block structure for findCCs.
#include <vector>

#include "dm.h"

namespace {

// Maximum bipartite matching by augmenting paths (iterative DFS);
// returns the size, fills rowOf[col] = matched row or -1.
int max_matching(const std::vector<int>& rptrs, const std::vector<int>& cols, int n, std::vector<int>& rowOf)
{
    rowOf.assign(n, -1);
    std::vector<int> colOf(n, -1), stamp(n, -1), next(n), parentCol(n);
    int size = 0;
    // cheap greedy start
    for (int r = 0; r < n; ++r)
        for (int p = rptrs[r]; p < rptrs[r + 1]; ++p)
            if (rowOf[cols[p]] < 0) {
                rowOf[cols[p]] = r;
                colOf[r] = cols[p];
                ++size;
                break;
            }
    std::vector<int> stack;
    for (int root = 0; root < n; ++root) {
        if (colOf[root] >= 0) continue;
        // DFS over rows; stack of rows, next[] = next edge to try
        stack.assign(1, root);
        next[root] = rptrs[root];
        stamp[root] = root;
        int freeCol = -1;
        while (!stack.empty() && freeCol < 0) {
            const int r = stack.back();
            if (next[r] >= rptrs[r + 1]) {
                stack.pop_back();
                continue;
            }
            const int c = cols[next[r]++];
            const int r2 = rowOf[c];
            if (r2 < 0) {
                freeCol = c;
                parentCol[r] = c;
            } else if (stamp[r2] != root) {
                stamp[r2] = root;
                parentCol[r] = c;
                next[r2] = rptrs[r2];
                stack.push_back(r2);
            }
        }
        if (freeCol < 0) continue;
        // augment along the stack: each row takes the column it came through
        for (int k = (int)stack.size() - 1; k >= 0; --k) {
            const int r = stack[k];
            const int c = parentCol[r];
            rowOf[c] = r;
            colOf[r] = c;
        }
        ++size;
    }
    return size;
}

// Tarjan's strongly connected components, iterative.
std::vector<int> scc(const std::vector<int>& rptrs, const std::vector<int>& cols, const std::vector<int>& rowOf, int n)
{
    std::vector<int> index(n, -1), low(n, 0), comp(n, -1), edge(n), st;
    std::vector<char> on(n, 0);
    std::vector<int> call;
    int counter = 0, ncomp = 0;
    for (int s = 0; s < n; ++s) {
        if (index[s] >= 0) continue;
        call.push_back(s);
        index[s] = low[s] = counter++;
        edge[s] = rptrs[s];
        st.push_back(s);
        on[s] = 1;
        while (!call.empty()) {
            const int v = call.back();
            if (edge[v] < rptrs[v + 1]) {
                const int w = rowOf[cols[edge[v]++]];
                if (index[w] < 0) {
                    index[w] = low[w] = counter++;
                    edge[w] = rptrs[w];
                    st.push_back(w);
                    on[w] = 1;
                    call.push_back(w);
                } else if (on[w] && index[w] < low[v]) {
                    low[v] = index[w];
                }
                continue;
            }
            call.pop_back();
            if (!call.empty() && low[v] < low[call.back()]) low[call.back()] = low[v];
            if (low[v] == index[v]) {
                int w;
                do {
                    w = st.back();
                    st.pop_back();
                    on[w] = 0;
                    comp[w] = ncomp;
                } while (w != v);
                ++ncomp;
            }
        }
    }
    return comp;
}

}  // namespace

bool dm_prune(std::vector<int>& rptrs, std::vector<int>& cols, int n)
{
    std::vector<int> rowOf;
    if (max_matching(rptrs, cols, n, rowOf) != n) {
        rptrs.assign(n + 1, 0);  // no perfect matching: structurally zero permanent
        cols.clear();
        return false;
    }
    const std::vector<int> comp = scc(rptrs, cols, rowOf, n);
    std::vector<int> nr(n + 1, 0), nc;
    nc.reserve(cols.size());
    for (int r = 0; r < n; ++r) {
        for (int p = rptrs[r]; p < rptrs[r + 1]; ++p)
            if (comp[r] == comp[rowOf[cols[p]]]) nc.push_back(cols[p]);
        nr[r + 1] = (int)nc.size();
    }
    rptrs.swap(nr);
    cols.swap(nc);
    return true;
}
