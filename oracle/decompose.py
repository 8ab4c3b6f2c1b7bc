"""TEST INFRASTRUCTURE ONLY — the checker, never the product.

Exact permanent of sparse matrices, restating in exact rational arithmetic
the structural steps the reference applies before its sparse Ryser:
  * perfect-matching pruning (IO/dm.cpp:441-501) and connected components
    (IO/dm.h:43-107): perm = product over components;
  * the folds of CommonFiles/DecomposePerman.h: a line with one nonzero
    (:201-291), a line with two nonzeros merged into one combined line
    (:294-431), and a line with three or four nonzeros split into two
    matrices that each fold one pair (:434-557);
  * pieces of n <= DIRECT_MAX go to the exact CRT permanent (oracle.py).
Unlike the reference, which folds in floating point and stops at n = 30,
every step here is exact, so the result is the exact permanent of the input.
"""
from __future__ import annotations

from fractions import Fraction

import oracle as O

DIRECT_MAX = 24


def _prune(a):
    """Keep entries on some perfect matching (None if there is none)."""
    n = len(a)
    adj = [[j for j in range(n) if a[i][j] != 0] for i in range(n)]
    row_of = [-1] * n

    def augment(r, seen):
        for c in adj[r]:
            if c in seen:
                continue
            seen.add(c)
            if row_of[c] < 0 or augment(row_of[c], seen):
                row_of[c] = r
                return True
        return False

    for r in range(n):
        if not augment(r, set()):
            return None
    # SCCs of rows with arcs r -> row_of[c] for entries (r, c)
    graph = [[row_of[c] for c in adj[r]] for r in range(n)]
    index, low, on, stack, comp = {}, {}, set(), [], [-1] * n
    counter = [0, 0]

    def strong(v):
        index[v] = low[v] = counter[0]
        counter[0] += 1
        stack.append(v)
        on.add(v)
        for w in graph[v]:
            if w not in index:
                strong(w)
                low[v] = min(low[v], low[w])
            elif w in on:
                low[v] = min(low[v], index[w])
        if low[v] == index[v]:
            while True:
                w = stack.pop()
                on.discard(w)
                comp[w] = counter[1]
                if w == v:
                    break
            counter[1] += 1

    for v in range(n):
        if v not in index:
            strong(v)
    return [[a[i][j] if a[i][j] != 0 and comp[i] == comp[row_of[j]] else Fraction(0) for j in range(n)]
            for i in range(n)]


def _components(a):
    n = len(a)
    seen = [False] * (2 * n)
    out = []
    for s in range(2 * n):
        if seen[s]:
            continue
        rows, cols, todo = [], [], [s]
        seen[s] = True
        while todo:
            v = todo.pop()
            if v < n:
                rows.append(v)
                nb = [n + c for c in range(n) if a[v][c] != 0]
            else:
                cols.append(v - n)
                nb = [r for r in range(n) if a[r][v - n] != 0]
            for w in nb:
                if not seen[w]:
                    seen[w] = True
                    todo.append(w)
        out.append((sorted(rows), sorted(cols)))
    return out


def _fold_pair(a, r, c1, c2):
    """Row r restricted to columns c1, c2: drop row r and column c2, column c1
    becomes a[r][c2]*A[:,c1] + a[r][c1]*A[:,c2]."""
    n = len(a)
    out = []
    for i in range(n):
        if i == r:
            continue
        row = []
        for j in range(n):
            if j == c2:
                continue
            row.append(a[i][c1] * a[r][c2] + a[i][c2] * a[r][c1] if j == c1 else a[i][j])
        out.append(row)
    return out


def _perm(a):
    n = len(a)
    if n == 0:
        return Fraction(1)
    if n <= DIRECT_MAX:
        return O.exact_perm_fractions(a)
    p = _prune(a)
    if p is None:
        return Fraction(0)
    comps = _components(p)
    if len(comps) > 1:
        total = Fraction(1)
        for rows, cols in comps:
            if len(rows) != len(cols):
                return Fraction(0)
            total *= _perm([[p[i][j] for j in cols] for i in rows])
        return total
    # one component: fold along the sparsest line (rows, or columns via transpose)
    degs = [(sum(1 for v in p[i] if v != 0), 0, i) for i in range(n)]
    degs += [(sum(1 for i in range(n) if p[i][j] != 0), 1, j) for j in range(n)]
    d, is_col, k = min(degs)
    m = [list(r) for r in zip(*p)] if is_col else p
    nz = [j for j in range(n) if m[k][j] != 0]
    if d == 0:
        return Fraction(0)
    if d == 1:
        j = nz[0]
        return m[k][j] * _perm([[m[i][c] for c in range(n) if c != j] for i in range(n) if i != k])
    # pair the nonzeros; an odd one out is paired with a zero column
    if len(nz) % 2:
        nz.append(next(j for j in range(n) if m[k][j] == 0))
    return sum((_perm(_fold_pair(m, k, nz[t], nz[t + 1])) for t in range(0, len(nz), 2)), Fraction(0))


def exact_perm_sparse(a) -> Fraction:
    """Exact permanent of a float (or Fraction) matrix via exact folds."""
    return _perm([[Fraction(v) for v in row] for row in a])
