"""Approximate minimum degree (AMD) fill-reducing ordering.

Written from the published algorithm: P. R. Amestoy, T. A. Davis and I. S.
Duff, "An Approximate Minimum Degree Ordering Algorithm", SIAM J. Matrix Anal.
Appl. 17(4), 1996, and T. A. Davis, "Direct Methods for Sparse Linear
Systems", SIAM 2006, ch. 7.  The reference obtains its permutation from the
third-party ``qdldl`` Python package (QDLDL + SuiteSparse AMD, not vendored in
the reference; called at ``warpmpc/jax_qdldl/core.py:276-278``).  That package
is not available, so this ordering is this project's own implementation of the
same published method; the permutation itself is therefore not pinned to the
package's output, while every symbolic step downstream of a given permutation
is (see ``planning.py``).  ``build_qdldl_plan`` accepts an explicit
permutation so a known permutation can always be supplied.

Elements of the method implemented here:

* quotient graph: variables carry variable adjacency ``A_i`` and element
  adjacency ``E_i``; eliminating pivot ``p`` creates element ``L_p`` and
  absorbs the elements adjacent to ``p``;
* approximate external degree
  ``d_i = min(n - k, d_i + |L_p \\ i|, |A_i \\ i| + |L_p \\ i| + sum_e |L_e \\ L_p|)``;
* aggressive element absorption (``|L_e \\ L_p| = 0``);
* supervariable detection by hashing ``(A_i, E_i)`` and mass elimination;
* dense-row postponement (rows with degree above ``max(16, 10 sqrt(n))``);
* a final postorder of the assembly tree so that each subtree is contiguous.

Ties in the minimum degree are broken by the most recently (re)inserted
variable, as in a degree-bucket implementation with head insertion.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp


def _symmetric_adjacency(a_upper: sp.spmatrix) -> list[set[int]]:
    a = sp.csc_matrix(a_upper)
    n = a.shape[0]
    coo = a.tocoo()
    rows = np.concatenate([coo.row, coo.col])
    cols = np.concatenate([coo.col, coo.row])
    keep = rows != cols
    pattern = sp.csr_matrix(
        (np.ones(int(np.count_nonzero(keep)), dtype=np.int8), (rows[keep], cols[keep])),
        shape=(n, n),
    )
    pattern.sum_duplicates()
    return [set(pattern.indices[pattern.indptr[i] : pattern.indptr[i + 1]].tolist()) for i in range(n)]


class _DegreeBuckets:
    """Degree lists with head insertion (most recent first)."""

    def __init__(self, n: int):
        self.buckets: list[list[int]] = [[] for _ in range(n + 1)]
        self.where = np.full(n, -1, dtype=np.int64)
        self.min_deg = 0

    def insert(self, i: int, deg: int) -> None:
        self.buckets[deg].append(i)
        self.where[i] = deg
        if deg < self.min_deg:
            self.min_deg = deg

    def remove(self, i: int) -> None:
        deg = int(self.where[i])
        if deg >= 0:
            bucket = self.buckets[deg]
            # buckets are small for sparse problems; linear removal is fine
            for pos in range(len(bucket) - 1, -1, -1):
                if bucket[pos] == i:
                    bucket.pop(pos)
                    break
            self.where[i] = -1

    def pop_min(self) -> int:
        while not self.buckets[self.min_deg]:
            self.min_deg += 1
        i = self.buckets[self.min_deg].pop()
        self.where[i] = -1
        return i


def amd_order(a_upper: sp.spmatrix, dense_factor: float = 10.0) -> np.ndarray:
    """Return an AMD permutation ``p`` (new index -> old index) as int32."""

    a = sp.csc_matrix(a_upper)
    n = a.shape[0]
    if a.shape[0] != a.shape[1]:
        raise ValueError("AMD ordering needs a square matrix")
    if n == 0:
        return np.zeros(0, dtype=np.int32)

    adj_var = _symmetric_adjacency(a)
    adj_elem: list[set[int]] = [set() for _ in range(n)]
    elem_vars: dict[int, set[int]] = {}
    nv = np.ones(n, dtype=np.int64)          # supervariable weight (0 = merged/absorbed)
    members: list[list[int]] = [[i] for i in range(n)]
    degree = np.array([len(s) for s in adj_var], dtype=np.int64)
    alive = np.ones(n, dtype=bool)           # variable not yet eliminated
    elim_parent = np.full(n, -1, dtype=np.int64)  # assembly tree (element -> absorbing element)

    dense_threshold = max(16, int(dense_factor * math.sqrt(n)))
    dense = [i for i in range(n) if degree[i] > dense_threshold] if n > 16 else []
    dense_set = set(dense)
    for i in dense:
        alive[i] = False
        nv[i] = 0
        for j in adj_var[i]:
            adj_var[j].discard(i)
        adj_var[i] = set()
    for i in range(n):
        if alive[i]:
            degree[i] = len(adj_var[i])

    buckets = _DegreeBuckets(n)
    for i in range(n):
        if alive[i]:
            buckets.insert(i, int(degree[i]))

    elimination: list[int] = []  # pivots in order (supervariable representatives)
    k = 0
    n_live = n - len(dense)
    while k < n_live:
        p = buckets.pop_min()
        # element L_p: union of variable neighbours and neighbour elements' variables
        lp: set[int] = set(v for v in adj_var[p] if nv[v] > 0)
        for e in adj_elem[p]:
            lp |= elem_vars[e]
            elim_parent[e] = p
            del elem_vars[e]
        lp.discard(p)
        lp = {v for v in lp if nv[v] > 0 and alive[v]}
        absorbed = set(adj_elem[p])
        alive[p] = False
        elimination.append(p)
        k += int(nv[p])
        adj_var[p] = set()
        adj_elem[p] = set()
        elem_vars[p] = lp

        # update adjacency of the variables in L_p
        for i in lp:
            buckets.remove(i)
            adj_elem[i] -= absorbed
            adj_elem[i].add(p)
            adj_var[i] -= lp
            adj_var[i].discard(p)

        # |L_e \ L_p| for elements adjacent to L_p
        w: dict[int, int] = {}
        for i in lp:
            for e in adj_elem[i]:
                if e == p:
                    continue
                if e not in w:
                    w[e] = int(sum(nv[v] for v in elem_vars[e]))
                w[e] -= int(nv[i])
        # aggressive absorption
        for e, we in list(w.items()):
            if we <= 0:
                for i in elem_vars[e]:
                    adj_elem[i].discard(e)
                elim_parent[e] = p
                del elem_vars[e]
                del w[e]

        lp_weight = int(sum(nv[v] for v in lp))
        # approximate degrees
        for i in lp:
            ext = lp_weight - int(nv[i])
            da = int(sum(nv[v] for v in adj_var[i] if nv[v] > 0))
            de = 0
            for e in adj_elem[i]:
                if e != p:
                    de += w.get(e, int(sum(nv[v] for v in elem_vars[e])))
            d_new = min(int(degree[i]) + ext, da + ext + de, n_live - k - int(nv[i]))
            degree[i] = max(d_new, 0)

        # supervariable detection among L_p
        hashes: dict[tuple, list[int]] = {}
        for i in sorted(lp):
            key = (frozenset(adj_var[i]), frozenset(adj_elem[i]))
            hashes.setdefault(key, []).append(i)
        for group in hashes.values():
            if len(group) < 2:
                continue
            rep = group[0]
            for j in group[1:]:
                nv[rep] += nv[j]
                nv[j] = 0
                alive[j] = False
                members[rep].extend(members[j])
                members[j] = []
                for v in adj_var[j]:
                    adj_var[v].discard(j)
                for e in adj_elem[j]:
                    if e in elem_vars:
                        elem_vars[e].discard(j)
                adj_var[j] = set()
                adj_elem[j] = set()
                elim_parent[j] = rep

        # mass elimination: variables whose only neighbour is element p
        for i in sorted(lp):
            if nv[i] > 0 and alive[i] and not adj_var[i] and adj_elem[i] == {p}:
                alive[i] = False
                elimination.append(i)
                k += int(nv[i])
                elem_vars[p].discard(i)
                elim_parent[i] = p
                adj_elem[i] = set()
        for i in elem_vars[p]:
            if alive[i] and nv[i] > 0:
                buckets.insert(i, int(min(degree[i], n)))

    order: list[int] = []
    for piv in elimination:
        order.extend(members[piv])
    order.extend(dense)
    perm = np.asarray(order, dtype=np.int64)
    if perm.size != n or np.unique(perm).size != n:
        raise AssertionError("AMD produced an invalid permutation")
    return _postorder_permutation(a, perm).astype(np.int32)


def _postorder_permutation(a: sp.csc_matrix, perm: np.ndarray) -> np.ndarray:
    """Reorder ``perm`` by a postorder of the elimination tree of ``P A P^T``.

    Postordering keeps the fill of the factor unchanged and makes every
    subtree of the elimination tree a contiguous range of columns.
    """

    n = perm.size
    pinv = np.empty(n, dtype=np.int64)
    pinv[perm] = np.arange(n)
    coo = sp.triu(a, format="coo")
    r = pinv[coo.row]
    c = pinv[coo.col]
    rows = np.minimum(r, c)
    cols = np.maximum(r, c)
    pa = sp.csc_matrix((np.ones(rows.size), (rows, cols)), shape=(n, n))
    pa.sum_duplicates()
    parent = np.full(n, -1, dtype=np.int64)
    ancestor = np.full(n, -1, dtype=np.int64)
    for j in range(n):
        for ptr in range(pa.indptr[j], pa.indptr[j + 1]):
            i = int(pa.indices[ptr])
            while i != -1 and i < j:
                nxt = int(ancestor[i])
                ancestor[i] = j
                if nxt == -1:
                    parent[i] = j
                    break
                i = nxt
    children: list[list[int]] = [[] for _ in range(n)]
    roots: list[int] = []
    for j in range(n):
        if parent[j] >= 0:
            children[int(parent[j])].append(j)
        else:
            roots.append(j)
    post: list[int] = []
    for root in roots:
        stack = [(root, 0)]
        while stack:
            node, idx = stack.pop()
            if idx < len(children[node]):
                stack.append((node, idx + 1))
                stack.append((children[node][idx], 0))
            else:
                post.append(node)
    return perm[np.asarray(post, dtype=np.int64)]
