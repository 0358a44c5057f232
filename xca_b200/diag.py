"""Diagram topologies: connected pairings of the 2m vertices of an order-m backbone.

Interface of ``python/triqs_xca/diag.py:62-71`` (``all_pairings``, ``all_connected_pairings``):
each topology is ``(sign, pairs)`` with ``pairs`` a list of m vertex pairs ``(a, b)``, ``a < b``,
listed by increasing first vertex, and ``sign`` the signature of the vertex permutation
``(a_0, b_0, a_1, b_1, ...)``.  A pairing is connected when every hybridization line can be reached
from the line(s) attached to vertex 0 through a chain of crossing lines.  The enumeration order is
lexicographic in the pair list, which is the order the reference produces.
"""


def _perm_sign(seq):
    inv = 0
    for i in range(len(seq)):
        for j in range(i + 1, len(seq)):
            if seq[i] > seq[j]:
                inv += 1
    return -1 if inv % 2 else 1


def _matchings(free):
    if not free:
        yield []
        return
    a = free[0]
    for k in range(1, len(free)):
        rest = free[1:k] + free[k + 1:]
        for tail in _matchings(rest):
            yield [(a, free[k])] + tail


def _crosses(p, q):
    return p[0] < q[0] < p[1] < q[1] or q[0] < p[0] < q[1] < p[1]


def is_connected(pairs):
    seen = [i for i, p in enumerate(pairs) if p[0] == 0]
    frontier = list(seen)
    while frontier:
        i = frontier.pop()
        for j, q in enumerate(pairs):
            if j not in seen and _crosses(pairs[i], q):
                seen.append(j)
                frontier.append(j)
    return len(seen) == len(pairs)


def all_pairings(order):
    for pairs in _matchings(list(range(2 * order))):
        yield _perm_sign([v for p in pairs for v in p]), pairs


def all_connected_pairings(order):
    for sign, pairs in all_pairings(order):
        if is_connected(pairs):
            yield sign, pairs
