"""Spanning-forest winding oracle (test infrastructure only).

Restates the reference's independent wrapping check, ``brute_force_winding``
in ``tests/test_wrapping.py:22-64``: give every site an unwrapped position by
breadth-first search over the active bonds, then every non-tree active bond
closes one fundamental cycle, and the cycle winds along an axis iff its
summed displacement along that axis is nonzero.  It shares no code with the
union-find oracle or the CUDA engine.
"""

from __future__ import annotations

from collections import deque

import numpy as np

__all__ = ["spanning_forest_winding"]


def spanning_forest_winding(active: np.ndarray, L: int):
    """``(wraps_x, wraps_y)`` of the active-bond graph on the ``L x L`` torus."""
    n_sites = L * L
    active = np.asarray(active, dtype=bool).reshape(-1)
    nbrs = [[] for _ in range(n_sites)]
    bonds = []
    for k in np.flatnonzero(active):
        k = int(k)
        a = k >> 1
        x, y = divmod(a, L)
        if k & 1:
            b, dx, dy = x * L + (y + 1) % L, 0, 1
        else:
            b, dx, dy = ((x + 1) % L) * L + y, 1, 0
        bonds.append((k, a, b, dx, dy))
        nbrs[a].append((b, dx, dy, k))
        nbrs[b].append((a, -dx, -dy, k))
    pos = [None] * n_sites
    tree = set()
    for start in range(n_sites):
        if pos[start] is not None:
            continue
        pos[start] = (0, 0)
        q = deque([start])
        while q:
            u = q.popleft()
            ux, uy = pos[u]
            for v, dx, dy, k in nbrs[u]:
                if pos[v] is None:
                    pos[v] = (ux + dx, uy + dy)
                    tree.add(k)
                    q.append(v)
    wx = wy = False
    for k, a, b, dx, dy in bonds:
        if k in tree:
            continue
        if pos[a][0] + dx - pos[b][0] != 0:
            wx = True
        if pos[a][1] + dy - pos[b][1] != 0:
            wy = True
    return wx, wy
