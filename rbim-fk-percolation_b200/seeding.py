"""Chain keys of many ``SeedSequence`` children at once.

A scan seeds task k with child k of a ``SeedSequence`` (reference
``simulation.py:367-368, 384-393``), and the engine keys a chain with the
child's ``generate_state(2, uint32)`` (:func:`engine.chain_key`).  Spawning a
few thousand children one by one costs tens of milliseconds of Python per
scan.  Children of one parent differ only in the last word of their entropy
(their spawn index), so the same hash runs here over all of them at once as
numpy array arithmetic.

The hash is numpy's ``SeedSequence`` (after M. E. O'Neill's ``seed_seq_fe``),
restated:

* the entropy words are the parent's entropy as little-endian 32-bit words,
  zero-padded to the pool size when a spawn key follows, then the words of
  the spawn key;
* mixing: every word passes through ``hashmix`` (xor with a running constant,
  the constant times ``MULT_A``, multiply, xor-shift by 16); the first
  ``pool_size`` words fill the pool, each pool word is mixed into every other
  one, then each remaining entropy word is mixed into every pool word, with
  ``mix(x, y) = (MIX_L * x - MIX_R * y) ^ >> 16``;
* ``generate_state`` runs the pool words through the same kind of hash with
  its own constants.

All arithmetic is modulo 2**32.  ``tests/test_host.py`` checks the keys
against numpy's own ``spawn`` + ``generate_state`` for many parents.
"""

from __future__ import annotations

from typing import List

import numpy as np

__all__ = ["child_keys"]

_INIT_A = 0x43B0D7E5
_MULT_A = 0x931E8875
_INIT_B = 0x8B51F9DD
_MULT_B = 0x58F38DED
_MIX_L = 0xCA01F9DD
_MIX_R = 0x4973F715
_M32 = 0xFFFFFFFF


def _words(v: int) -> List[int]:
    """Little-endian 32-bit words of a non-negative int (0 -> [0])."""
    v = int(v)
    if v < 0:
        raise ValueError("negative entropy")
    if v == 0:
        return [0]
    out = []
    while v:
        out.append(v & _M32)
        v >>= 32
    return out


def _entropy_words(entropy) -> List[int]:
    if entropy is None:
        raise ValueError("no entropy")
    if isinstance(entropy, (int, np.integer)):
        return _words(int(entropy))
    out: List[int] = []
    for v in entropy:
        out += _words(int(v))
    return out


class _Hash:
    """Running constant of one hash pass."""

    def __init__(self, init: int, mult: int):
        self.c = init
        self.mult = mult

    def __call__(self, value: np.ndarray) -> np.ndarray:
        v = np.asarray(value, dtype=np.uint32) ^ np.uint32(self.c)
        self.c = (self.c * self.mult) & _M32
        v = v * np.uint32(self.c)
        return v ^ (v >> np.uint32(16))


def _mix(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    r = np.uint32(_MIX_L) * x - np.uint32(_MIX_R) * y
    return r ^ (r >> np.uint32(16))


def child_keys(parent: np.random.SeedSequence, n: int) -> np.ndarray:
    """``chain_key`` of the parent's next ``n`` children, as ``parent.spawn(n)`` would make them.

    Unlike ``spawn``, the parent is left as it was (numpy keeps its spawn
    counter read-only).  Children this vectorised form does not cover (a spawn
    index of 2**32 or more) go through numpy's ``spawn``.
    """
    from .engine import chain_key

    n = int(n)
    start = int(parent.n_children_spawned)
    if n <= 0:
        return np.zeros(0, dtype=np.uint64)
    if start + n > 1 << 32:
        return np.array([chain_key(c) for c in parent.spawn(n)], dtype=np.uint64)
    pool_size = int(parent.pool_size)
    run = _entropy_words(parent.entropy)
    if len(run) < pool_size:
        run = run + [0] * (pool_size - len(run))
    prefix = [w for v in parent.spawn_key for w in _words(v)]
    with np.errstate(over="ignore"):
        idx = np.arange(start, start + n, dtype=np.uint64).astype(np.uint32)
        entropy = [np.full(n, w, dtype=np.uint32) for w in run + prefix] + [idx]
        h = _Hash(_INIT_A, _MULT_A)
        pool = [h(entropy[i]) if i < len(entropy) else h(np.zeros(n, np.uint32)) for i in range(pool_size)]
        for i_src in range(pool_size):
            for i_dst in range(pool_size):
                if i_src != i_dst:
                    pool[i_dst] = _mix(pool[i_dst], h(pool[i_src]))
        for i_src in range(pool_size, len(entropy)):
            for i_dst in range(pool_size):
                pool[i_dst] = _mix(pool[i_dst], h(entropy[i_src]))
        g = _Hash(_INIT_B, _MULT_B)
        w0 = g(pool[0 % pool_size])
        w1 = g(pool[1 % pool_size])
    return w0.astype(np.uint64) | (w1.astype(np.uint64) << np.uint64(32))
