#!/usr/bin/env python3
"""Uneven batches: many (n, M, d) instances, each modulo its own need(n, M, d) primes.

The reference runs one instance set per process and per d, with one table size per batch of
primes: the largest n among the queries that still need the batch's first prime
(fast/cuckoo_fast.cu:787-795).  Instances of one d share their tables: prime i's table is built
to the largest n among the instances with i < need, and every such instance is answered from it.

This module holds the seeded instance generator of the uneven-batch workload (512 instances, n
log-uniform in [256, 16384], M = n U{2, 3, 4}, d uniform in {2, 3, 4}).
"""
import math

import numpy as np

CONFIG4_SEED = 20261204


def instances(count=512, seed=CONFIG4_SEED, n_lo=256, n_hi=16384, m_mult=(2, 3, 4), d_choices=(2, 3, 4)):
    """Seeded instances [(n, M, d)]: n = round(exp(U[ln n_lo, ln n_hi])), M = n * choice(m_mult),
    d = choice(d_choices), drawn in that order per instance (so a prefix of a longer list is the
    same as a shorter list from the same seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        M = n * int(rng.choice(m_mult))
        d = int(rng.choice(d_choices))
        out.append((n, M, d))
    return out
