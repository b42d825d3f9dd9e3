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


def tables(instances, need, first=0, count=-1, stride=1):
    """The (d, prime) tables of an uneven batch, restated from the reference's driver rule: per d,
    prime i serves the instances of that d with i < need, and its table is built to their largest n
    (fast/cuckoo_fast.cu:787-795, 859-866).  need(n, M, d) gives the primes an instance needs.
    Returns {(d, i): [instance indices]} for the planned prime indices first + j stride."""
    out = {}
    needs = [need(n, M, d) for n, M, d in instances]
    top = max(needs) if count < 0 else min(first + count, max(needs))
    for d in sorted({x[2] for x in instances}):
        ks = [k for k, x in enumerate(instances) if x[2] == d]
        for i in range(first, top, stride):
            act = [k for k in ks if i < needs[k]]
            if act:
                out[(d, i)] = act
    return out


def run(engine, instances, model=0, bits=50, first=0, count=-1, stride=1, stream_ptr=None):
    """Residues of every instance through one uneven-batch graph: [array over the instance's primes]
    (entries of prime indices left out of a sampled plan stay zero)."""
    with engine.uneven(instances, model, bits, first, count, stride) as u:
        u.launch(stream_ptr)
        return u.results(stream_ptr)


def per_instance(engine, instances, prime_range, need, model=0, first=0, count=-1, stride=1):
    """The plain form: every instance alone, one table per prime at its own n (one cf_residues call,
    a launch per chunk of primes, per instance), over the same planned prime indices."""
    out = []
    for n, M, d in instances:
        k = need(n, M, d)
        top = k if count < 0 else min(first + count, k)
        idx = list(range(first, top, stride))
        res = [0] * k
        if idx:
            ps = prime_range(0, top)
            r = engine.residues([ps[i] for i in idx], n, d, [(n, M)], model=model)
            for i, v in zip(idx, r[:, 0]):
                res[i] = int(v)
        out.append(res)
    return out
