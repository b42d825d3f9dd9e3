// Uneven batches (host side): many instances (n_k, M_k, d_k), each modulo its own need(n_k, M_k,
// d_k) primes of the fixed list, turned into a list of (d, prime) tables for one work-queue launch.
//
// The reference computes one instance set per run and per d; within a run one table per prime
// serves every query that still needs the prime, and a batch of primes takes its table size from
// the largest n that still needs the batch's first prime (fast/cuckoo_fast.cu:787-795, 859-866).
// Here the rule is applied per prime: table (d, i) is built to the largest n among the instances of
// degree d with i < need, and answers each of them.  The tables are grouped by transform length
// (one persistent launch per length) and ordered heaviest first inside a group.
#pragma once
#include <algorithm>
#include <cstdint>
#include <map>
#include <vector>

#include "host_common.hpp"

namespace cfh {

struct UnevenTable {
    int d, lg, n, F, J;  // degree, log2 transform length, table size, factorial range, queries
    long i;              // prime index in the fixed list
    u64 prime;
    long q0;             // its queries are [q0, q0 + J) of the plan's query arrays
};

struct UnevenPlan {
    std::vector<long> need, off;  // per instance: primes needed, first output index
    long outputs = 0;             // sum of the needs
    std::vector<UnevenTable> tables;        // ordered: transform length descending, then n, J
    std::vector<int> qn, qM;                // per table query lists, concatenated
    std::vector<long long> qout;            // output index of each query: off[k] + i
};

// Instances k < K; prime indices first + j * stride (j >= 0) below first + count are planned, the
// others left out (count < 0: every prime any instance needs).  jcap > 0 splits a table whose
// instances exceed jcap queries into several tables of at most jcap queries.  Returns false on
// invalid instances (the rules of cf_residues: 1 <= n < M, d <= M for the subset model).
inline bool plan_uneven(const int* n, const int* M, const int* d, int K, int model, int bits, long first, long count,
                        long stride, int jcap, UnevenPlan& pl) {
    pl = UnevenPlan();
    if (K < 0 || first < 0 || stride < 1 || (model != 0 && model != 1)) return false;
    long maxneed = 0;
    for (int k = 0; k < K; ++k) {
        if (n[k] < 1 || M[k] <= n[k] || d[k] < 1 || (model == 0 && d[k] > M[k])) return false;
        pl.need.push_back(need(n[k], M[k], d[k], model, bits));
        pl.off.push_back(pl.outputs);
        pl.outputs += pl.need.back();
        maxneed = std::max(maxneed, pl.need.back());
    }
    const long stop = count < 0 ? maxneed : std::min(first + count, maxneed);
    if (stop <= first) return true;
    const std::vector<u64> primes = prime_range(0, stop, bits);
    if ((long)primes.size() < stop) return false;
    std::map<int, std::vector<int>> byd;  // instances by degree, in instance order
    for (int k = 0; k < K; ++k) byd[d[k]].push_back(k);
    struct Pending {
        UnevenTable t;
        std::vector<int> ks;
    };
    std::vector<Pending> pend;
    for (const auto& kv : byd) {
        const int dd = kv.first;
        for (long i = first; i < stop; i += stride) {
            std::vector<int> act;
            for (int k : kv.second)
                if (i < pl.need[k]) act.push_back(k);
            if (act.empty()) continue;
            for (size_t a = 0; a < act.size(); a += (size_t)(jcap > 0 ? jcap : act.size())) {
                const size_t b = std::min(act.size(), a + (size_t)(jcap > 0 ? jcap : act.size()));
                Pending p;
                p.ks.assign(act.begin() + a, act.begin() + b);
                int nm = 0, F = 0;
                for (int k : p.ks) nm = std::max(nm, n[k]), F = std::max(F, M[k]);
                F = std::max(F, nm);
                if (model == 0) F = std::max(F, dd);
                const u64 L = transform_length((u64)nm);
                int lg = 0;
                while ((1ull << lg) < L) ++lg;
                p.t = UnevenTable{dd, lg, nm, F, (int)p.ks.size(), i, primes[i], 0};
                pend.push_back(p);
            }
        }
    }
    // heaviest first: transform length, then table size, then queries; ties in (d, i) order
    std::stable_sort(pend.begin(), pend.end(), [](const Pending& a, const Pending& b) {
        if (a.t.lg != b.t.lg) return a.t.lg > b.t.lg;
        if (a.t.n != b.t.n) return a.t.n > b.t.n;
        return a.t.J > b.t.J;
    });
    for (Pending& p : pend) {
        p.t.q0 = (long)pl.qn.size();
        for (int k : p.ks) {
            pl.qn.push_back(n[k]);
            pl.qM.push_back(M[k]);
            pl.qout.push_back((long long)(pl.off[k] + p.t.i));
        }
        pl.tables.push_back(p.t);
    }
    return true;
}

}  // namespace cfh
