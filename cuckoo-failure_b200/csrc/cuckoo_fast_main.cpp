// cuckoo_fast_b200: the host driver of the reference's batch engine (fast/cuckoo_fast.cu:648-904)
// with the GPU behind the C ABI of include/cuckoo_b200.h.  Same command line, same resume rules,
// same output lines, so fast/post_gmp.py (or this package's crt.py, which needs no gmpy2) combines the residues as before.
//
//   cuckoo_fast_b200 D QUERIES FIRST COUNT [--batch B] [--out FILE] [--device N] [--replacement] [--prime-bits 62]
//
// QUERIES: lines "n M".  Prime number i is the i-th largest prime p < 2^50 with 2^20 | p - 1.  A
// query is evaluated for prime i only if i < need(n, M).  Output lines: "i p n M residue".  With
// --out the file is appended to and primes already complete in it are skipped.
// --replacement selects the model with d independent draws (Q = M^d, the library's
// OneTableModel::replacement); the reference's fast engine has only the d-subset model.
// --prime-bits 62 uses the prime list below 2^62 and need() over 61 bits, the output of the
// reference built with -DFP_RB=64 (fast/cuckoo_fast.cu:48-57); combine with --pbits 61.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "../../include/cuckoo_b200.h"
#include "host_common.hpp"

struct Query {
    int n, M;
    long need;
};

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: cuckoo_fast_b200 D QUERIES FIRST COUNT [--batch B] [--out FILE] [--device N] [--replacement] [--prime-bits 62]\n");
        return 2;
    }
    const int d = std::atoi(argv[1]);
    const long first = std::atol(argv[3]), count = std::atol(argv[4]);
    long batch = 0;
    int device = 0, model = CF_MODEL_SUBSET, bits = cfh::PRIME_BITS;
    const char* out_path = nullptr;
    for (int i = 5; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--batch") && i + 1 < argc) batch = std::atol(argv[++i]);
        else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) out_path = argv[++i];
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--replacement")) model = CF_MODEL_REPLACEMENT;
        else if (!std::strcmp(argv[i], "--prime-bits") && i + 1 < argc) {
            bits = std::atoi(argv[++i]);
            if (bits != 50 && bits != 62) {
                std::fprintf(stderr, "--prime-bits takes 50 or 62\n");
                return 2;
            }
        }
        else {
            std::fprintf(stderr, "unknown option %s\n", argv[i]);
            return 2;
        }
    }
    std::vector<Query> qs;
    int nmax = 0, Mmax = 0;
    long maxneed = 0;
    {
        FILE* f = std::fopen(argv[2], "r");
        if (!f) {
            std::fprintf(stderr, "cannot open %s\n", argv[2]);
            return 2;
        }
        int n, M;
        while (std::fscanf(f, "%d %d", &n, &M) == 2) {
            if (n < 1 || M <= n || d < 1 || (model == CF_MODEL_SUBSET && d > M)) {
                std::fprintf(stderr, "bad query %d %d\n", n, M);
                std::fclose(f);
                return 2;
            }
            qs.push_back({n, M, cf_need_bits(n, M, d, model, bits)});
            nmax = std::max(nmax, n);
            Mmax = std::max(Mmax, M);
            maxneed = std::max(maxneed, qs.back().need);
        }
        std::fclose(f);
    }
    if (qs.empty() || nmax < 8 || nmax + 1 > (1 << cfh::TWO_ADIC)) {
        std::fprintf(stderr, "need queries with 8 <= max n < 2^%d\n", cfh::TWO_ADIC);
        return 2;
    }
    if (cf_transform_length((uint64_t)nmax) > 65536) {
        std::fprintf(stderr, "this build handles tables up to n = 65536 (got %d)\n", nmax);
        return 2;
    }

    // primes already finished in the output file (fast/cuckoo_fast.cu:697-720)
    std::set<long> done;
    FILE* out = stdout;
    if (out_path) {
        if (FILE* f = std::fopen(out_path, "r")) {
            std::vector<long> cnt(first + count > 0 ? first + count : 1, 0);
            long i;
            unsigned long long p, r;
            int n, M;
            while (std::fscanf(f, "%ld %llu %d %d %llu", &i, &p, &n, &M, &r) == 5)
                if (i >= 0 && i < (long)cnt.size()) ++cnt[i];
            std::fclose(f);
            for (long i2 = first; i2 < first + count; ++i2) {
                long want = 0;
                for (const Query& q : qs) want += i2 < q.need;
                if (want > 0 && cnt[i2] == want) done.insert(i2);
            }
        }
        out = std::fopen(out_path, "a");
        if (!out) {
            std::fprintf(stderr, "cannot append to %s\n", out_path);
            return 2;
        }
    }
    std::vector<long> todo;
    for (long i = first; i < first + count && i < maxneed; ++i)
        if (!done.count(i)) todo.push_back(i);
    if (todo.empty()) {
        std::fprintf(stderr, "nothing to do (%zu primes already in the output)\n", done.size());
        return 0;
    }
    const std::vector<uint64_t> primes = cfh::prime_range(first, count, bits);  // primes[i - first]
    if (primes.empty() || primes.back() < (1ull << (bits - 1))) {
        std::fprintf(stderr, "prime list exhausted above 2^%d\n", bits - 1);
        return 4;
    }

    cf_engine* eng = nullptr;
    if (cf_engine_create(device, &eng) != CF_OK) {
        std::fprintf(stderr, "cannot open CUDA device %d\n", device);
        return 1;
    }
    const uint64_t per_prime = cf_workspace_bytes(nmax, Mmax, (int)qs.size());
    if (batch <= 0) {  // what fits, rounded down to whole waves of the primes the GPU runs at once
        batch = cf_max_batch(eng, nmax, Mmax, (int)qs.size());
        const long wave = cf_resident_primes(eng, nmax, Mmax, (int)qs.size());
        if (wave > 0 && batch > wave) batch -= batch % wave;
    }
    if (batch < 1) {
        std::fprintf(stderr, "not enough device memory: %.2f GB per prime\n", per_prime / 1073741824.0);
        cf_engine_destroy(eng);
        return 3;
    }
    const size_t B = (size_t)std::min<long>(batch, (long)todo.size());
    std::fprintf(stderr, "[cuda-b200] %d-bit primes, d=%d, %s, nmax=%d, L=%llu, %.3f GB per prime, batch %zu, %zu primes to do\n",
                 bits, d, model == CF_MODEL_SUBSET ? "d-subset" : "replacement", nmax,
                 (unsigned long long)cf_transform_length((uint64_t)nmax), per_prime / 1073741824.0, B, todo.size());

    const auto t0 = std::chrono::steady_clock::now();
    auto secs = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    std::vector<uint64_t> bp, res;
    for (size_t at = 0; at < todo.size(); at += B) {
        const size_t nb = std::min(B, todo.size() - at);
        int nm = 0;  // largest n that still needs any prime of this batch (fast/cuckoo_fast.cu:789-792)
        std::vector<size_t> act;
        std::vector<int> qn, qM;
        for (size_t j = 0; j < qs.size(); ++j)
            if (todo[at] < qs[j].need) {
                act.push_back(j);
                qn.push_back(qs[j].n);
                qM.push_back(qs[j].M);
                nm = std::max(nm, qs[j].n);
            }
        bp.resize(nb);
        for (size_t b = 0; b < nb; ++b) bp[b] = primes[todo[at + b] - first];
        res.assign(nb * act.size(), 0);
        const int rc = cf_residues(eng, bp.data(), (int)nb, nm, d, model, qn.data(), qM.data(), (int)act.size(), res.data());
        if (rc != CF_OK) {
            std::fprintf(stderr, "engine error %d: %s\n", rc, cf_engine_last_error(eng));
            cf_engine_destroy(eng);
            return rc == CF_ERR_NOMEM ? 3 : 1;
        }
        for (size_t b = 0; b < nb; ++b) {
            const long i = todo[at + b];
            for (size_t jj = 0; jj < act.size(); ++jj) {
                const Query& q = qs[act[jj]];
                if (i >= q.need) continue;
                std::fprintf(out, "%ld %llu %d %d %llu\n", i, (unsigned long long)bp[b], q.n, q.M,
                             (unsigned long long)res[b * act.size() + jj]);
            }
        }
        std::fflush(out);
        std::fprintf(stderr, "primes %ld..%ld (n<=%d): done at %.1f s\n", todo[at], todo[at + nb - 1], nm, secs());
    }
    if (out != stdout) std::fclose(out);
    cf_engine_destroy(eng);
    return 0;
}
