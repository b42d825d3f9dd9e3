/* C ABI of the B200 engine for the one-table suffix-table path of zcy05331/Cuckoo-Failure.
 *
 * The reference has no FFI: its host driver (fast/cuckoo_fast.cu main) calls a compile-time
 * execution back end (launch / convolve / dev_alloc / to_dev / from_dev, :325-386, :623-646) and
 * launches k_query directly (:867-876).  These entry points replace that seam, one call per batch
 * of primes: everything from the per-prime tables to the residues runs on the GPU.
 *
 * Conventions: every function returns an int status (CF_OK = 0, negative on error) and never
 * exits the process (the reference's cuda_check calls exit(1), :329-334).  The caller owns host
 * buffers, the engine owns device workspace.  Calls on one engine must not overlap.
 * Residues are canonical (0 <= r < p), exactly what the reference prints as its fifth column.
 */
#ifndef CUCKOO_B200_H
#define CUCKOO_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cf_status {
    CF_OK = 0,
    CF_ERR_ARG = -1,         /* invalid argument (sizes, prime not NTT-friendly, query out of range) */
    CF_ERR_CUDA = -2,        /* CUDA runtime error (message in cf_engine_last_error) */
    CF_ERR_NOMEM = -3,       /* not enough device memory for even one prime */
    CF_ERR_UNSUPPORTED = -4, /* transform length beyond what this build handles */
    CF_ERR_DEVICE = -5       /* a device-side check failed (e.g. no root of unity of order L) */
};

/* Sampling models (include/cuckoo/single_table.hpp:16-23). */
enum cf_model { CF_MODEL_SUBSET = 0, CF_MODEL_REPLACEMENT = 1 };

typedef struct cf_engine cf_engine;

/* ---- host helpers with the reference's exact semantics ---- */

/* Primes number first .. first+count-1 of the fixed list (p = c 2^20 + 1 < 2^50, prime, largest
 * first).  Replaces prime_range, fast/cuckoo_fast.cu:403-432.  Returns the number written. */
long cf_prime_range(long first, long count, uint64_t* out);

/* Number of 50-bit primes query (n, M) needs: ceil((n log2 Q + 3) / 49) + 1 in long double.
 * Replaces need / log2_Q, fast/cuckoo_fast.cu:452-459 (CF_MODEL_REPLACEMENT: log2 Q = d log2 M). */
long cf_need(int n, int M, int d, int model);

/* The same two for the list below 2^62 of the reference's -DFP_RB=64 build (PRIME_BITS = 62,
 * fast/cuckoo_fast.cu:48-57): bits = 50 or 62.  cf_residues accepts primes of either list (it
 * selects the kernels for primes below 2^62 when a prime is 2^50 or above). */
long cf_prime_range_bits(long first, long count, int bits, uint64_t* out);
long cf_need_bits(int n, int M, int d, int model, int bits);

/* max(16, next_pow2(nmax)).  Replaces transform_length, fast/cuckoo_fast.cu:460-472. */
uint64_t cf_transform_length(uint64_t nmax);

/* The 32-bit NTT primes the library CLI (`cuckoo_fail single -n n -M M -d d [--replacement]`)
 * reconstructs N_bad from, largest first: replaces ntt_primes and the prime-count loop,
 * include/cuckoo/modint.hpp:183-196 and src/cuckoo_fail.cpp:151-170.  Every one is usable by
 * cf_residues for a table of nmax = n.  Returns how many there are (writing at most `cap`), or
 * -1 on bad arguments. */
long cf_lib_primes(int n, int M, int d, int model, uint64_t* out, long cap);

/* ---- engine ---- */

/* Bind a CUDA device and create the engine's stream.  Replaces the CUDA back end's implicit
 * device setup and the up-front dev_alloc calls, fast/cuckoo_fast.cu:345-358, :759-780. */
int cf_engine_create(int device, cf_engine** out);
void cf_engine_destroy(cf_engine* e);
/* Text of the last error on this engine ("" if none).  Valid until the next call. */
const char* cf_engine_last_error(const cf_engine* e);

/* One batch: for every prime b, build the suffix table V up to nmax for (d, model) and evaluate
 * the J queries (qn[j], qM[j]); residues[b*J + j] = N_bad(qn[j], qM[j]) mod primes[b].
 * Replaces the body of the batch loop, fast/cuckoo_fast.cu:787-901: per-prime tables (:797-839),
 * the step loop (:841-855), k_query (:867-876) and the Horner finish (:877-890).
 * Requirements: 1 <= qn[j] <= nmax <= 65536, qM[j] > qn[j], d <= qM[j] for the subset model, every
 * prime odd, < 2^62, > max(nmax, qM), with transform_length(nmax) dividing p - 1.  Tables up to nmax = 16384 take one CTA per prime; larger ones a thread-block
 * cluster of 4 to 16 CTAs per prime (the reference runs up to nmax < 2^20, :61, :692, with all of
 * a GPU's threads on a batch of primes).
 * Host buffers; returns when the residues are in `residues`. */
int cf_residues(cf_engine* e, const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM,
                int J, uint64_t* residues);

/* Same computation with the primes and residues in device memory, enqueued on `stream`
 * (a cudaStream_t; NULL is the CUDA default stream); returns without waiting.  The primes are
 * not read on the host: they must lie below 2^50 unless cf_engine_set_prime_bits(e, 62). */
int cf_engine_set_prime_bits(cf_engine* e, int bits);
int cf_residues_async(cf_engine* e, const uint64_t* d_primes, int B, int nmax, int d, int model, const int* qn,
                      const int* qM, int J, uint64_t* d_residues, void* stream);

/* Device workspace per prime in bytes for a table of nmax with J queries up to Mmax. */
uint64_t cf_workspace_bytes(int nmax, int Mmax, int J);

/* Largest number of primes one launch can hold in the device's free memory (0 if none). */
long cf_max_batch(cf_engine* e, int nmax, int Mmax, int J);

/* Primes one launch runs at the same time for a table of nmax (J queries up to Mmax): the SMs times
 * the CTAs per SM of the kernel, or for nmax > 16384 the thread-block clusters (one per prime)
 * the device holds at once.  A batch that is a multiple of it runs in whole waves; 0 on error.
 * No counterpart in the reference, whose batch is bounded by memory only (:743-780). */
long cf_resident_primes(cf_engine* e, int nmax, int Mmax, int J);

/* Kernel launches issued by the last cf_residues / cf_residues_async call. */
long cf_last_launches(const cf_engine* e);

/* ---- graph-captured batches (no counterpart in the reference) ----
 * The reference re-issues about 12 launches per step from the host (fast/cuckoo_fast.cu:841-855).
 * Here a batch is already one persistent launch per chunk of primes; a batch graph captures that
 * launch sequence (error-word reset and kernel launches) once as a CUDA graph, so a repeated
 * batch is replayed with a single cudaGraphLaunch and no per-call host work.  The graph owns its
 * own workspace, query table and error word, sized at capture for (B, nmax, d, model, queries):
 * later engine calls do not disturb it.  d_primes[B] and d_residues[B*J] are device buffers bound
 * at capture; their contents may change between launches (new primes, same sizes).  Launches of
 * one graph must not overlap on the GPU: they share its workspace. */
typedef struct cf_batch_graph cf_batch_graph;
int cf_batch_graph_create(cf_engine* e, const uint64_t* d_primes, int B, int nmax, int d, int model, const int* qn,
                          const int* qM, int J, uint64_t* d_residues, cf_batch_graph** out);
/* Enqueue one replay on `stream` (a cudaStream_t; NULL is the CUDA default stream). */
int cf_batch_graph_launch(cf_batch_graph* g, void* stream);
/* Wait for the work on `stream` and report the device-side checks of the graph's last replay:
 * CF_OK, or CF_ERR_DEVICE (e.g. a prime without a root of unity of order L). */
int cf_batch_graph_status(cf_batch_graph* g, void* stream);
/* Kernel launches (persistent-kernel nodes) in one replay. */
long cf_batch_graph_launches(const cf_batch_graph* g);
void cf_batch_graph_destroy(cf_batch_graph* g);

/* ---- geometry autotuning (no counterpart in the reference: it fixes the convolution's block
 * size at compile time, CONV_LG, fast/cuckoo_fast.cu:518) ----
 * The engine compiles a few geometries of the 50-bit kernel per transform length 2^lg: 2^r entries
 * per thread in registers (the register-pass radix), threads per prime = L / 2^r, and the resident
 * CTAs per SM its register budget targets.  cf_tune_variants describes them (the default first) and
 * returns their number; cf_autotune times each on B primes of a table of nmax (one query (nmax,
 * Mmax), d) through cf_residues, checks that all give the same residues, and makes the fastest
 * the engine's choice for that length (rates[i]: primes per second of geometry i, *chosen: the
 * index).  cf_tune_set / cf_tune_get pin or read the choice (e.g. from a cache of earlier runs).
 * Primes below 2^62 always use the default geometry.
 * Transform lengths 2^15 and 2^16 (nmax > 16384) run one prime per thread-block cluster: their
 * variants are the cluster geometries compiled (threads = CTA size, 2^log2_entries entries each,
 * one CTA per SM; the cluster size is L / (threads 2^log2_entries)).  The default is the first,
 * the fastest measured on B200; cf_tune_set(e, lg, i) pins variant i (-1: the default again),
 * cf_tune_get returns the pinned index or -1, and cf_autotune times them like the others. */
int cf_tune_variants(int lg, int* log2_entries, int* threads, int* ctas_per_sm, int cap);
int cf_autotune(cf_engine* e, int nmax, int Mmax, int d, int B, double* rates, int cap, int* chosen);
int cf_tune_set(cf_engine* e, int lg, int variant);
int cf_tune_get(const cf_engine* e, int lg);

/* ---- resident tables for serving (no counterpart in the reference) ----
 * The reference rebuilds the suffix table for every run.  A served workload keeps, per (d, prime),
 * the whole table V and the factorial tables on the device, and answers later queries with
 * n' <= n and M' <= F from them in O(n'^2) per prime, with the same residues
 * (include/cuckoo/single_table.hpp:103-119 evaluates nbad from a retained table the same way). */
typedef struct cf_tables cf_tables;

/* Device bytes one prime's resident table takes for tables up to nmax and M up to Fmax. */
uint64_t cf_tables_bytes(int nmax, int Fmax);
/* Build and keep the tables of B primes (same requirements as cf_residues, with every prime above
 * Fmax).  Returns when they are on the device; *out owns that memory until cf_tables_free. */
int cf_tables_build(cf_engine* e, const uint64_t* primes, int B, int nmax, int Fmax, int d, int model, cf_tables** out);
/* residues[b*J + j] = N_bad(qn[j], qM[j]) mod primes[b] for the table set's primes, 1 <= qn[j] <= nmax,
 * qn[j] < qM[j] <= Fmax.  Host buffers; returns when the residues are in `residues`. */
int cf_tables_query(cf_engine* e, const cf_tables* t, const int* qn, const int* qM, int J, uint64_t* residues);
int cf_tables_count(const cf_tables* t);
/* Frees at once; tables built by cf_tables_build_async go back to the stream-ordered pool without
 * waiting for the device, so the caller must know no query on them is still in flight. */
void cf_tables_free(cf_tables* t);

/* Serving forms that never wait (the serving loop overlaps builds, queries and plain rebuilds).
 * cf_tables_build_async: the build of cf_tables_build enqueued on `stream` (memory from the
 * stream-ordered allocator); cf_tables_ready polls it: 1 when done, 0 while running, CF_ERR_DEVICE
 * if its device checks failed.  cf_tables_query_async: the residues of J queries into device memory,
 * d_residues[b * J + j], enqueued on `stream` after whatever the stream already holds (make the
 * stream wait for the build, or query only ready tables); the query sizes travel in the kernel
 * parameters, so queries on several streams share no buffer.  No counterpart in the reference. */
int cf_tables_build_async(cf_engine* e, const uint64_t* primes, int B, int nmax, int Fmax, int d, int model, void* stream,
                          cf_tables** out);
int cf_tables_ready(const cf_tables* t);
int cf_tables_query_async(cf_engine* e, const cf_tables* t, const int* qn, const int* qM, int J, uint64_t* d_residues,
                          void* stream);
/* At most n primes per launch for this engine's batches (0: no cap): n CTAs up to nmax = 16384,
 * n clusters above.  A long batch then leaves SMs to work on other streams, and the engine's
 * workspace holds at most n primes, leaving the rest of the device memory to others too. */
int cf_engine_set_max_ctas(cf_engine* e, int n);

/* Transforms of at least 2^lg entries for this engine's batches (0, the default: the reference's
 * transform_length(nmax)).  The convolutions are exact at every length from transform_length(nmax)
 * up, so the residues do not change; it runs the kernels of long transforms on small tables (tests)
 * and needs primes with 2^lg | p - 1 (every prime of the fixed lists, whose p - 1 has the factor
 * 2^20).  No counterpart in the reference, which fixes the length per batch (:460-472). */
int cf_engine_set_transform_lg(cf_engine* e, int lg);

/* ---- uneven batches: many instances in one graph of work-queue launches ----
 * Instances k = 0 .. K-1, (n[k], M[k], d[k]) under one model and prime list (bits = 50 or 62):
 * instance k needs N_bad(n[k], M[k]) modulo primes 0 .. need_k - 1 of the list, written at
 * residues[off_k + i] with off_k = cf_uneven_offset(u, k) (the prefix sums of the needs).  One table
 * per (d, prime index) serves every instance of degree d that needs the prime, built to the largest
 * such n: the reference's rule for a batch of primes (fast/cuckoo_fast.cu:787-795, 859-866) applied
 * per prime.  The tables are grouped by transform length; each group is one persistent launch whose
 * CTAs take tables heaviest first from a device counter; the groups are captured as one CUDA graph.
 * Only prime indices first + j stride < first + count are planned (count < 0: all), the rest of
 * the residues are left zero; a sampled plan times a whole workload on part of its primes.
 * Instances need 1 <= n < M, n <= 16384, and d <= M for the subset model.
 * The reference runs one instance set per process and d (fast/cuckoo_fast.cu:648-904). */
typedef struct cf_uneven cf_uneven;
int cf_uneven_create(cf_engine* e, const int* n, const int* M, const int* d, int K, int model, int bits, long first,
                     long count, long stride, cf_uneven** out);
/* Words of the residue array (the sum of the needs), instance k's offset in it, tables planned,
 * kernel launches per replay. */
long cf_uneven_outputs(const cf_uneven* u);
long cf_uneven_offset(const cf_uneven* u, int k);
long cf_uneven_tables(const cf_uneven* u);
long cf_uneven_launches(const cf_uneven* u);
/* Replay the graph on `stream` (NULL: the default stream); returns without waiting. */
int cf_uneven_launch(cf_uneven* u, void* stream);
/* Wait for `stream`, copy all residues to the host buffer; CF_ERR_DEVICE if a device check failed. */
int cf_uneven_results(cf_uneven* u, uint64_t* residues, void* stream);
void cf_uneven_destroy(cf_uneven* u);
/* The plan without a device (tests, tooling): rows of 7 longs per table, in launch order:
 * d, prime index, log2 transform length, table n, F, queries J, first query.  jcap > 0 splits tables
 * with more queries.  Returns the number of tables (writing at most cap rows), -1 on bad input. */
long cf_uneven_describe(const int* n, const int* M, const int* d, int K, int model, int bits, long first, long count,
                        long stride, int jcap, long* tables, long cap);

/* ---- allocation-free variant (no counterpart in the reference) ---- */

/* Bytes of the static device scratch used by cf_residues_noalloc (64 MiB).  One prime's table
 * fits up to about nmax = 4000; smaller tables are batched several primes per launch. */
#define CF_NOALLOC_SCRATCH_BYTES (64ull << 20)

/* The computation of cf_residues (primes of either list, below 2^50 or below 2^62), for callers
 * that cannot allocate device memory (their device memory belongs to another allocator,
 * allocation is forbidden where they run, or their device footprint must stay fixed after
 * start-up).  No engine, no cudaMalloc/cudaFree: all scratch is
 * a file-scope device array of CF_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until exit.  Host buffers; runs on `stream` (NULL = default stream) of the current device and
 * returns when the residues are in `residues`.  The first call on a device resolves the array's
 * address (make it before any stream capture).  All calls share the array, so calls that overlap
 * on the GPU race.  Returns CF_ERR_NOMEM, without launching, when one prime's workspace exceeds
 * the array.  No counterpart in the reference. */
int cf_residues_noalloc(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM, int J,
                        uint64_t* residues, void* stream);
/* Message for the last failed cf_residues_noalloc call ("" if none). */
const char* cf_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
