// C ABI for uneven batches (include/cuckoo_b200.h, cf_uneven_*): many instances (n, M, d), each
// modulo its own need(n, M, d) primes, computed by one persistent work-queue launch per transform
// length, all captured in one CUDA graph.
//
// The plan (uneven_plan.hpp) gives one table per (d, prime index), built to the largest n among
// that d's instances still needing the prime; k_suffix_queue's CTAs take the tables heaviest first
// from a device counter.  Compared with one launch per run of primes that share a query set (the
// reference driver's batches, fast/cuckoo_fast.cu:787-901), no SM idles while a short run's few
// primes finish, and each table is no larger than its own prime needs.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "engine_internal.hpp"
#include "uneven_plan.hpp"

using namespace cfb;

struct cf_uneven {
    int device = 0;
    cfh::UnevenPlan plan;
    QItem* d_items = nullptr;
    int* d_qn = nullptr;
    int* d_qM = nullptr;
    long long* d_qout = nullptr;
    int* d_next = nullptr;  // one counter per transform length
    int* d_err = nullptr;
    u64* d_out = nullptr;   // [plan.outputs]
    u64* ws = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long launches = 0;
    long slots = 0;  // CTAs of the largest launch
};

namespace {

// Queries per table the launch's shared memory holds at transform length 2^lg.
int jcap_for(int lg, bool wide) {
    const KInfo ki = kernel_for(lg, wide);
    int dev = 0, optin = 0;
    if (!ki.fn || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 0;
    const int nw = ki.threads >= 32 ? ki.threads / 32 : 1;
    return optin > (int)ki.smem ? (int)((optin - ki.smem) / (8 * (size_t)nw)) : 0;
}

void destroy(cf_uneven* u) {
    if (!u) return;
    cudaSetDevice(u->device);
    if (u->exec) cudaGraphExecDestroy(u->exec);
    if (u->graph) cudaGraphDestroy(u->graph);
    cudaFree(u->d_items);
    cudaFree(u->d_qn);
    cudaFree(u->d_qM);
    cudaFree(u->d_qout);
    cudaFree(u->d_next);
    cudaFree(u->d_err);
    cudaFree(u->d_out);
    cudaFree(u->ws);
    delete u;
}

}  // namespace

extern "C" {

long cf_uneven_describe(const int* n, const int* M, const int* d, int K, int model, int bits, long first, long count,
                        long stride, int jcap, long* tables, long cap) {
    if (K < 0 || (K > 0 && (!n || !M || !d)) || (bits != 50 && bits != 62)) return -1;
    cfh::UnevenPlan pl;
    if (!cfh::plan_uneven(n, M, d, K, model, bits, first, count, stride, jcap, pl)) return -1;
    for (size_t t = 0; t < pl.tables.size() && (long)t < cap; ++t) {
        const cfh::UnevenTable& x = pl.tables[t];
        long* o = tables + 7 * t;
        o[0] = x.d, o[1] = x.i, o[2] = x.lg, o[3] = x.n, o[4] = x.F, o[5] = x.J, o[6] = x.q0;
    }
    return (long)pl.tables.size();
}

int cf_uneven_create(cf_engine* e, const int* n, const int* M, const int* d, int K, int model, int bits, long first,
                     long count, long stride, cf_uneven** out) {
    if (!e || !out) return CF_ERR_ARG;
    *out = nullptr;
    e->err.clear();
    if (K < 1 || !n || !M || !d || (bits != 50 && bits != 62)) return fail(e, CF_ERR_ARG, "bad instance arrays or prime bits");
    const bool wide = bits == 62;
    CF_CUDA(cudaSetDevice(e->device), "set device");
    for (int k = 0; k < K; ++k)
        if (cfh::transform_length((u64)std::max(n[k], 1)) > (1ull << MAX_LG))
            return fail(e, CF_ERR_UNSUPPORTED, "an instance has n above 16384");
    // the query cap of the widest length bounds every table (shorter lengths hold more)
    const int jcap = jcap_for(MAX_LG, wide);
    cf_uneven* u = new cf_uneven();
    u->device = e->device;
    if (!cfh::plan_uneven(n, M, d, K, model, bits, first, count, stride, jcap, u->plan)) {
        destroy(u);
        return fail(e, CF_ERR_ARG, "invalid instances (need 1 <= n < M, d <= M for the subset model) or prime range");
    }
    const cfh::UnevenPlan& pl = u->plan;
    cudaStream_t cs = nullptr;
    auto run = [&]() -> int {
        const size_t T = pl.tables.size(), Q = pl.qn.size();
        std::vector<QItem> items(T);
        for (size_t t = 0; t < T; ++t) {
            const cfh::UnevenTable& x = pl.tables[t];
            items[t] = QItem{x.prime, x.n, x.F, x.d, model, x.J, (int)x.q0};
        }
        CF_CUDA(cudaMalloc(&u->d_out, 8 * (size_t)std::max<long>(pl.outputs, 1)), "residue buffer");
        CF_CUDA(cudaMemset(u->d_out, 0, 8 * (size_t)std::max<long>(pl.outputs, 1)), "residue buffer");
        CF_CUDA(cudaMalloc(&u->d_err, sizeof(int)), "error word");
        CF_CUDA(cudaMalloc(&u->d_next, sizeof(int) * (MAX_LG + 1)), "queue counters");
        if (T == 0) return CF_OK;
        CF_CUDA(cudaMalloc(&u->d_items, sizeof(QItem) * T), "table list");
        CF_CUDA(cudaMalloc(&u->d_qn, sizeof(int) * Q), "query list");
        CF_CUDA(cudaMalloc(&u->d_qM, sizeof(int) * Q), "query list");
        CF_CUDA(cudaMalloc(&u->d_qout, sizeof(long long) * Q), "query list");
        CF_CUDA(cudaMemcpy(u->d_items, items.data(), sizeof(QItem) * T, cudaMemcpyHostToDevice), "table upload");
        CF_CUDA(cudaMemcpy(u->d_qn, pl.qn.data(), sizeof(int) * Q, cudaMemcpyHostToDevice), "query upload");
        CF_CUDA(cudaMemcpy(u->d_qM, pl.qM.data(), sizeof(int) * Q, cudaMemcpyHostToDevice), "query upload");
        CF_CUDA(cudaMemcpy(u->d_qout, pl.qout.data(), sizeof(long long) * Q, cudaMemcpyHostToDevice), "query upload");
        // one launch per transform length (the list is ordered by length), each over its own slots
        struct Group {
            int lg;
            size_t a, b;  // tables [a, b)
            int nmax, F, J;
            Layout lay;
            long slots;
            KInfo ki;
            size_t smem;
        };
        std::vector<Group> gs;
        int sms = 0, dev = e->device;
        CF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        size_t ws_words_max = 0;
        long slots_max = 0;
        for (size_t a = 0; a < T;) {
            size_t b = a;
            Group g{pl.tables[a].lg, a, a, 0, 0, 0, Layout(), 0, KInfo(), 0};
            while (b < T && pl.tables[b].lg == g.lg) {
                g.nmax = std::max(g.nmax, pl.tables[b].n);
                g.F = std::max(g.F, pl.tables[b].F);
                g.J = std::max(g.J, pl.tables[b].J);
                ++b;
            }
            g.b = b;
            g.ki = kernel_for(g.lg, wide);
            if (!g.ki.qfn) return fail(e, CF_ERR_UNSUPPORTED, "no kernel for this transform length");
            const int nw = g.ki.threads >= 32 ? g.ki.threads / 32 : 1;
            g.lay = make_layout(g.nmax, g.F, 1 << g.lg, g.J, nw, g.ki.r);
            g.smem = g.ki.smem_for(g.J);
            int rc = check_smem(e, g.smem, g.J);
            if (rc) return rc;
            CF_CUDA(cudaFuncSetAttribute((const void*)g.ki.qfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem),
                    "shared memory attribute");
            int per_sm = 0;
            CF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, g.ki.qfn, g.ki.threads, g.smem), "occupancy");
            g.slots = std::min<long>((long)(b - a), (long)std::max(per_sm, 1) * sms);
            ws_words_max = std::max(ws_words_max, g.lay.total);
            slots_max = std::max(slots_max, g.slots);
            gs.push_back(g);
            a = b;
        }
        // the groups run one after another, so they share one workspace sized for the largest
        size_t fr = 0, tot = 0;
        CF_CUDA(cudaMemGetInfo(&fr, &tot), "free memory");
        const size_t reserve = (size_t)1 << 30, per = 8 * ws_words_max;
        const long fit = fr > reserve ? (long)((fr - reserve) / per) : 0;
        if (fit < 1) return fail(e, CF_ERR_NOMEM, "not enough device memory for one table");
        for (Group& g : gs) g.slots = std::min(g.slots, fit);
        slots_max = std::min(slots_max, fit);
        CF_CUDA(cudaMalloc(&u->ws, per * (size_t)slots_max), "workspace allocation");
        u->slots = slots_max;
        CF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
        CF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t ce = cudaMemsetAsync(u->d_err, 0, sizeof(int), cs);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(u->d_next, 0, sizeof(int) * (MAX_LG + 1), cs);
        for (const Group& g : gs) {
            if (ce != cudaSuccess) break;
            KParams kp;
            kp.primes = nullptr;  // per table, from the list
            kp.B = 1;
            kp.ws = u->ws;
            kp.ws_words = g.lay.total;
            kp.lay = g.lay;
            kp.out = u->d_out;
            kp.err = u->d_err;
            QueueParams qp;
            qp.items = u->d_items + g.a;
            qp.count = (int)(g.b - g.a);
            qp.next = u->d_next + g.lg;
            qp.qn = u->d_qn, qp.qM = u->d_qM, qp.qout = u->d_qout;
            g.ki.qfn<<<(unsigned)g.slots, g.ki.threads, g.smem, cs>>>(kp, qp);
            ce = cudaGetLastError();
            ++u->launches;
        }
        cudaGraph_t gr = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(cs, &gr);
        u->graph = gr;
        CF_CUDA(ce, "capture");
        CF_CUDA(ee, "end capture");
        CF_CUDA(cudaGraphInstantiate(&u->exec, u->graph, 0), "graph instantiation");
        return CF_OK;
    };
    const int rc = run();
    if (cs) cudaStreamDestroy(cs);
    if (rc) {
        destroy(u);
        return rc;
    }
    *out = u;
    return CF_OK;
}

long cf_uneven_outputs(const cf_uneven* u) { return u ? u->plan.outputs : 0; }
long cf_uneven_offset(const cf_uneven* u, int k) {
    return u && k >= 0 && k < (int)u->plan.off.size() ? u->plan.off[k] : -1;
}
long cf_uneven_tables(const cf_uneven* u) { return u ? (long)u->plan.tables.size() : 0; }
long cf_uneven_launches(const cf_uneven* u) { return u ? u->launches : 0; }

int cf_uneven_launch(cf_uneven* u, void* stream) {
    if (!u) return CF_ERR_ARG;
    if (!u->exec) return CF_OK;  // nothing planned
    if (cudaSetDevice(u->device) != cudaSuccess) return CF_ERR_CUDA;
    return cudaGraphLaunch(u->exec, (cudaStream_t)stream) == cudaSuccess ? CF_OK : CF_ERR_CUDA;
}

int cf_uneven_results(cf_uneven* u, uint64_t* residues, void* stream) {
    if (!u || (u->plan.outputs > 0 && !residues)) return CF_ERR_ARG;
    if (cudaSetDevice(u->device) != cudaSuccess) return CF_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    int herr = 0;
    if (u->plan.outputs > 0 &&
        cudaMemcpyAsync(residues, u->d_out, 8 * (size_t)u->plan.outputs, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return CF_ERR_CUDA;
    if (cudaMemcpyAsync(&herr, u->d_err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CF_ERR_CUDA;
    return herr ? CF_ERR_DEVICE : CF_OK;
}

void cf_uneven_destroy(cf_uneven* u) { destroy(u); }

}  // extern "C"
