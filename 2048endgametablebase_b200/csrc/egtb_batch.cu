// Batched build of libegtb_gpu: many tables advance together, one kernel
// launch per global layer step for all of them (egtb_batch.cuh), the per-step
// loops captured once as CUDA graphs and replayed, one radix sort for the
// layers of every table, one packing pass for every book.
//
// Capacities: every table gets slices of pooled device buffers. A table whose
// slice overflows during the forward pass flags it; the forward is re-run
// with that table's slice grown. After a successful forward the exact sizes
// are known and remembered for this set of tables (with the autotuned launch
// parameters), so a repeated build of the same tables neither re-runs nor
// re-captures its graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "egtb_batch.cuh"
#include "egtb_host.h"

namespace egtb {
namespace {

constexpr unsigned long long kMinArena = 1ull << 14, kMinStage = 1ull << 12, kMinSet = 1ull << 13;

unsigned long long align16u(unsigned long long x) { return (x + 15ull) & ~15ull; }

unsigned long long pow2_at_least(unsigned long long x, unsigned long long lo) {
    unsigned long long c = lo;
    while (c < x) c <<= 1;
    return c;
}

// Grow-only device allocation (contents are not kept across growth).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    void ensure(size_t want, const char *what) {
        if (p && want <= bytes) return;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        const size_t sz = std::max<size_t>(want + want / 4, 4096);
        if (cudaMalloc(&p, sz) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            throw Error(EGTB_ERR_CAPACITY, std::string("device allocation of ") + std::to_string(sz >> 20) +
                                               " MiB for the batch's " + what + " failed");
        }
        bytes = sz;
    }
    template <typename T> T *as() const { return (T *)p; }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

struct TableCaps {
    unsigned long long arena = kMinArena, stage = kMinStage, set = kMinSet;
    int filter_bits = 12;
};

// Host view of one table.
struct TablePlan {
    egtb_pattern_spec spec;
    const egtb_run_options *opt;
    const uint64_t *seeds;
    unsigned long long n_seeds;
    long long s0;
    int steps, docheck;
    FreeNibbles fn;
    DevSpec ds;
    TableCaps caps;
    int lbase = 0;
    unsigned long long abase = 0, stage_off = 0, set_off = 0, filter_off = 0, index_off = 0, index_slots = 0;
    unsigned long long max_len = 0;
};

struct Remembered {
    std::vector<TableCaps> caps;
    egtb_batch_params params;
    bool tuned = false;
};

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned long long> key;
    unsigned long long nodes = 0;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        nodes = 0;
    }
};

struct BatchEngine {
    int device = 0;
    cudaStream_t cap_stream = nullptr;  // capture only: graphs are launched on the build stream
    cudaEvent_t ev[6];
    DevBuf arena, rates, stage, sets, filters, index, book, comp, status, seeds;
    DevBuf layer_off, layer_len, book_len, layer_max, first_tile, tile_cnt, tile_off;
    DevBuf tables, ctl, sync, devctl, hist, counters, seed_at, seg_tab, seg_hist;
    unsigned char *pinned = nullptr;
    size_t pinned_cap = 0;
    unsigned epoch = 1;
    GraphCache fwd, bwd;
    std::map<unsigned long long, Remembered> memory;
    // the last batch, for egtb_batch_book_copy
    std::vector<int> last_lbase, last_steps;
    std::vector<unsigned long long> last_off, last_blen;
    size_t last_rec = 0;
    unsigned long long last_book_bytes = 0;

    void init(int dev) {
        device = dev;
        EGTB_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
        for (auto &e : ev) EGTB_CUDA(cudaEventCreate(&e));
        hist.ensure(sizeof(unsigned) * kMaxPasses * 256, "histograms");
        EGTB_CUDA(cudaMemset(hist.p, 0, hist.bytes));
        counters.ensure(sizeof(unsigned) * 16, "tile counters");
        devctl.ensure(sizeof(DevCtl), "control block");
        sync.ensure(sizeof(BatchSync), "control block");
    }

    unsigned char *ensure_pinned(size_t bytes) {
        if (bytes <= pinned_cap) return pinned;
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        pinned_cap = 0;
        const size_t want = std::max<size_t>(bytes, 16ull << 20);
        if (cudaHostAlloc((void **)&pinned, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            pinned = nullptr;
            throw Error(EGTB_ERR_NOMEM, "pinned host allocation of " + std::to_string(want >> 20) + " MiB failed");
        }
        pinned_cap = want;
        return pinned;
    }
};

std::mutex g_batch_mu;
std::vector<std::unique_ptr<BatchEngine>> g_batch;

BatchEngine &batch_engine(int device) {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    if ((int)g_batch.size() <= device) g_batch.resize(device + 1);
    if (!g_batch[device]) {
        auto b = std::make_unique<BatchEngine>();
        b->init(device);
        g_batch[device] = std::move(b);
    }
    return *g_batch[device];
}

long long tile_sum_host(uint64_t b) {
    long long s = 0;
    for (int k = 0; k < 16; ++k) {
        const int v = (int)((b >> (4 * k)) & 0xF);
        s += v ? (1ll << v) : 0ll;
    }
    return s;
}

unsigned long long fnv(unsigned long long h, const void *p, size_t n) {
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 0x100000001B3ull;
    return h;
}

// Identity of a set of tables: everything that shapes their layers.
unsigned long long batch_signature(const std::vector<TablePlan> &tp) {
    unsigned long long h = 0xCBF29CE484222325ull;
    for (const auto &t : tp) {
        h = fnv(h, t.spec.pattern_masks, sizeof(uint64_t) * t.spec.n_masks);
        h = fnv(h, t.spec.success_shifts, t.spec.n_shifts);
        h = fnv(h, &t.spec.symm_mode, sizeof t.spec.symm_mode);
        h = fnv(h, &t.opt->target, sizeof t.opt->target);
        h = fnv(h, &t.steps, sizeof t.steps);
        h = fnv(h, &t.docheck, sizeof t.docheck);
        h = fnv(h, &t.opt->spawn_rate4, sizeof t.opt->spawn_rate4);
        h = fnv(h, &t.opt->success_rate_dtype, sizeof t.opt->success_rate_dtype);
        h = fnv(h, t.seeds, sizeof(uint64_t) * t.n_seeds);
        h = fnv(h, "|", 1);
    }
    return h;
}

egtb_batch_params default_params() {
    egtb_batch_params p;
    std::memset(&p, 0, sizeof p);
    p.expand_chunk = 128;
    p.expand_blocks_per_sm = 3;
    p.digit_nibbles = 2;
    p.index_load = 2;
    p.use_graphs = 1;
    return p;
}

// Fields of `given` that are set override `base`.
egtb_batch_params merge_params(egtb_batch_params base, const egtb_batch_params *given) {
    if (!given) return base;
    if (given->expand_chunk) base.expand_chunk = given->expand_chunk;
    if (given->expand_blocks_per_sm) base.expand_blocks_per_sm = given->expand_blocks_per_sm;
    if (given->digit_nibbles) base.digit_nibbles = given->digit_nibbles;
    if (given->index_load) base.index_load = given->index_load;
    if (given->use_graphs) base.use_graphs = given->use_graphs > 0 ? 1 : 0;
    return base;
}

void check_params(const egtb_batch_params &p) {
    if (p.expand_chunk < 32 || p.expand_chunk > 4096 || p.expand_chunk % 32)
        throw Error(EGTB_ERR_ARG, "expand_chunk must be a multiple of 32 in 32..4096");
    if (p.expand_blocks_per_sm < 1 || p.expand_blocks_per_sm > 8)
        throw Error(EGTB_ERR_ARG, "expand_blocks_per_sm must be 1..8");
    if (p.digit_nibbles != 1 && p.digit_nibbles != 2) throw Error(EGTB_ERR_ARG, "digit_nibbles must be 1 or 2");
    if (p.index_load != 2 && p.index_load != 4) throw Error(EGTB_ERR_ARG, "index_load must be 2 or 4");
}

std::vector<TablePlan> make_plans(int n, const uint64_t *const *seeds, const uint64_t *n_seeds,
                                  const egtb_pattern_spec *specs, const egtb_run_options *opts) {
    if (n <= 0 || n > kMaxBatchTables) throw Error(EGTB_ERR_ARG, "n_tables must be 1..1024");
    if (!seeds || !n_seeds || !specs || !opts) throw Error(EGTB_ERR_ARG, "seeds, n_seeds, specs and options are required");
    std::vector<TablePlan> tp(n);
    for (int i = 0; i < n; ++i) {
        const egtb_run_options &o = opts[i];
        TablePlan &t = tp[i];
        if (o.device != opts[0].device) throw Error(EGTB_ERR_ARG, "all tables of a batch must use one device");
        if (o.success_rate_dtype != opts[0].success_rate_dtype)
            throw Error(EGTB_ERR_ARG, "all tables of a batch must use one success_rate_dtype");
        dtype_size(o.success_rate_dtype);
        if (o.is_variant)
            throw Error(EGTB_ERR_UNSUPPORTED, "variant boards (wall-merge mover) are built one at a time: use egtb_build");
        if (o.compress) throw Error(EGTB_ERR_UNSUPPORTED, "compressed books (compress) are not built");
        if (o.steps < 3 || o.steps > (1 << 16)) throw Error(EGTB_ERR_ARG, "steps of a batched table must be 3..65536");
        if (o.deletion_threshold > 0.0 || o.optimal_branch_only)
            throw Error(EGTB_ERR_UNSUPPORTED,
                        "deletion_threshold / optimal_branch_only rewrite book files: build such a table with egtb_build");
        if (specs[i].symm_mode < 0 || specs[i].symm_mode > 3)
            throw Error(EGTB_ERR_UNSUPPORTED, "symmetry modes min33/min24/min34 are not built");
        if (n_seeds[i] == 0 || !seeds[i]) throw Error(EGTB_ERR_ARG, "every table needs seed boards");
        t.spec = specs[i];
        t.opt = &o;
        t.seeds = seeds[i];
        t.n_seeds = n_seeds[i];
        t.s0 = tile_sum_host(seeds[i][0]);
        for (unsigned long long j = 1; j < n_seeds[i]; ++j)
            if (tile_sum_host(seeds[i][j]) != t.s0)
                throw Error(EGTB_ERR_ARG, "seed boards must share one tile sum (as the pattern catalog keeps them)");
        t.steps = o.steps;
        t.docheck = o.docheck_step;
        t.ds = make_dev_spec(specs[i], o.target);
        std::memset(&t.fn, 0, sizeof t.fn);
        t.fn.pinned = pattern_pinned_nibbles(specs[i]);
        for (int k = 0; k < 16; ++k)
            if (((t.fn.pinned >> (4 * k)) & 0xF) != 0xF) t.fn.idx[t.fn.count++] = k;
    }
    return tp;
}

__global__ void batch_seed_kernel(const BatchTable *__restrict__ T, int n, const uint64_t *__restrict__ seeds,
                                  const unsigned long long *__restrict__ at) {
    for (int i = blockIdx.x; i < n; i += gridDim.x)
        for (unsigned long long j = at[i] + threadIdx.x; j < at[i + 1]; j += blockDim.x) T[i].stage[0][j - at[i]] = seeds[j];
}


struct Run {
    BatchEngine &B;
    EngineRef R;
    std::vector<TablePlan> &tp;
    egtb_batch_params prm;
    int n = 0, max_steps = 0, G = 0;
    int dtype = 0;
    size_t rec = 0;
    unsigned long long arena_total = 0, stage_total = 0, set_total = 0, filter_total = 0;
    unsigned long long launches = 0, graph_launches = 0;
    bool graphs_used = false;
    std::vector<unsigned long long> len;  // host copy of layer_len (G)
    std::vector<BatchTable> host_tables;

    cudaStream_t s() const { return *R.stream; }

    void layout() {
        n = (int)tp.size();
        max_steps = 0;
        G = 0;
        arena_total = stage_total = set_total = filter_total = 0;
        for (auto &t : tp) {
            t.lbase = G;
            G += t.steps + 1;
            max_steps = std::max(max_steps, t.steps);
            t.abase = arena_total;
            arena_total += align16u(t.caps.arena);
            t.stage_off = stage_total;
            stage_total += 3 * t.caps.stage;
            t.set_off = set_total;
            set_total += 2 * t.caps.set;
            t.filter_off = filter_total;
            filter_total += 1ull << t.caps.filter_bits;
        }
        B.arena.ensure(sizeof(uint64_t) * arena_total, "layer arena");
        B.stage.ensure(sizeof(uint64_t) * stage_total, "staging buffers");
        B.sets.ensure(sizeof(uint64_t) * set_total, "dedup sets");
        B.filters.ensure(sizeof(uint64_t) * filter_total, "repeat filters");
        B.layer_off.ensure(sizeof(unsigned long long) * (G + 1), "layer offsets");
        B.layer_len.ensure(sizeof(unsigned long long) * (G + 1), "layer lengths");
        B.tables.ensure(sizeof(BatchTable) * n, "table descriptors");
        B.ctl.ensure(sizeof(BatchCtl) * n, "table counters");
        host_tables.assign(n, BatchTable{});
        for (int i = 0; i < n; ++i) {
            const TablePlan &t = tp[i];
            BatchTable &b = host_tables[i];
            std::memset(&b, 0, sizeof b);
            b.spec = t.ds;
            b.fn = t.fn;
            b.s0 = t.s0;
            b.p4 = t.opt->spawn_rate4;
            b.steps = t.steps;
            b.docheck = t.docheck;
            b.lbase = t.lbase;
            b.filter_bits = t.caps.filter_bits;
            b.abase = t.abase;
            b.acap = t.caps.arena;
            for (int k = 0; k < 3; ++k) b.stage[k] = B.stage.as<uint64_t>() + t.stage_off + k * t.caps.stage;
            b.stage_cap = t.caps.stage;
            for (int k = 0; k < 2; ++k) b.set[k] = B.sets.as<uint64_t>() + t.set_off + k * t.caps.set;
            b.set_mask = t.caps.set - 1;
            b.filter = B.filters.as<uint64_t>() + t.filter_off;
        }
    }

    void upload_tables() {
        EGTB_CUDA(cudaMemcpyAsync(B.tables.p, host_tables.data(), sizeof(BatchTable) * n, cudaMemcpyHostToDevice, s()));
    }

    // Run a per-step loop directly or as a cached CUDA graph keyed by every
    // pointer and size the launches embed.
    template <typename F>
    void run_loop(GraphCache &gc, const std::vector<unsigned long long> &key, unsigned long long nodes, F enqueue) {
        if (!prm.use_graphs) {
            enqueue(s());
            launches += nodes;
            return;
        }
        if (!gc.exec || gc.key != key) {
            gc.reset();
            cudaGraph_t g = nullptr;
            EGTB_CUDA(cudaStreamBeginCapture(B.cap_stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue(B.cap_stream);
            } catch (...) {
                cudaStreamEndCapture(B.cap_stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            EGTB_CUDA(cudaStreamEndCapture(B.cap_stream, &g));
            const cudaError_t e = cudaGraphInstantiate(&gc.exec, g, 0);
            cudaGraphDestroy(g);
            EGTB_CUDA(e);
            gc.key = key;
            gc.nodes = nodes;
        }
        EGTB_CUDA(cudaGraphLaunch(gc.exec, s()));
        ++graph_launches;
        launches += gc.nodes;
        graphs_used = true;
    }

    std::vector<unsigned long long> base_key() const {
        return {(unsigned long long)n, (unsigned long long)max_steps, (unsigned long long)(uintptr_t)B.tables.p,
                (unsigned long long)(uintptr_t)B.ctl.p, (unsigned long long)(uintptr_t)B.arena.p,
                (unsigned long long)(uintptr_t)B.layer_off.p, (unsigned long long)(uintptr_t)B.layer_len.p,
                (unsigned long long)(uintptr_t)B.sync.p, (unsigned long long)(uintptr_t)R.tab};
    }

    // Forward pass of every table. Returns the OR of the tables' error flags.
    unsigned forward() {
        for (auto &t : tp)
            if (t.n_seeds > t.caps.stage) t.caps.stage = pow2_at_least(t.n_seeds, kMinStage);
        layout();
        // counters, sets, filters, layer arrays
        std::vector<BatchCtl> hc(n);
        std::memset(hc.data(), 0, sizeof(BatchCtl) * n);
        std::vector<unsigned long long> at(n + 1, 0);
        for (int i = 0; i < n; ++i) {
            hc[i].stage_count[0] = tp[i].n_seeds;
            at[i + 1] = at[i] + tp[i].n_seeds;
        }
        std::vector<unsigned long long> off0(G + 1, 0);
        for (auto &t : tp) off0[t.lbase] = t.abase;
        upload_tables();
        EGTB_CUDA(cudaMemcpyAsync(B.ctl.p, hc.data(), sizeof(BatchCtl) * n, cudaMemcpyHostToDevice, s()));
        EGTB_CUDA(cudaMemsetAsync(B.sync.p, 0, sizeof(BatchSync), s()));
        EGTB_CUDA(cudaMemsetAsync(B.sets.p, 0, sizeof(uint64_t) * set_total, s()));
        EGTB_CUDA(cudaMemsetAsync(B.filters.p, 0, sizeof(uint64_t) * filter_total, s()));
        EGTB_CUDA(cudaMemsetAsync(B.layer_len.p, 0, sizeof(unsigned long long) * (G + 1), s()));
        EGTB_CUDA(cudaMemcpyAsync(B.layer_off.p, off0.data(), sizeof(unsigned long long) * (G + 1),
                                  cudaMemcpyHostToDevice, s()));
        // seeds: one copy, one scatter kernel
        B.seeds.ensure(sizeof(uint64_t) * at[n], "seeds");
        B.seed_at.ensure(sizeof(unsigned long long) * (n + 1), "seed offsets");
        unsigned char *h = B.ensure_pinned(sizeof(uint64_t) * at[n] + sizeof(unsigned long long) * (n + 1));
        for (int i = 0; i < n; ++i) std::memcpy(h + sizeof(uint64_t) * at[i], tp[i].seeds, sizeof(uint64_t) * tp[i].n_seeds);
        std::memcpy(h + sizeof(uint64_t) * at[n], at.data(), sizeof(unsigned long long) * (n + 1));
        EGTB_CUDA(cudaMemcpyAsync(B.seeds.p, h, sizeof(uint64_t) * at[n], cudaMemcpyHostToDevice, s()));
        EGTB_CUDA(cudaMemcpyAsync(B.seed_at.p, h + sizeof(uint64_t) * at[n], sizeof(unsigned long long) * (n + 1),
                                  cudaMemcpyHostToDevice, s()));
        batch_seed_kernel<<<std::min(n, 1024), 256, 0, s()>>>(B.tables.as<BatchTable>(), n, B.seeds.as<uint64_t>(),
                                                             B.seed_at.as<unsigned long long>());
        EGTB_CUDA(cudaGetLastError());
        ++launches;
        // one launch per global step
        const int grid = R.sm_count * prm.expand_blocks_per_sm;
        unsigned *progress = build_progress_ptr();
        std::vector<unsigned long long> key = base_key();
        key.push_back((unsigned long long)grid);
        key.push_back((unsigned long long)prm.expand_chunk);
        EGTB_CUDA(cudaEventRecord(B.ev[0], s()));
        run_loop(B.fwd, key, (unsigned long long)max_steps, [&](cudaStream_t st) {
            for (int t = 0; t < max_steps; ++t)
                batch_expand_kernel<<<grid, kBatchThreads, 0, st>>>(
                    B.tables.as<BatchTable>(), B.ctl.as<BatchCtl>(), n, t, B.arena.as<uint64_t>(),
                    B.layer_off.as<unsigned long long>(), B.layer_len.as<unsigned long long>(), R.tab,
                    (unsigned)prm.expand_chunk, B.sync.as<BatchSync>(), progress, (unsigned)(t + 1));
            EGTB_CUDA(cudaGetLastError());
        });
        EGTB_CUDA(cudaEventRecord(B.ev[1], s()));
        EGTB_CUDA(cudaMemcpyAsync(hc.data(), B.ctl.p, sizeof(BatchCtl) * n, cudaMemcpyDeviceToHost, s()));
        EGTB_CUDA(cudaStreamSynchronize(s()));
        EGTB_CUDA(cudaGetLastError());
        unsigned any = 0;
        for (int i = 0; i < n; ++i) {
            const unsigned e = hc[i].err & kErrBatchForward;
            any |= e;
            TableCaps &c = tp[i].caps;
            if (e & kErrCandOverflow) c.stage *= 4;
            if (e & kErrDedupOverflow) {
                c.set *= 4;
                c.filter_bits = std::min(20, c.filter_bits + 2);
            }
            if (e & kErrArenaOverflow) c.arena *= 4;
            cand_[i] = hc[i].candidates;
        }
        return any;
    }
    std::vector<unsigned long long> cand_;

    // Layers 1..steps-1 of every table sorted, each in its own arena region,
    // by the free nibbles of its table (per-layer digit positions), digit
    // width digit_nibbles (1 or 2 nibbles).
    void sort_layers() {
        len.assign(G + 1, 0);
        EGTB_CUDA(cudaMemcpyAsync(len.data(), B.layer_len.p, sizeof(unsigned long long) * (G + 1),
                                  cudaMemcpyDeviceToHost, s()));
        EGTB_CUDA(cudaStreamSynchronize(s()));
        std::vector<int> lt(G + 1, 0);
        int fmax = 0;
        for (int i = 0; i < n; ++i) {
            const TablePlan &t = tp[i];
            fmax = std::max(fmax, t.fn.count);
            for (int L = 0; L <= t.steps; ++L) lt[t.lbase + L] = i;
        }
        std::vector<int> tab;
        std::vector<int> tile0(G, 0);
        for (int g = 0; g < G; ++g) {
            const int i = lt[g];
            const int L = g - tp[i].lbase;
            if (L < 1 || L >= tp[i].steps) continue;
            tile0[g] = (int)tab.size();
            const unsigned long long nt = (len[g] + kTileKeys - 1) / kTileKeys;
            for (unsigned long long j = 0; j < nt; ++j) tab.push_back(g);
        }
        const unsigned ntiles = (unsigned)tab.size();
        if (ntiles == 0) return;
        tab.reserve(tab.size() + tile0.size());
    for (const int v : tile0) tab.push_back(v);
        int dn = prm.digit_nibbles == 1 ? 1 : 2;
        if ((fmax + dn - 1) / dn > kMaxPasses) dn = 2;
        const int passes = (fmax + dn - 1) / dn;
        std::vector<unsigned short> nib((size_t)G * kMaxPasses, 0xFFFFu);
        for (int g = 0; g < G; ++g) {
            const FreeNibbles &fn = tp[lt[g]].fn;
            for (int q = 0; q < passes; ++q) {
                const int a = dn * q, b = dn * q + 1;
                const unsigned lo = a < fn.count ? (unsigned)fn.idx[a] : 0xFFu;
                const unsigned hi = (dn == 2 && b < fn.count) ? (unsigned)fn.idx[b] : 0xFFu;
                nib[(size_t)g * kMaxPasses + q] = (unsigned short)(lo | (hi << 8));
            }
        }
        const size_t hist_words = (size_t)G * kMaxPasses * 256;
        B.seg_tab.ensure(sizeof(int) * tab.size(), "layer sort tile map");
        B.seg_hist.ensure(sizeof(unsigned) * hist_words + sizeof(unsigned short) * nib.size(), "layer sort histograms");
        B.comp.ensure(sizeof(uint64_t) * std::max<unsigned long long>(arena_total, 1), "sort buffer");
        if (B.status.bytes < sizeof(unsigned long long) * 256 * ((size_t)ntiles + 2)) {
            B.status.ensure(sizeof(unsigned long long) * 256 * ((size_t)ntiles + 2), "sort look-back");
            EGTB_CUDA(cudaMemsetAsync(B.status.p, 0, B.status.bytes, s()));
        }
        const int *tile_layer = B.seg_tab.as<int>(), *layer_tile0 = tile_layer + ntiles;
        unsigned *hist = B.seg_hist.as<unsigned>();
        unsigned short *seg_nib = reinterpret_cast<unsigned short *>(hist + hist_words);
        EGTB_CUDA(cudaMemcpyAsync(B.seg_tab.p, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, s()));
        EGTB_CUDA(cudaMemcpyAsync(seg_nib, nib.data(), sizeof(unsigned short) * nib.size(), cudaMemcpyHostToDevice, s()));
        EGTB_CUDA(cudaMemsetAsync(hist, 0, sizeof(unsigned) * hist_words, s()));
        DevCtl *dc = B.devctl.as<DevCtl>();
        EGTB_CUDA(cudaMemsetAsync(dc, 0, sizeof(DevCtl), s()));
        const unsigned long long *loff = B.layer_off.as<unsigned long long>(), *llen = B.layer_len.as<unsigned long long>();
        seg_hist_kernel<<<R.sm_count * 2, kHistThreads, 0, s()>>>(B.arena.as<uint64_t>(), tile_layer, layer_tile0, loff, llen,
                                                                  ntiles, passes, seg_nib, hist, B.counters.as<unsigned>());
        ++launches;
        uint64_t *src = B.arena.as<uint64_t>(), *dst = B.comp.as<uint64_t>();
        // this file's copy of the kernel (it is static in the header) needs its own attribute
        EGTB_CUDA(cudaFuncSetAttribute(seg_onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSegSweepSmem));
        for (int q = 0; q < passes; ++q) {
            seg_onesweep_kernel<<<R.seg_grid, kSweepThreads, kSegSweepSmem, s()>>>(src, dst, tile_layer, layer_tile0, loff, llen,
                                                                        ntiles, seg_nib, q, hist,
                                                                        B.counters.as<unsigned>(),
                                                                        B.status.as<unsigned long long>(), B.epoch++, dc,
                                                                        look_back_spin_limit());
            std::swap(src, dst);
            ++launches;
        }
        if (src != B.arena.as<uint64_t>()) {
            seg_copy_kernel<<<R.sm_count * 8, 256, 0, s()>>>(src, B.arena.as<uint64_t>(), tile_layer, layer_tile0, loff,
                                                             llen, ntiles);
            ++launches;
        }
        EGTB_CUDA(cudaGetLastError());
    }

    template <typename T>
    void backward() {
        const T zero = (T)dtype_zero(dtype), maxv = (T)dtype_max(dtype);
        unsigned long long index_total = 0;
        for (int i = 0; i < n; ++i) {
            TablePlan &t = tp[i];
            t.max_len = 0;
            for (int L = 0; L < t.steps; ++L) t.max_len = std::max(t.max_len, len[t.lbase + L]);
            t.index_slots = pow2_at_least((unsigned long long)prm.index_load * std::max(1ull, t.max_len), 64);
            t.index_off = index_total;
            index_total += 4 * t.index_slots;
        }
        B.index.ensure(sizeof(ulonglong2) * index_total, "rate index");
        B.rates.ensure(sizeof(T) * arena_total, "rates");
        for (int i = 0; i < n; ++i) {
            for (int k = 0; k < 4; ++k)
                host_tables[i].index[k] = B.index.as<ulonglong2>() + tp[i].index_off + k * tp[i].index_slots;
            host_tables[i].index_mask = tp[i].index_slots - 1;
        }
        upload_tables();
        EGTB_CUDA(cudaMemsetAsync(B.index.p, 0, sizeof(ulonglong2) * index_total, s()));
        const int g = R.sm_count * 8;
        unsigned *progress = build_progress_ptr();
        const unsigned total_prog = (unsigned)(2 * max_steps);
        std::vector<unsigned long long> key = base_key();
        key.push_back((unsigned long long)(uintptr_t)B.rates.p);
        key.push_back((unsigned long long)sizeof(T));
        key.push_back((unsigned long long)dtype);
        run_loop(B.bwd, key, (unsigned long long)max_steps - 1, [&](cudaStream_t st) {
            batch_final_kernel<T><<<g, 256, 0, st>>>(B.tables.as<BatchTable>(), B.ctl.as<BatchCtl>(), n,
                                                     B.arena.as<uint64_t>(), B.rates.as<T>(),
                                                     B.layer_off.as<unsigned long long>(),
                                                     B.layer_len.as<unsigned long long>(), zero, maxv);
            for (int t = max_steps - 3; t >= 0; --t)
                batch_solve_kernel<T><<<g, 256, 0, st>>>(B.tables.as<BatchTable>(), B.ctl.as<BatchCtl>(), n, t,
                                                         B.arena.as<uint64_t>(), B.rates.as<T>(),
                                                         B.layer_off.as<unsigned long long>(),
                                                         B.layer_len.as<unsigned long long>(), R.tab, zero, maxv,
                                                         B.sync.as<BatchSync>(), progress, total_prog - (unsigned)t - 2u);
            EGTB_CUDA(cudaGetLastError());
        });
    }

    template <typename T>
    void pack() {
        const T zero = (T)dtype_zero(dtype);
        std::vector<unsigned long long> ft(G + 1, 0);
        for (int g = 0; g < G; ++g) ft[g + 1] = ft[g] + (len[g] + kTileKeys - 1) / kTileKeys;
        const unsigned long long n_tiles = ft[G];
        B.first_tile.ensure(sizeof(unsigned long long) * (G + 1), "tile map");
        B.tile_cnt.ensure(sizeof(unsigned) * (n_tiles + 1), "tile counts");
        B.tile_off.ensure(sizeof(unsigned long long) * (n_tiles + 1), "tile offsets");
        B.book_len.ensure(sizeof(unsigned long long) * (G + 1), "book lengths");
        B.layer_max.ensure(sizeof(unsigned long long) * (G + 1), "layer maxima");
        B.book.ensure(rec * arena_total, "books");
        EGTB_CUDA(cudaMemcpyAsync(B.first_tile.p, ft.data(), sizeof(unsigned long long) * (G + 1), cudaMemcpyHostToDevice, s()));
        EGTB_CUDA(cudaMemsetAsync(B.layer_max.p, 0, sizeof(unsigned long long) * (G + 1), s()));
        EGTB_CUDA(cudaMemsetAsync(B.book_len.p, 0, sizeof(unsigned long long) * (G + 1), s()));
        const int g = R.sm_count * 4;
        DevCtl *dc = B.devctl.as<DevCtl>();
        book_count_all_kernel<T><<<g, kSortThreads, 0, s()>>>(B.rates.as<T>(), B.layer_off.as<unsigned long long>(),
                                                            B.layer_len.as<unsigned long long>(),
                                                            B.first_tile.as<unsigned long long>(), G, n_tiles, zero,
                                                            B.tile_cnt.as<unsigned>(), B.layer_max.as<unsigned long long>());
        scan_tiles_kernel<<<1, 1024, 0, s()>>>(B.tile_cnt.as<unsigned>(), n_tiles, B.tile_off.as<unsigned long long>(),
                                               &dc->n_unique);
        book_lens_kernel<<<(G + 255) / 256, 256, 0, s()>>>(B.first_tile.as<unsigned long long>(), G, n_tiles,
                                                           B.tile_off.as<unsigned long long>(), &dc->n_unique,
                                                           B.book_len.as<unsigned long long>());
        book_write_all_kernel<T><<<g, kSortThreads, 0, s()>>>(
            B.arena.as<uint64_t>(), B.rates.as<T>(), B.layer_off.as<unsigned long long>(),
            B.layer_len.as<unsigned long long>(), B.first_tile.as<unsigned long long>(), G, n_tiles, zero,
            B.tile_off.as<unsigned long long>(), B.book.as<unsigned char>(), (unsigned long long)B.book.bytes, dc);
        launches += 4;
        EGTB_CUDA(cudaGetLastError());
    }
};

double elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    EGTB_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

template <typename T>
void run_batch(Run &X, egtb_build_stats *table_stats, egtb_batch_stats *bs, double *device_ms) {
    BatchEngine &B = X.B;
    const auto t_start = std::chrono::steady_clock::now();
    const int n = (int)X.tp.size();
    X.cand_.assign(n, 0);
    int retries = 0;
    int max_steps = 0;
    for (auto &t : X.tp) max_steps = std::max(max_steps, t.steps);
    const uint32_t total_prog = (uint32_t)(2 * max_steps);
    build_progress_set(0, total_prog);
    for (;;) {
        if (X.forward() == 0) break;
        if (++retries > 24) throw Error(EGTB_ERR_CAPACITY, "batched forward did not fit after repeated regrowth");
    }
    X.sort_layers();
    EGTB_CUDA(cudaEventRecord(B.ev[2], X.s()));
    X.template backward<T>();
    EGTB_CUDA(cudaEventRecord(B.ev[3], X.s()));
    X.template pack<T>();
    EGTB_CUDA(cudaEventRecord(B.ev[4], X.s()));
    const int G = X.G;
    std::vector<BatchCtl> hc(n);
    std::vector<unsigned long long> off(G + 1), blen(G + 1), maxb(G + 1);
    BatchSync hs;
    DevCtl dctl;
    EGTB_CUDA(cudaMemcpyAsync(hc.data(), B.ctl.p, sizeof(BatchCtl) * n, cudaMemcpyDeviceToHost, X.s()));
    EGTB_CUDA(cudaMemcpyAsync(off.data(), B.layer_off.p, sizeof(unsigned long long) * (G + 1), cudaMemcpyDeviceToHost, X.s()));
    EGTB_CUDA(cudaMemcpyAsync(blen.data(), B.book_len.p, sizeof(unsigned long long) * (G + 1), cudaMemcpyDeviceToHost, X.s()));
    EGTB_CUDA(cudaMemcpyAsync(maxb.data(), B.layer_max.p, sizeof(unsigned long long) * (G + 1), cudaMemcpyDeviceToHost, X.s()));
    EGTB_CUDA(cudaMemcpyAsync(&hs, B.sync.p, sizeof hs, cudaMemcpyDeviceToHost, X.s()));
    EGTB_CUDA(cudaMemcpyAsync(&dctl, B.devctl.p, sizeof dctl, cudaMemcpyDeviceToHost, X.s()));
    EGTB_CUDA(cudaStreamSynchronize(X.s()));
    EGTB_CUDA(cudaGetLastError());
    for (int i = 0; i < n; ++i)
        if (hc[i].err & kErrIndexOverflow) throw Error(EGTB_ERR_CAPACITY, "rate index probe chain too long");
    if (dctl.err & kErrTimeout) throw Error(EGTB_ERR_TIMEOUT, "a bounded device wait gave up in the batch's layer sort");
    if (dctl.err) throw Error(EGTB_ERR_CAPACITY, "book buffer overflow");
    const double fwd_ms = elapsed(B.ev[0], B.ev[1]), sort_ms = elapsed(B.ev[1], B.ev[2]),
                 bwd_ms = elapsed(B.ev[2], B.ev[3]), pack_ms = elapsed(B.ev[3], B.ev[4]);
    if (device_ms) *device_ms = elapsed(B.ev[0], B.ev[4]);
    // remember exact capacities for the next build of these tables
    {
        Remembered &m = B.memory[batch_signature(X.tp)];
        m.caps.resize(n);
        for (int i = 0; i < n; ++i) {
            const TablePlan &t = X.tp[i];
            unsigned long long need = 0, mx = 0;
            for (int L = 0; L < t.steps; ++L) {
                need += align16u(X.len[t.lbase + L]);
                mx = std::max(mx, X.len[t.lbase + L]);
            }
            TableCaps c = t.caps;
            c.arena = std::max(kMinArena, need + 16);
            c.stage = std::max<unsigned long long>(kMinStage, std::max<unsigned long long>(mx, t.n_seeds));
            m.caps[i] = c;
        }
    }
    // the last batch, for egtb_batch_book_copy
    B.last_lbase.resize(n);
    B.last_steps.resize(n);
    for (int i = 0; i < n; ++i) {
        B.last_lbase[i] = X.tp[i].lbase;
        B.last_steps[i] = X.tp[i].steps;
    }
    B.last_off = off;
    B.last_blen = blen;
    B.last_rec = X.rec;
    B.last_book_bytes = B.book.bytes;
    // files
    const double sec_per_layer = (fwd_ms + sort_ms + bwd_ms + pack_ms) * 1e-3 / std::max(1, max_steps);
    unsigned long long file_bytes = 0;
    for (int i = 0; i < n; ++i)
        if (X.tp[i].opt->write_files)
            for (int L = 0; L < X.tp[i].steps; ++L) file_bytes += blen[X.tp[i].lbase + L] * X.rec;
    if (file_bytes) {
        unsigned char *h = B.ensure_pinned(file_bytes);
        std::vector<std::string> paths;
        std::vector<unsigned long long> hoff, bytes;
        unsigned long long pos = 0;
        for (int i = 0; i < n; ++i) {
            const TablePlan &t = X.tp[i];
            if (!t.opt->write_files) continue;
            for (int L = 0; L < t.steps; ++L) {
                const int g = t.lbase + L;
                const unsigned long long b = blen[g] * X.rec;
                if (b) EGTB_CUDA(cudaMemcpyAsync(h + pos, B.book.as<unsigned char>() + off[g] * X.rec, b,
                                                 cudaMemcpyDeviceToHost, X.s()));
                paths.push_back(std::string(t.opt->pathname) + std::to_string(L) + ".book");
                hoff.push_back(pos);
                bytes.push_back(b);
                pos += b;
            }
        }
        EGTB_CUDA(cudaStreamSynchronize(X.s()));
        WriterPool pool(X.tp[0].opt->num_threads > 0 ? std::min(X.tp[0].opt->num_threads, 32) : 8);
        for (size_t k = 0; k < paths.size(); ++k) pool.submit(paths[k], h + hoff[k], bytes[k]);
        pool.wait();
    }
    for (int i = 0; i < n; ++i) {
        const TablePlan &t = X.tp[i];
        if (!t.opt->write_files) continue;
        std::vector<unsigned long long> rl(t.steps), bl(t.steps), mb(t.steps);
        for (int L = 0; L < t.steps; ++L) {
            rl[L] = X.len[t.lbase + L];
            bl[L] = blen[t.lbase + L];
            mb[L] = maxb[t.lbase + L];
        }
        std::vector<int> order;
        for (int L = t.steps - 3; L >= 0; --L) order.push_back(L);
        write_stats_file(*t.opt, X.dtype, order, rl, bl, mb, sec_per_layer);
    }
    build_progress_set(total_prog, total_prog);
    const double total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    egtb_batch_stats agg;
    std::memset(&agg, 0, sizeof agg);
    for (int i = 0; i < n; ++i) {
        const TablePlan &t = X.tp[i];
        egtb_build_stats st;
        std::memset(&st, 0, sizeof st);
        for (int L = 0; L < t.steps; ++L) {
            const unsigned long long l = X.len[t.lbase + L];
            if (L <= t.steps - 3) st.raw_boards += l;
            st.book_entries += blen[t.lbase + L];
            st.max_layer = std::max<uint64_t>(st.max_layer, l);
        }
        st.candidates = hc[i].candidates;
        st.layers = t.steps;
        st.retries = retries;
        st.forward_ms = fwd_ms + sort_ms;
        st.backward_ms = bwd_ms + pack_ms;
        st.total_ms = total_ms;
        st.kernel_launches = X.launches;
        if (table_stats) table_stats[i] = st;
        agg.raw_boards += st.raw_boards;
        agg.book_entries += st.book_entries;
        agg.candidates += st.candidates;
    }
    agg.lookups = hs.lookups;
    agg.tables = n;
    agg.max_steps = max_steps;
    agg.retries = retries;
    agg.graphs_used = X.graphs_used ? 1 : 0;
    agg.forward_ms = fwd_ms;
    agg.sort_ms = sort_ms;
    agg.backward_ms = bwd_ms;
    agg.pack_ms = pack_ms;
    agg.total_ms = total_ms;
    agg.kernel_launches = X.launches;
    agg.graph_launches = X.graph_launches;
    agg.params = X.prm;
    if (bs) *bs = agg;
}

// One build under params; returns device ms.
double build_once(BatchEngine &B, EngineRef &R, std::vector<TablePlan> &tp, const egtb_batch_params &prm,
                  egtb_build_stats *table_stats, egtb_batch_stats *bs) {
    Run X{B, R, tp, prm};
    X.dtype = tp[0].opt->success_rate_dtype;
    X.rec = record_size(X.dtype);
    double ms = 0;
    switch (X.dtype) {
        case EGTB_DTYPE_UINT32: run_batch<uint32_t>(X, table_stats, bs, &ms); break;
        case EGTB_DTYPE_UINT64: run_batch<uint64_t>(X, table_stats, bs, &ms); break;
        case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32: run_batch<float>(X, table_stats, bs, &ms); break;
        default: run_batch<double>(X, table_stats, bs, &ms); break;
    }
    return ms;
}

// Capacities of a set of tables: remembered ones, else the small defaults.
void apply_memory(BatchEngine &B, std::vector<TablePlan> &tp, egtb_batch_params *tuned) {
    auto it = B.memory.find(batch_signature(tp));
    if (it == B.memory.end()) return;
    for (size_t i = 0; i < tp.size() && i < it->second.caps.size(); ++i) tp[i].caps = it->second.caps[i];
    if (tuned && it->second.tuned) *tuned = it->second.params;
}

}  // namespace

// egtb_release: free the batch buffers of a device (the caller holds the
// device's build lock). Captured graphs name the old buffers: dropped too.
void batch_release_buffers(int device) {
    BatchEngine *B = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        if (device < (int)g_batch.size()) B = g_batch[device].get();
    }
    if (!B) return;
    B->fwd.reset();
    B->bwd.reset();
    for (DevBuf *d : {&B->arena, &B->rates, &B->stage, &B->sets, &B->filters, &B->index, &B->book, &B->comp,
                      &B->status, &B->seeds, &B->layer_off, &B->layer_len, &B->book_len, &B->layer_max,
                      &B->first_tile, &B->tile_cnt, &B->tile_off, &B->tables, &B->ctl, &B->seed_at, &B->seg_tab,
                      &B->seg_hist})
        d->release();
    if (B->pinned) cudaFreeHost(B->pinned);
    B->pinned = nullptr;
    B->pinned_cap = 0;
    B->last_lbase.clear();
    B->last_steps.clear();
    B->last_off.clear();
    B->last_blen.clear();
    B->last_book_bytes = 0;
}

}  // namespace egtb

using namespace egtb;

extern "C" int egtb_build_batch(int32_t n_tables, const uint64_t *const *seeds, const uint64_t *n_seeds,
                                const egtb_pattern_spec *specs, const egtb_run_options *options,
                                const egtb_batch_params *params, egtb_build_stats *table_stats, egtb_batch_stats *stats) {
    return guarded([&] {
        std::vector<TablePlan> tp = make_plans(n_tables, seeds, n_seeds, specs, options);
        EngineRef R = engine_ref(options[0].device);
        std::lock_guard<std::mutex> lk(*R.mu);
        EGTB_CUDA(cudaSetDevice(R.device));
        BatchEngine &B = batch_engine(R.device);
        egtb_batch_params prm = default_params();
        apply_memory(B, tp, &prm);
        prm = merge_params(prm, params);
        check_params(prm);
        build_once(B, R, tp, prm, table_stats, stats);
    });
}

extern "C" int egtb_batch_autotune(int32_t n_tables, const uint64_t *const *seeds, const uint64_t *n_seeds,
                                   const egtb_pattern_spec *specs, const egtb_run_options *options,
                                   egtb_batch_params *best, double *best_ms) {
    return guarded([&] {
        std::vector<egtb_run_options> opts(options, options + (n_tables > 0 ? n_tables : 0));
        for (auto &o : opts) o.write_files = 0;
        std::vector<TablePlan> tp = make_plans(n_tables, seeds, n_seeds, specs, opts.data());
        EngineRef R = engine_ref(options[0].device);
        std::lock_guard<std::mutex> lk(*R.mu);
        EGTB_CUDA(cudaSetDevice(R.device));
        BatchEngine &B = batch_engine(R.device);
        egtb_batch_params cur = default_params();
        apply_memory(B, tp, nullptr);
        // settle capacities and graphs once, then time each candidate (best of two)
        build_once(B, R, tp, cur, nullptr, nullptr);
        apply_memory(B, tp, nullptr);
        auto timed = [&](const egtb_batch_params &p) {
            double a = build_once(B, R, tp, p, nullptr, nullptr);
            double b = build_once(B, R, tp, p, nullptr, nullptr);
            return std::min(a, b);
        };
        double cur_ms = timed(cur);
        auto try_field = [&](int32_t egtb_batch_params::*field, std::initializer_list<int32_t> values) {
            for (int32_t v : values) {
                if (cur.*field == v) continue;
                egtb_batch_params p = cur;
                p.*field = v;
                const double ms = timed(p);
                if (ms < cur_ms) {
                    cur_ms = ms;
                    cur = p;
                }
            }
        };
        try_field(&egtb_batch_params::expand_chunk, {32, 64, 128, 256, 512});
        try_field(&egtb_batch_params::expand_blocks_per_sm, {2, 3, 6});
        try_field(&egtb_batch_params::digit_nibbles, {1, 2});
        try_field(&egtb_batch_params::index_load, {2, 4});
        Remembered &m = B.memory[batch_signature(tp)];
        m.params = cur;
        m.tuned = true;
        if (best) *best = cur;
        if (best_ms) *best_ms = cur_ms;
    });
}

extern "C" int egtb_batch_book_copy(int device, int32_t table, int32_t layer, void *dst, size_t dst_bytes,
                                    size_t *bytes) {
    return guarded([&] {
        EngineRef R = engine_ref(device);
        std::lock_guard<std::mutex> lk(*R.mu);
        BatchEngine &B = batch_engine(R.device);
        if (table < 0 || table >= (int)B.last_lbase.size()) throw Error(EGTB_ERR_ARG, "no such table in the last batch");
        if (layer < 0 || layer >= B.last_steps[table]) throw Error(EGTB_ERR_ARG, "layer out of range");
        const int g = B.last_lbase[table] + layer;
        const size_t b = (size_t)(B.last_blen[g] * B.last_rec);
        if (bytes) *bytes = b;
        if (!dst) return;
        if (dst_bytes < b) throw Error(EGTB_ERR_ARG, "destination too small");
        if (b) EGTB_CUDA(cudaMemcpy(dst, B.book.as<unsigned char>() + B.last_off[g] * B.last_rec, b, cudaMemcpyDeviceToHost));
    });
}
