// Build engine of libegtb_gpu: the forward layer generation and backward solve
// of the classic tablebase path on one B200, behind the C ABI of
// include/egtb_gpu.h (egtb_build / egtb_generate / egtb_solve / progress /
// board primitives).
//
// Fused build (egtb_build with no layer files on disk): every raw layer stays
// in one device arena (16-aligned offsets) for the whole build. Forward step
// i is one kernel: it expands layer i-1 and enters the spawn-2 children of
// layer i and the spawn-4 children of layer i+1 into those layers' hash sets
// (exact dedup), appending the new keys to the layers' staging buffers; it
// copies layer i-1 into the arena. After the last step every layer is sorted
// in its own region (enqueue_sort_layers). All sizes stay on the device, so
// the host enqueues the whole forward without waiting; capacity overflows are
// flagged by the kernels and the forward is re-run with larger buffers.
// Backward solve runs layer by layer on the same arena, then every layer is
// packed into .book records on the device and written by a thread pool.
#include <cuda_runtime.h>
#include <dirent.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <future>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "egtb_host.h"
#include "egtb_kernels.cuh"
#include "egtb_sort.cuh"
#include "egtb_trie.h"

namespace egtb {

// ------------------------------------------------------------- progress ---

static std::atomic<uint32_t> g_progress_total{0};
static std::atomic<uint32_t> g_progress_host{0};
static unsigned *g_progress_mapped = nullptr;      // host view (device-written)
static unsigned *g_progress_mapped_dev = nullptr;  // device view
static std::mutex g_progress_mu;

static unsigned *progress_device_ptr() {
    std::lock_guard<std::mutex> lk(g_progress_mu);
    if (!g_progress_mapped) {
        unsigned *h = nullptr;
        if (cudaHostAlloc(&h, sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        *h = 0;
        unsigned *d = nullptr;
        if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
            cudaGetLastError();
            cudaFreeHost(h);
            return nullptr;
        }
        g_progress_mapped = h;
        g_progress_mapped_dev = d;
    }
    return g_progress_mapped_dev;
}

// update_build_progress, native_core/include/FormationRuntime.h:62-66
static void set_progress(uint32_t cur, uint32_t total) {
    g_progress_total.store(total, std::memory_order_relaxed);
    g_progress_host.store(cur, std::memory_order_relaxed);
    if (g_progress_mapped) *(volatile unsigned *)g_progress_mapped = cur;
}

static uint32_t read_progress() {
    uint32_t cur = g_progress_host.load(std::memory_order_relaxed);
    if (g_progress_mapped) {
        const uint32_t d = *(volatile unsigned *)g_progress_mapped;
        if (d > cur) cur = d;
    }
    return cur;
}

// ---------------------------------------------------------------- engine ---

static unsigned long long align16(unsigned long long x) { return (x + 15ull) & ~15ull; }

// Launch a kernel on the engine's stream and count it.
#define EGTB_LAUNCH(E, ...)  \
    do {                     \
        __VA_ARGS__;         \
        ++(E).launches;      \
    } while (0)

// Launch a kernel that may start while the kernel before it in the stream
// finishes (programmatic stream serialization). The kernel calls pdl_wait()
// before it reads anything the launch before wrote.
template <typename Eng, typename Kernel, typename... Args>
static void launch_dependent(Eng &E, Kernel kernel, int grid, int block, size_t smem, cudaStream_t s, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    EGTB_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
    ++E.launches;
}

static const char *kKindNames[] = {"expand", "sort_pass", "layer_sort", "solve", "book_pack", "final_layers",
                                   "rate_index"};
enum { K_EXPAND = 0, K_SORT_PASS, K_UNIQUE, K_SOLVE, K_PACK, K_FINAL, K_INDEX, K_NKINDS };

static unsigned long long env_bytes(const char *name) {
    const char *v = getenv(name);
    return (v && *v) ? strtoull(v, nullptr, 10) : 0ull;
}

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream in use
    cudaStream_t own_stream = nullptr;  // the library's stream
    unsigned long long launches = 0;
    // per-kind device timing: one event pair around a run of `count`
    // consecutive launches of one kind (a whole layer loop is one run, so the
    // timing adds two events per loop, not two per launch; a run's time
    // includes the gaps between its launches)
    bool prof = false;
    struct ProfPair {
        int kind;
        cudaEvent_t a, b;
        unsigned long long count;
    };
    std::vector<ProfPair> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    unsigned long long prof_launches[K_NKINDS] = {};
    double prof_ms[K_NKINDS] = {};

    int prof_begin(int kind, unsigned long long count = 1) {
        if (!prof) return -1;
        cudaEvent_t a, b;
        if (prof_pool.size() >= 2) {
            a = prof_pool.back();
            prof_pool.pop_back();
            b = prof_pool.back();
            prof_pool.pop_back();
        } else {
            EGTB_CUDA(cudaEventCreate(&a));
            EGTB_CUDA(cudaEventCreate(&b));
        }
        EGTB_CUDA(cudaEventRecord(a, stream));
        prof_pending.push_back({kind, a, b, count});
        return (int)prof_pending.size() - 1;
    }
    void prof_end(int idx) {
        if (idx < 0) return;
        EGTB_CUDA(cudaEventRecord(prof_pending[idx].b, stream));
    }
    // after a stream synchronisation: fold the recorded pairs into the totals
    void prof_resolve() {
        for (auto &p : prof_pending) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                prof_ms[p.kind] += ms;
                prof_launches[p.kind] += p.count;
            } else {
                cudaGetLastError();
            }
            prof_pool.push_back(p.a);
            prof_pool.push_back(p.b);
        }
        prof_pending.clear();
    }
    const uint32_t *tab = nullptr;                     // row table of the running build
    const uint32_t *classic_tab = nullptr, *variant_tab = nullptr;
    std::mutex mu;

    // Select the mover of the next build: classic, or the variant boards' wall merge.
    void use_mover(bool variant) { tab = variant ? variant_tab : classic_tab; }

    // capacities (elements)
    unsigned long long arena_cap = 0, cand_cap = 0;
    int steps_cap = 0;

    uint64_t *arena = nullptr;
    void *rates = nullptr;
    unsigned long long rates_bytes = 0;
    // the last fused build, for egtb_book_layer_copy
    int last_steps = 0;
    size_t last_rec = 0;
    std::vector<unsigned long long> last_off, last_blen;
    uint64_t *split = nullptr;
    // streamed forward: two sort buffers, a copy stream and its events
    uint64_t *sort_buf[2] = {nullptr, nullptr};
    unsigned long long sort_cap = 0;
    cudaStream_t copy_stream = nullptr;
    cudaStream_t pack_stream = nullptr;  // book packing of finished layer groups, beside the solve
    cudaEvent_t ev_sorted = nullptr, ev_copied = nullptr;
    uint64_t *cand[2] = {nullptr, nullptr};
    uint64_t *tmp = nullptr;
    unsigned *hist = nullptr;               // digit histograms, kMaxPasses x 256
    unsigned *counters = nullptr;           // tile counters of the sort passes and the unique kernel
    unsigned long long *status = nullptr;   // look-back words, sort_tiles x 256
    unsigned long long *ustatus = nullptr;  // look-back words of the unique kernel, sort_tiles
    unsigned epoch = 1;                     // tags the look-back words of one kernel launch
    int sweep_grid = 0;                     // resident blocks of the onesweep kernel
    int seg_grid = 0;                       // resident blocks of the per-layer onesweep kernel
    unsigned *tile_cnt = nullptr;
    unsigned long long *tile_off = nullptr;
    unsigned long long sort_tiles = 0, comp_tiles = 0;
    uint64_t *dset[3] = {nullptr, nullptr, nullptr};  // exact dedup sets: layer L in set L % 3
    unsigned long long dset_cap = 0;          // slots per set
    uint64_t *filter = nullptr;               // direct-mapped repeat filter in front of the sets
    int filter_bits = 20;
    int *seg_tab = nullptr;                    // per-layer sort: tile -> layer, then layer -> first tile
    unsigned long long seg_tab_cap = 0;
    unsigned *seg_hist = nullptr;              // per-layer sort: digit histograms (layer x pass x 256), digit positions
    unsigned long long seg_hist_cap = 0;
    unsigned long long candidates = 0;        // children probed by the last forward pass
    unsigned long long *layer_off = nullptr, *layer_len = nullptr, *book_len = nullptr;
    unsigned long long *layer_max = nullptr;  // ordered encoding of the largest rate per layer
    unsigned char *book = nullptr;
    unsigned long long book_cap_bytes = 0;
    ulonglong2 *index[4] = {nullptr, nullptr, nullptr, nullptr};  // rate index of layer L in index[L % 4]
    unsigned long long index_cap = 0;                    // slots per index
    unsigned long long *first_tile = nullptr;            // all-layer packing: first tile of every layer
    DevCtl *ctl = nullptr;
    cudaEvent_t ev[4];

    // pinned host staging
    unsigned char *pinned = nullptr;
    size_t pinned_cap = 0;

    int sm_count = 148;

    void init(int dev) {
        device = dev;
        EGTB_CUDA(cudaSetDevice(dev));
        EGTB_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        stream = own_stream;
        classic_tab = device_row_table(false);
        variant_tab = device_row_table(true);
        tab = classic_tab;
        cudaDeviceProp prop;
        EGTB_CUDA(cudaGetDeviceProperties(&prop, dev));
        sm_count = prop.multiProcessorCount;
        EGTB_CUDA(cudaMalloc(&ctl, sizeof(DevCtl)));
        for (auto &e : ev) EGTB_CUDA(cudaEventCreate(&e));
        const char *fb = getenv("EGTB_FILTER_BITS");
        if (fb) filter_bits = std::max(10, std::min(30, atoi(fb)));
        EGTB_CUDA(cudaMalloc(&filter, sizeof(uint64_t) << filter_bits));
        EGTB_CUDA(cudaMalloc(&hist, sizeof(unsigned) * kMaxPasses * 256));
        EGTB_CUDA(cudaMemset(hist, 0, sizeof(unsigned) * kMaxPasses * 256));
        EGTB_CUDA(cudaMalloc(&counters, sizeof(unsigned) * 16));
        int per_sm = 0;
        EGTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_kernel, kSweepThreads, 0));
        EGTB_CUDA(cudaFuncSetAttribute(expand_dedup_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowSmemBytes));
        EGTB_CUDA(cudaFuncSetAttribute(expand_dedup_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowSmemBytes));
        sweep_grid = sm_count * std::max(1, per_sm);
        EGTB_CUDA(cudaFuncSetAttribute(seg_onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSegSweepSmem));
        EGTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, seg_onesweep_kernel, kSweepThreads, kSegSweepSmem));
        seg_grid = sm_count * std::max(1, per_sm);
        progress_device_ptr();
    }

    template <typename P>
    static void release(P *&p) {
        if (p) cudaFree((void *)p);
        p = nullptr;
    }

    // egtb_release: every buffer that grows with the tables built (arena,
    // rates, books, sets, indexes, sort buffers, pinned staging); the next
    // build allocates again. The books of the last build go with them.
    void release_buffers() {
        for (auto *p : {&arena, &split, &tmp, &sort_buf[0], &sort_buf[1], &cand[0], &cand[1], &dset[0], &dset[1],
                        &dset[2]})
            release(*p);
        release(rates);
        release(book);
        for (auto &p : index) release(p);
        release(status);
        release(ustatus);
        release(tile_cnt);
        release(tile_off);
        release(seg_tab);
        release(seg_hist);
        release(layer_off);
        release(layer_len);
        release(book_len);
        release(layer_max);
        release(first_tile);
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        pinned_cap = 0;
        arena_cap = cand_cap = rates_bytes = sort_cap = sort_tiles = comp_tiles = dset_cap = 0;
        seg_tab_cap = seg_hist_cap = book_cap_bytes = index_cap = 0;
        steps_cap = 0;
        last_steps = 0;
        last_off.clear();
        last_blen.clear();
    }

    void alloc_or_throw(void **p, size_t bytes, const char *what) {
        // EGTB_MAX_ALLOC_BYTES: refuse larger single allocations, as a smaller
        // device would (exercises the streamed fallback on any GPU)
        static const unsigned long long max_alloc = env_bytes("EGTB_MAX_ALLOC_BYTES");
        if (max_alloc && bytes > max_alloc) {
            *p = nullptr;
            throw Error(EGTB_ERR_CAPACITY, std::string("device allocation of ") + std::to_string(bytes >> 20) +
                                               " MiB for " + what + " is above EGTB_MAX_ALLOC_BYTES");
        }
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            throw Error(EGTB_ERR_CAPACITY, std::string("device allocation of ") + std::to_string(bytes >> 20) +
                                               " MiB for " + what + " failed");
        }
    }

    // Run a grow step; if an allocation fails, forget the capacity (the
    // buffers it released are gone) and rethrow.
    template <typename F>
    void grow(unsigned long long &cap, F &&f) {
        try {
            f();
        } catch (...) {
            cap = 0;
            throw;
        }
    }

    void ensure_steps(int steps) {
        if (steps + 3 <= steps_cap) return;
        release(layer_off);
        release(layer_len);
        release(book_len);
        release(layer_max);
        steps_cap = std::max(steps + 3, 1024);
        alloc_or_throw((void **)&layer_off, sizeof(unsigned long long) * steps_cap, "layer offsets");
        alloc_or_throw((void **)&layer_len, sizeof(unsigned long long) * steps_cap, "layer lengths");
        alloc_or_throw((void **)&book_len, sizeof(unsigned long long) * steps_cap, "book lengths");
        alloc_or_throw((void **)&layer_max, sizeof(unsigned long long) * steps_cap, "layer maxima");
        release(first_tile);
        alloc_or_throw((void **)&first_tile, sizeof(unsigned long long) * steps_cap, "tile map");
    }

    void ensure_dedup(unsigned long long slots) {
        if (slots <= dset_cap) return;
        for (auto &p : dset) release(p);
        dset_cap = slots;
        grow(dset_cap, [&] {
            for (auto &p : dset) alloc_or_throw((void **)&p, sizeof(uint64_t) * dset_cap, "dedup set");
        });
    }

    // per-layer sort tables: `tiles` tile entries + `layers` layer entries, histograms of `layers` layers
    void ensure_seg(unsigned long long tiles, unsigned long long layers) {
        if (tiles + layers > seg_tab_cap) {
            release(seg_tab);
            seg_tab_cap = tiles + layers + (tiles + layers) / 4 + 64;
            alloc_or_throw((void **)&seg_tab, sizeof(int) * seg_tab_cap, "layer sort tile map");
        }
        // histograms (layer x pass x 256) followed by the digit positions (layer x pass, u16)
        const unsigned long long hist_words = layers * kMaxPasses * 256 + (layers * kMaxPasses + 1) / 2;
        if (hist_words > seg_hist_cap) {
            release(seg_hist);
            seg_hist_cap = hist_words;
            alloc_or_throw((void **)&seg_hist, sizeof(unsigned) * seg_hist_cap, "layer sort histograms");
        }
        ensure_status(tiles);
    }

    // look-back words for sorts of up to max(cand_cap, arena_cap) keys (and at least `tiles` tiles)
    void ensure_status(unsigned long long tiles = 0) {
        const unsigned long long need = std::max(std::max(cand_cap, arena_cap) / kTileKeys + 2, tiles);
        if (need <= sort_tiles) return;
        release(status);
        release(ustatus);
        sort_tiles = need;
        alloc_or_throw((void **)&status, sizeof(unsigned long long) * 256 * sort_tiles, "sort look-back");
        alloc_or_throw((void **)&ustatus, sizeof(unsigned long long) * sort_tiles, "unique look-back");
        EGTB_CUDA(cudaMemset(status, 0, sizeof(unsigned long long) * 256 * sort_tiles));
        EGTB_CUDA(cudaMemset(ustatus, 0, sizeof(unsigned long long) * sort_tiles));
    }

    void ensure_index(unsigned long long slots) {
        if (slots <= index_cap) return;
        for (auto &p : index) release(p);
        index_cap = slots;
        grow(index_cap, [&] {
            for (auto &p : index) alloc_or_throw((void **)&p, sizeof(ulonglong2) * index_cap, "rate index");
        });
    }

    void ensure_arena(unsigned long long cap) {
        if (cap <= arena_cap) return;
        release(arena);
        release(rates);
        rates_bytes = 0;
        release(split);
        release(book);
        arena_cap = align16(cap);
        grow(arena_cap, [&] {
            alloc_or_throw((void **)&arena, sizeof(uint64_t) * arena_cap, "layer arena");
            alloc_or_throw((void **)&split, sizeof(uint64_t) * (arena_cap / kSplitStride + 1), "splitters");
            book_cap_bytes = arena_cap * 16ull;
            alloc_or_throw((void **)&book, book_cap_bytes, "books");
        });
        ensure_comp_tiles();
        ensure_status();
    }

    // rates of every arena slot, in the build's dtype
    void ensure_rates(size_t elem_bytes) {
        const unsigned long long need = arena_cap * elem_bytes;
        if (need <= rates_bytes) return;
        release(rates);
        rates_bytes = need;
        grow(rates_bytes, [&] { alloc_or_throw(&rates, need, "rates"); });
    }

    void ensure_cand(unsigned long long cap) {
        if (cap <= cand_cap) return;
        if (cap >= (1ull << 32)) throw Error(EGTB_ERR_CAPACITY, "candidate buffer above 2^32 keys");
        release(cand[0]);
        release(cand[1]);
        release(tmp);
        cand_cap = cap;
        grow(cand_cap, [&] {
            alloc_or_throw((void **)&cand[0], sizeof(uint64_t) * cand_cap, "candidates");
            alloc_or_throw((void **)&cand[1], sizeof(uint64_t) * cand_cap, "candidates");
            alloc_or_throw((void **)&tmp, sizeof(uint64_t) * cand_cap, "sort buffer");
        });
        ensure_status();
        ensure_comp_tiles();
    }

    void ensure_comp_tiles() {
        const unsigned long long need = std::max(arena_cap, cand_cap) / kTileKeys + 2;
        if (need <= comp_tiles) return;
        release(tile_cnt);
        release(tile_off);
        comp_tiles = need;
        alloc_or_throw((void **)&tile_cnt, sizeof(unsigned) * comp_tiles, "tile counts");
        alloc_or_throw((void **)&tile_off, sizeof(unsigned long long) * comp_tiles, "tile offsets");
    }

    void ensure_copy_stream() {
        if (copy_stream) return;
        EGTB_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
        EGTB_CUDA(cudaStreamCreateWithFlags(&pack_stream, cudaStreamNonBlocking));
        EGTB_CUDA(cudaEventCreateWithFlags(&ev_sorted, cudaEventDisableTiming));
        EGTB_CUDA(cudaEventCreateWithFlags(&ev_copied, cudaEventDisableTiming));
    }

    void ensure_sort_bufs(unsigned long long cap) {
        if (cap <= sort_cap) return;
        for (auto &p : sort_buf) release(p);
        sort_cap = cap;
        grow(sort_cap, [&] {
            for (auto &p : sort_buf) alloc_or_throw((void **)&p, sizeof(uint64_t) * sort_cap, "layer sort buffer");
        });
        ensure_copy_stream();
    }

    unsigned char *ensure_pinned(size_t bytes) {
        if (bytes <= pinned_cap) return pinned;
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        pinned_cap = 0;
        size_t want = std::max<size_t>(bytes, 64ull << 20);
        if (cudaHostAlloc((void **)&pinned, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            pinned = nullptr;
            throw Error(EGTB_ERR_NOMEM, "pinned host allocation of " + std::to_string(want >> 20) + " MiB failed");
        }
        pinned_cap = want;
        return pinned;
    }

    int grid_for(int threads_per_block, int blocks_per_sm) const { return sm_count * blocks_per_sm; }
};

static std::mutex g_engines_mu;
static std::vector<std::unique_ptr<Engine>> g_engines;

static Engine &engine_for(int device) {
    int n = 0;
    EGTB_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw Error(EGTB_ERR_ARG, "device " + std::to_string(device) + " not present");
    std::lock_guard<std::mutex> lk(g_engines_mu);
    if ((int)g_engines.size() < n) g_engines.resize(n);
    if (!g_engines[device]) {
        EGTB_CUDA(cudaSetDevice(device));
        auto e = std::make_unique<Engine>();
        e->init(device);
        g_engines[device] = std::move(e);
    }
    EGTB_CUDA(cudaSetDevice(device));
    return *g_engines[device];
}

// Nibbles that can differ between canonical keys: a nibble pinned to 0xF by
// every mask, and by every symmetry image of that intersection, is 0xF in
// every canonical key, so the sort skips it.
static uint64_t pinned_nibbles(const egtb_pattern_spec &s) {
    uint64_t pinned = 0;
    if (s.n_masks > 0) {
        pinned = ~0ull;
        for (int i = 0; i < s.n_masks; ++i) pinned &= s.pattern_masks[i];
        // keep only nibbles that are fully 0xF
        uint64_t nib = 0;
        for (int k = 0; k < 16; ++k)
            if (((pinned >> (4 * k)) & 0xF) == 0xF) nib |= 0xFull << (4 * k);
        pinned = nib;
        auto sym = [](uint64_t b, int idx) {
            uint64_t o = 0;
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) {
                    uint64_t v = (b >> (4 * ((3 - r) * 4 + (3 - c)))) & 0xF;
                    int R = r, C = c;
                    switch (idx) {
                        case 1: C = 3 - c; break;
                        case 2: R = 3 - r; break;
                        case 3: R = c; C = r; break;
                        case 4: R = 3 - c; C = 3 - r; break;
                        case 5: R = 3 - r; C = 3 - c; break;
                        case 6: R = 3 - c; C = r; break;
                        case 7: R = c; C = 3 - r; break;
                        default: break;
                    }
                    o |= v << (4 * ((3 - R) * 4 + (3 - C)));
                }
            return o;
        };
        uint64_t inter = pinned;
        if (s.symm_mode == EGTB_SYMM_DIAGONAL) inter &= sym(pinned, 3);
        if (s.symm_mode == EGTB_SYMM_HORIZONTAL) inter &= sym(pinned, 1);
        if (s.symm_mode == EGTB_SYMM_FULL)
            for (int g = 1; g < 8; ++g) inter &= sym(pinned, g);
        pinned = inter;
    }
    return pinned;
}

// Digits of the LSD passes: the free nibbles from least significant up, two per pass.
static SortPlan sort_plan(const egtb_pattern_spec &s) {
    const uint64_t pinned = pinned_nibbles(s);
    std::vector<int> free_nib;
    for (int k = 0; k < 16; ++k)
        if (((pinned >> (4 * k)) & 0xF) != 0xF) free_nib.push_back(k);
    SortPlan sp;
    std::memset(&sp, 0, sizeof sp);
    sp.passes = (int)(free_nib.size() + 1) / 2;
    for (int p = 0; p < sp.passes; ++p) {
        sp.lo[p] = free_nib[2 * p];
        sp.hi[p] = 2 * p + 1 < (int)free_nib.size() ? free_nib[2 * p + 1] : -1;
    }
    return sp;
}

// ------------------------------------------------------------ forward -----

struct ForwardPlan {
    int steps, docheck, first_step;  // first_step: generation starts at step i = first_step
    DevSpec spec;
    SortPlan sort;
    long long s0;      // tile sum of layer 0; layer t has tile sum s0 + 2t
    FreeNibbles free;  // nibbles that vary between keys
};

// The expand and solve kernels come in two builds: with the variant boards'
// symmetry modes (min33/min24/min34) and without; a table takes the one its
// mode needs, so the classic tables' kernels carry no variant code.
static auto expand_kernel_for(const DevSpec &spec) {
    return spec.symm >= 4 ? expand_dedup_kernel<true> : expand_dedup_kernel<false>;
}

template <typename T>
static auto solve_kernel_for(const DevSpec &spec) {
    return spec.symm >= 4 ? solve_kernel<T, true> : solve_kernel<T, false>;
}

// Enqueue forward steps first_step .. steps-2 (one fused expand + dedup
// kernel each) and close the last two layers. Preconditions on the device:
// layer first_step-1 in its staging buffer, layer first_step's keys so far in
// its staging buffer and set, layer_off[first_step-1] set.
static void enqueue_forward(Engine &E, const ForwardPlan &P, unsigned *progress) {
    cudaStream_t s = E.stream;
    const int g_exp = E.sm_count;  // one 1024-thread block per SM (the row table fills its shared memory)
    uint64_t *stage[3] = {E.cand[0], E.cand[1], E.tmp};
    const auto expand = expand_kernel_for(P.spec);
    const int pe = E.prof_begin(K_EXPAND, (unsigned long long)std::max(0, P.steps - 1 - P.first_step));
    for (int i = P.first_step; i < P.steps - 1; ++i) {
        const int t = i - 1;
        // consecutive steps overlap: the next step stages its row table while this one finishes
        launch_dependent(E, expand, g_exp, kExpandThreads, kRowSmemBytes, s, stage[t % 3], stage[(t + 1) % 3],
                         stage[(t + 2) % 3], t % 3, (t + 1) % 3, (t + 2) % 3, E.arena, E.layer_off, E.layer_len,
                         E.arena_cap, t, P.spec, i > P.docheck ? 1 : 0, (const uint32_t *)E.tab, E.dset[(t + 1) % 3],
                         E.dset[(t + 2) % 3], E.dset_cap - 1, E.cand_cap, E.filter, E.filter_bits, E.dset[t % 3],
                         E.ctl, progress, (unsigned)i);
    }
    E.prof_end(pe);
    for (int L = std::max(P.first_step, P.steps - 2); L < P.steps; ++L)
        EGTB_LAUNCH(E, flush_layer_kernel<<<E.sm_count * 2, 256, 0, s>>>(stage[L % 3], L % 3, E.arena, E.layer_off,
                                                                          E.layer_len, E.arena_cap, L, E.ctl));
}

static DevCtl read_ctl(Engine &E) {
    DevCtl c;
    EGTB_CUDA(cudaMemcpyAsync(&c, E.ctl, sizeof c, cudaMemcpyDeviceToHost, E.stream));
    EGTB_CUDA(cudaStreamSynchronize(E.stream));
    return c;
}

__global__ void set_u64_kernel(unsigned long long *p, unsigned long long v) { *p = v; }

// Reset control state and place the starting layers: layer first_step-1
// (`base`) and what is known of layer first_step (`partial`, also entered in
// that layer's set).
static void stage_start(Engine &E, const ForwardPlan &P, const uint64_t *base, size_t n_base, const uint64_t *partial,
                        size_t n_partial) {
    cudaStream_t s = E.stream;
    EGTB_CUDA(cudaMemsetAsync(E.ctl, 0, sizeof(DevCtl), s));
    EGTB_CUDA(cudaMemsetAsync(E.hist, 0, sizeof(unsigned) * kMaxPasses * 256, s));
    for (auto *d : E.dset) EGTB_CUDA(cudaMemsetAsync(d, 0, sizeof(uint64_t) * E.dset_cap, s));
    EGTB_CUDA(cudaMemsetAsync(E.filter, 0, sizeof(uint64_t) << E.filter_bits, s));
    EGTB_CUDA(cudaMemsetAsync(E.layer_off, 0, sizeof(unsigned long long) * E.steps_cap, s));
    EGTB_CUDA(cudaMemsetAsync(E.layer_len, 0, sizeof(unsigned long long) * E.steps_cap, s));
    if (n_base > E.cand_cap || n_partial > E.cand_cap)
        throw Error(EGTB_ERR_CAPACITY, "start layer larger than the staging buffers");
    uint64_t *stage[3] = {E.cand[0], E.cand[1], E.tmp};
    const int t0 = P.first_step - 1, t1 = P.first_step;
    if (n_base) EGTB_CUDA(cudaMemcpyAsync(stage[t0 % 3], base, sizeof(uint64_t) * n_base, cudaMemcpyHostToDevice, s));
    EGTB_LAUNCH(E, set_u64_kernel<<<1, 1, 0, s>>>(&E.ctl->stage_count[t0 % 3], (unsigned long long)n_base));
    if (n_partial) {
        EGTB_CUDA(cudaMemcpyAsync(stage[t1 % 3], partial, sizeof(uint64_t) * n_partial, cudaMemcpyHostToDevice, s));
        EGTB_LAUNCH(E, set_u64_kernel<<<1, 1, 0, s>>>(&E.ctl->stage_count[t1 % 3], (unsigned long long)n_partial));
        EGTB_LAUNCH(E, dedup_seed_kernel<<<E.sm_count * 4, 256, 0, s>>>(stage[t1 % 3], n_partial, E.dset[t1 % 3],
                                                                          E.dset_cap - 1, E.ctl));
    }
    // the host buffers above may be pageable: finish the copies before returning
    EGTB_CUDA(cudaStreamSynchronize(s));
}

static unsigned long long env_keys(const char *name, unsigned long long dflt) {
    const char *v = getenv(name);
    if (!v || !*v) return dflt;
    const unsigned long long x = strtoull(v, nullptr, 10);
    return x ? x : dflt;
}

// Sort layers 1 .. steps-1 in place (layer 0 keeps the seeds' order), each in
// its own arena region by its free nibbles: one digit-histogram kernel for
// every layer and pass, then one segmented onesweep kernel per pass (tiles
// aligned to layers), ping-ponging with the book buffer, which is free until
// the solve. len: host copy of the layer lengths.
static void enqueue_sort_layers(Engine &E, const ForwardPlan &P, const std::vector<unsigned long long> &len) {
    cudaStream_t s = E.stream;
    const int steps = P.steps;
    if (steps < 2) return;
    // layers 1..steps-1 (layer 0 keeps the seeds as given), each sorted in its own
    // arena region by its free nibbles: tiles never straddle two layers
    std::vector<int> tab;
    std::vector<int> tile0(steps, 0);
    for (int L = 1; L < steps; ++L) {
        tile0[L] = (int)tab.size();
        const unsigned long long nt = (len[L] + kTileKeys - 1) / kTileKeys;
        for (unsigned long long j = 0; j < nt; ++j) tab.push_back(L);
    }
    const unsigned ntiles = (unsigned)tab.size();
    if (ntiles == 0) return;
    tab.reserve(tab.size() + tile0.size());
    for (const int v : tile0) tab.push_back(v);
    E.ensure_seg(ntiles, (unsigned long long)steps);
    EGTB_CUDA(cudaMemcpyAsync(E.seg_tab, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, s));
    const int *tile_layer = E.seg_tab, *layer_tile0 = E.seg_tab + ntiles;
    // digit positions of every pass (two free nibbles each), the same for every layer
    const int F = P.free.count;
    const int passes = (F + 1) / 2;
    std::vector<unsigned short> nib((size_t)steps * kMaxPasses, 0xFFFFu);
    for (int L = 0; L < steps; ++L)
        for (int q = 0; q < passes; ++q)
            nib[(size_t)L * kMaxPasses + q] =
                (unsigned short)(P.free.idx[2 * q] | ((2 * q + 1 < F ? P.free.idx[2 * q + 1] : 0xFF) << 8));
    unsigned short *seg_nib = reinterpret_cast<unsigned short *>(E.seg_hist + (size_t)steps * kMaxPasses * 256);
    EGTB_CUDA(cudaMemcpyAsync(seg_nib, nib.data(), sizeof(unsigned short) * nib.size(), cudaMemcpyHostToDevice, s));
    const int pu = E.prof_begin(K_UNIQUE);
    EGTB_CUDA(cudaMemsetAsync(E.seg_hist, 0, sizeof(unsigned) * (size_t)steps * kMaxPasses * 256, s));
    EGTB_LAUNCH(E, seg_hist_kernel<<<E.sm_count * 2, kHistThreads, 0, s>>>(E.arena, tile_layer, layer_tile0, E.layer_off,
                                                                         E.layer_len, ntiles, passes, seg_nib,
                                                                         E.seg_hist, E.counters));
    uint64_t *src = E.arena, *dst = (uint64_t *)E.book;  // the book buffer is free until the solve
    for (int q = 0; q < passes; ++q) {
        const int pi = E.prof_begin(K_SORT_PASS);
        EGTB_LAUNCH(E, seg_onesweep_kernel<<<E.seg_grid, kSweepThreads, kSegSweepSmem, s>>>(
                           src, dst, tile_layer, layer_tile0, E.layer_off, E.layer_len, ntiles, seg_nib, q, E.seg_hist,
                           E.counters, E.status, E.epoch++, E.ctl, look_back_spin_limit()));
        E.prof_end(pi);
        std::swap(src, dst);
    }
    if (src != E.arena)
        EGTB_LAUNCH(E, seg_copy_kernel<<<E.sm_count * 8, 256, 0, s>>>(src, E.arena, tile_layer, layer_tile0, E.layer_off,
                                                                     E.layer_len, ntiles));
    E.prof_end(pu);
}

// Run the forward with capacity regrowth, then sort the layers. Returns the
// number of retries.
static int run_forward(Engine &E, const ForwardPlan &P, const uint64_t *base, size_t n_base, const uint64_t *partial,
                       size_t n_partial, float *ms) {
    int retries = 0;
    E.ensure_steps(P.steps);
    // first capacities: 4 Mi keys per staging buffer, 128 Mi layer keys, 1 Mi
    // slots per dedup set (small sets stay in L2) (EGTB_INIT_CAND_KEYS / EGTB_INIT_ARENA_KEYS /
    // EGTB_INIT_SET_SLOTS override); a pass that outgrows them is re-run larger
    static const unsigned long long init_cand = env_keys("EGTB_INIT_CAND_KEYS", 1ull << 22);
    static const unsigned long long init_arena = env_keys("EGTB_INIT_ARENA_KEYS", 1ull << 27);
    static const unsigned long long init_set = env_keys("EGTB_INIT_SET_SLOTS", 1ull << 20);
    E.ensure_cand(std::max<unsigned long long>(E.cand_cap, std::max<unsigned long long>(init_cand,
                                                                                         2 * std::max(n_partial, n_base))));
    E.ensure_arena(std::max<unsigned long long>(E.arena_cap, std::max<unsigned long long>(init_arena, n_base * 4)));
    unsigned long long set_need = init_set;
    while (set_need < 4 * std::max<unsigned long long>(n_partial, 1)) set_need <<= 1;
    E.ensure_dedup(std::max(E.dset_cap, set_need));
    unsigned *progress = progress_device_ptr();
    for (;;) {
        stage_start(E, P, base, n_base, partial, n_partial);
        EGTB_CUDA(cudaEventRecord(E.ev[0], E.stream));
        enqueue_forward(E, P, progress);
        DevCtl c = read_ctl(E);
        EGTB_CUDA(cudaGetLastError());
        E.prof_resolve();
        if (c.err == 0) {
            std::vector<unsigned long long> len(P.steps + 1);
            EGTB_CUDA(cudaMemcpy(len.data(), E.layer_len, sizeof(unsigned long long) * (P.steps + 1),
                                 cudaMemcpyDeviceToHost));
            E.candidates = c.candidates;
            enqueue_sort_layers(E, P, len);
            EGTB_CUDA(cudaEventRecord(E.ev[1], E.stream));
            DevCtl c2 = read_ctl(E);
            EGTB_CUDA(cudaGetLastError());
            E.prof_resolve();
            if (c2.err & kErrTimeout) throw Error(EGTB_ERR_TIMEOUT, "a bounded device wait gave up in the layer sort");
            EGTB_CUDA(cudaEventElapsedTime(ms, E.ev[0], E.ev[1]));
            return retries;
        }
        if (c.err & kErrTimeout) throw Error(EGTB_ERR_TIMEOUT, "a bounded device wait gave up in the forward pass");
        ++retries;
        if (retries > 24) throw Error(EGTB_ERR_CAPACITY, "forward pass did not fit after repeated regrowth");
        if (c.err & kErrCandOverflow) E.ensure_cand(E.cand_cap * 2);
        if (c.err & kErrArenaOverflow) E.ensure_arena(E.arena_cap + E.arena_cap / 2);
        if (c.err & kErrDedupOverflow) E.ensure_dedup(E.dset_cap * 2);
    }
}

// ------------------------------------------------------ streamed forward --
//
// Forward pass for tables larger than device memory: after step t expands
// layer t, the layer (unique keys in its staging buffer) is radix-sorted on
// the device, and while step t+1 runs it is copied on a second stream into
// one of two pinned host buffers and written to the raw layer file
// <pathname><t> by a host thread. The device holds the window of layers t..t+2
// (staging buffers, dedup sets, two sort buffers) instead of the whole table.
// The last two layers end sorted in the arena for the success-only books.

static bool stream_layers_forced() {
    const char *v = getenv("EGTB_STREAM_LAYERS");
    return v && *v && std::strcmp(v, "0") != 0;
}

// Enqueue the sort of the n (*n_ptr, on the device) unique keys at src;
// returns the buffer that holds them sorted.
static uint64_t *enqueue_layer_sort(Engine &E, const SortPlan &sp, const uint64_t *src,
                                    const unsigned long long *n_ptr) {
    cudaStream_t s = E.stream;
    EGTB_CUDA(cudaMemsetAsync(E.hist, 0, sizeof(unsigned) * kMaxPasses * 256, s));
    EGTB_LAUNCH(E, sort_hist_kernel<<<E.sm_count * 2, kHistThreads, 0, s>>>(src, n_ptr, E.sort_cap, sp, E.hist, E.counters,
                                                                   E.ctl));
    const uint64_t *in = src;
    uint64_t *out = E.sort_buf[0];
    for (int q = 0; q < sp.passes; ++q) {
        const int pi = E.prof_begin(K_SORT_PASS);
        EGTB_LAUNCH(E, onesweep_kernel<<<E.sweep_grid, kSweepThreads, 0, s>>>(in, out, n_ptr, E.sort_cap, sp, q, E.hist,
                                                                             E.counters, E.status, E.epoch++, E.ctl, look_back_spin_limit()));
        E.prof_end(pi);
        in = out;
        out = out == E.sort_buf[0] ? E.sort_buf[1] : E.sort_buf[0];
    }
    return const_cast<uint64_t *>(in);
}

// Returns the retries; off/len: the layers' arena offsets and lengths (only
// the last two layers are in the arena).
static int run_forward_streamed(Engine &E, const ForwardPlan &P, const uint64_t *base, size_t n_base,
                                const uint64_t *partial, size_t n_partial, const std::string &prefix, float *ms,
                                std::vector<unsigned long long> &off, std::vector<unsigned long long> &len) {
    int retries = 0;
    E.ensure_steps(P.steps);
    // streamed tables are large: start at 16 Mi keys per layer buffer and
    // grow 4x, since an overflow re-runs the pass from its first step
    static const unsigned long long init_cand = env_keys("EGTB_INIT_CAND_KEYS", 1ull << 24);
    static const unsigned long long init_set = env_keys("EGTB_INIT_SET_SLOTS", 1ull << 23);
    E.ensure_cand(std::max<unsigned long long>(E.cand_cap, std::max<unsigned long long>(init_cand,
                                                                                         2 * std::max(n_partial, n_base))));
    unsigned long long set_need = init_set;
    while (set_need < 4 * std::max<unsigned long long>(n_partial, 1)) set_need <<= 1;
    E.ensure_dedup(std::max(E.dset_cap, set_need));
    unsigned *progress = progress_device_ptr();
    cudaStream_t s = E.stream;
    const int steps = P.steps;
    struct Small {
        unsigned long long n;
        DevCtl ctl;
    };
    Small *hs = nullptr;
    EGTB_CUDA(cudaHostAlloc((void **)&hs, sizeof(Small), cudaHostAllocDefault));
    std::unique_ptr<Small, void (*)(Small *)> hs_guard(hs, [](Small *q) { cudaFreeHost(q); });
    cudaEvent_t ev_buf[2];
    for (auto &e : ev_buf) EGTB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    std::unique_ptr<cudaEvent_t, void (*)(cudaEvent_t *)> ev_guard(ev_buf, [](cudaEvent_t *e) {
        cudaEventDestroy(e[0]);
        cudaEventDestroy(e[1]);
    });
    for (;;) {
        E.ensure_sort_bufs(E.cand_cap);
        E.ensure_status();
        stage_start(E, P, base, n_base, partial, n_partial);
        unsigned char *pin = E.ensure_pinned(2 * E.cand_cap * sizeof(uint64_t));
        std::future<void> writer[2];
        std::string write_error;
        std::mutex write_mu;
        uint64_t *stage[3] = {E.cand[0], E.cand[1], E.tmp};
        len.assign(steps + 1, 0);
        unsigned long long sorted_keys = 0;
        unsigned err = 0;
        int pending = -1;
        uint64_t *pending_buf = nullptr;
        bool copied_any = false;
        EGTB_CUDA(cudaEventRecord(E.ev[0], s));
        // ship layer t: its length, then the copy into pinned buffer t % 2 and the file write
        auto ship = [&](int t, uint64_t *sorted) {
            EGTB_CUDA(cudaEventSynchronize(E.ev_sorted));
            err |= hs->ctl.err;
            if (err) return;
            const unsigned long long n = hs->n;
            len[t] = n;
            sorted_keys += n;
            const int b = t & 1;
            if (writer[b].valid()) writer[b].get();
            unsigned char *dst = pin + (size_t)b * E.cand_cap * sizeof(uint64_t);
            EGTB_CUDA(cudaStreamWaitEvent(E.copy_stream, E.ev_sorted, 0));
            if (n) EGTB_CUDA(cudaMemcpyAsync(dst, sorted, n * 8, cudaMemcpyDeviceToHost, E.copy_stream));
            EGTB_CUDA(cudaEventRecord(ev_buf[b], E.copy_stream));
            EGTB_CUDA(cudaEventRecord(E.ev_copied, E.copy_stream));
            copied_any = true;
            const std::string path = prefix + std::to_string(t);
            cudaEvent_t done = ev_buf[b];
            const int dev = E.device;
            writer[b] = std::async(std::launch::async, [=, &write_error, &write_mu] {
                try {
                    EGTB_CUDA(cudaSetDevice(dev));
                    EGTB_CUDA(cudaEventSynchronize(done));
                    write_file(path, dst, n * 8);
                } catch (const std::exception &e) {
                    std::lock_guard<std::mutex> lk(write_mu);
                    write_error = e.what();
                }
            });
        };
        const auto expand = expand_kernel_for(P.spec);
        for (int i = P.first_step; i < steps - 1 && !err; ++i) {
            const int t = i - 1;
            const int pe = E.prof_begin(K_EXPAND);
            EGTB_LAUNCH(E, expand<<<E.sm_count, kExpandThreads, kRowSmemBytes, s>>>(
                               stage[t % 3], stage[(t + 1) % 3], stage[(t + 2) % 3], t % 3, (t + 1) % 3, (t + 2) % 3,
                               nullptr, E.layer_off, E.layer_len, 0, t, P.spec, i > P.docheck ? 1 : 0, E.tab,
                               E.dset[(t + 1) % 3], E.dset[(t + 2) % 3], E.dset_cap - 1, E.cand_cap, E.filter,
                               E.filter_bits, E.dset[t % 3], E.ctl, progress, (unsigned)i));
            E.prof_end(pe);
            if (pending >= 0) {  // ship the layer sorted last step while this step runs
                ship(pending, pending_buf);
                pending = -1;
            }
            if (t >= P.first_step && t <= steps - 3) {
                if (copied_any) EGTB_CUDA(cudaStreamWaitEvent(s, E.ev_copied, 0));  // sort buffers are free again
                pending_buf = enqueue_layer_sort(E, P.sort, stage[t % 3], E.layer_len + t);
                EGTB_CUDA(cudaMemcpyAsync(&hs->n, E.layer_len + t, 8, cudaMemcpyDeviceToHost, s));
                EGTB_CUDA(cudaMemcpyAsync(&hs->ctl, E.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
                EGTB_CUDA(cudaEventRecord(E.ev_sorted, s));
                pending = t;
            }
        }
        if (pending >= 0 && !err) ship(pending, pending_buf);
        for (auto &w : writer)
            if (w.valid()) w.get();
        if (!write_error.empty()) throw Error(EGTB_ERR_IO, write_error);
        EGTB_CUDA(cudaStreamSynchronize(E.copy_stream));
        DevCtl c = read_ctl(E);
        err |= c.err;
        if (err == 0) {
            // the last two layers: sorted into the arena for the final books
            off.assign(steps + 1, 0);
            std::vector<unsigned long long> nl(2, 0);
            for (int k = 0; k < 2; ++k) nl[k] = c.stage_count[(steps - 2 + k) % 3];
            E.ensure_arena(align16(nl[0]) + nl[1] + 16);
            unsigned long long at = 0;
            for (int k = 0; k < 2; ++k) {
                const int L = steps - 2 + k;
                off[L] = at;
                len[L] = nl[k];
                if (nl[k]) {
                    uint64_t *sorted = enqueue_layer_sort(E, P.sort, stage[L % 3], &E.ctl->stage_count[L % 3]);
                    EGTB_CUDA(cudaMemcpyAsync(E.arena + at, sorted, nl[k] * 8, cudaMemcpyDeviceToDevice, s));
                    sorted_keys += nl[k];
                }
                at += align16(nl[k]);
            }
            EGTB_CUDA(cudaMemcpyAsync(E.layer_off, off.data(), sizeof(unsigned long long) * (steps + 1),
                                      cudaMemcpyHostToDevice, s));
            EGTB_CUDA(cudaMemcpyAsync(E.layer_len, len.data(), sizeof(unsigned long long) * (steps + 1),
                                      cudaMemcpyHostToDevice, s));
            EGTB_CUDA(cudaEventRecord(E.ev[1], s));
            DevCtl c2 = read_ctl(E);
            E.prof_resolve();
            if (c2.err & kErrTimeout) throw Error(EGTB_ERR_TIMEOUT, "a bounded device wait gave up in a layer sort");
            E.candidates = c2.candidates - sorted_keys;  // the sorts' histogram pass counts its keys too
            EGTB_CUDA(cudaEventElapsedTime(ms, E.ev[0], E.ev[1]));
            return retries;
        }
        E.prof_resolve();
        if (err & kErrTimeout) throw Error(EGTB_ERR_TIMEOUT, "a bounded device wait gave up in the forward pass");
        ++retries;
        if (retries > 24) throw Error(EGTB_ERR_CAPACITY, "forward pass did not fit after repeated regrowth");
        if (err & kErrCandOverflow) E.ensure_cand(E.cand_cap * 4);
        if (err & kErrDedupOverflow) E.ensure_dedup(E.dset_cap * 4);
    }
}

// ----------------------------------------------------------- backward -----

static double ordered_to_double(unsigned long long o) {
    unsigned long long b = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    double d;
    std::memcpy(&d, &b, sizeof d);
    return d;
}

template <typename T>
__global__ void layer_max_kernel(const T *__restrict__ rates, const unsigned long long *__restrict__ layer_off,
                                 const unsigned long long *__restrict__ layer_len, int t, T zero,
                                 unsigned long long *__restrict__ out) {
    const unsigned long long n = layer_len[t], o = layer_off[t];
    double m = -INFINITY;
    bool any = false;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const T r = rates[o + i];
        if (r > zero) {
            any = true;
            const double d = (double)r;
            m = d > m ? d : m;
        }
    }
    unsigned long long b = any ? ordered_bits(m) : 0ull;
    for (int s = 16; s > 0; s >>= 1) {
        unsigned long long y = __shfl_xor_sync(0xFFFFFFFFu, b, s);
        b = y > b ? y : b;
    }
    if ((threadIdx.x & 31) == 0 && b) atomicMax(out + t, b);
}

__global__ void book_len_kernel(const unsigned long long *total, unsigned long long *book_len, int t) {
    book_len[t] = *total;
}

template <typename T>
static void enqueue_pack(Engine &E, int t, T zero) {
    cudaStream_t s = E.stream;
    const int g = E.sm_count * 4;
    EGTB_LAUNCH(E, book_count_kernel<T><<<g, kSortThreads, 0, s>>>((const T *)E.rates, E.layer_off, E.layer_len, t, zero, E.tile_cnt));
    EGTB_LAUNCH(E, tile_scan_kernel<<<1, 1024, 0, s>>>(E.layer_len + t, E.arena_cap, E.tile_off, E.tile_cnt, &E.ctl->n_unique));
    EGTB_LAUNCH(E, book_len_kernel<<<1, 1, 0, s>>>(&E.ctl->n_unique, E.book_len, t));
}

template <typename T>
static void enqueue_pack_write(Engine &E, int t, T zero, unsigned long long book_off_bytes) {
    const int g = E.sm_count * 4;
    EGTB_LAUNCH(E, book_write_kernel<T><<<g, kSortThreads, 0, E.stream>>>(E.arena, (const T *)E.rates, E.layer_off, E.layer_len, t, zero, E.tile_off, E.book, book_off_bytes, E.book_cap_bytes, E.ctl));
}

struct BackwardPlan {
    int steps, docheck, dtype;
    double p4;
    DevSpec spec;
};

// Slots of the rate index of a layer of n entries: a power of two >= 2n.
static unsigned long long index_slots(unsigned long long n) {
    unsigned long long c = 64;
    while (c < 2 * n) c <<= 1;
    return c;
}

// Build the rate index of layer L (live entries only) into idx.
template <typename T>
static void enqueue_index_at(Engine &E, int L, unsigned long long n, T zero, ulonglong2 *idx) {
    const unsigned long long slots = index_slots(n);
    EGTB_CUDA(cudaMemsetAsync(idx, 0, sizeof(ulonglong2) * slots, E.stream));
    EGTB_LAUNCH(E, index_insert_kernel<T><<<E.sm_count * 8, 256, 0, E.stream>>>(E.arena, (const T *)E.rates, E.layer_off,
                                                                             E.layer_len, L, zero, idx, slots - 1, E.ctl));
}

// ... in index L % 4 (fused build).
template <typename T>
static void enqueue_index(Engine &E, int L, unsigned long long n, T zero) {
    enqueue_index_at<T>(E, L, n, zero, E.index[L % 4]);
}

// Pack every layer's live entries as .book records in one pass; the book of
// layer t starts at byte layer_off[t] * rec of E.book.
template <typename T>
static void enqueue_pack_all(Engine &E, int steps, const std::vector<unsigned long long> &len, T zero) {
    cudaStream_t s = E.stream;
    std::vector<unsigned long long> ft(steps + 1, 0);
    for (int L = 0; L < steps; ++L) ft[L + 1] = ft[L] + (len[L] + kTileKeys - 1) / kTileKeys;
    const unsigned long long n_tiles = ft[steps];
    if (n_tiles > E.comp_tiles) throw Error(EGTB_ERR_CAPACITY, "tile buffers too small for packing");
    EGTB_CUDA(cudaMemcpyAsync(E.first_tile, ft.data(), sizeof(unsigned long long) * (steps + 1), cudaMemcpyHostToDevice, s));
    EGTB_CUDA(cudaMemsetAsync(E.layer_max, 0, sizeof(unsigned long long) * steps, s));
    const int g = E.sm_count * 4;
    EGTB_LAUNCH(E, book_count_all_kernel<T><<<g, kSortThreads, 0, s>>>((const T *)E.rates, E.layer_off, E.layer_len,
                                                                   E.first_tile, steps, n_tiles, zero, E.tile_cnt,
                                                                   E.layer_max));
    EGTB_LAUNCH(E, scan_tiles_kernel<<<1, 1024, 0, s>>>(E.tile_cnt, n_tiles, E.tile_off, &E.ctl->n_unique));
    EGTB_LAUNCH(E, book_lens_kernel<<<(steps + 255) / 256, 256, 0, s>>>(E.first_tile, steps, n_tiles, E.tile_off,
                                                                       &E.ctl->n_unique, E.book_len));
    EGTB_LAUNCH(E, book_write_all_kernel<T><<<g, kSortThreads, 0, s>>>(E.arena, (const T *)E.rates, E.layer_off,
                                                                   E.layer_len, E.first_tile, steps, n_tiles, zero,
                                                                   E.tile_off, E.book, E.book_cap_bytes, E.ctl));
}

// Pack the books of layers l0 .. l1-1 (the same kernels over a range of layers).
template <typename T>
static void enqueue_pack_range(Engine &E, int l0, int l1, const std::vector<unsigned long long> &len, T zero,
                               cudaStream_t s) {
    const int nl = l1 - l0;
    std::vector<unsigned long long> ft(nl + 1, 0);
    for (int k = 0; k < nl; ++k) ft[k + 1] = ft[k] + (len[l0 + k] + kTileKeys - 1) / kTileKeys;
    const unsigned long long n_tiles = ft[nl];
    if (n_tiles > E.comp_tiles) throw Error(EGTB_ERR_CAPACITY, "tile buffers too small for packing");
    // stream-ordered after the previous range's kernels, which read the same buffer
    EGTB_CUDA(cudaMemcpyAsync(E.first_tile, ft.data(), sizeof(unsigned long long) * (nl + 1), cudaMemcpyHostToDevice, s));
    const int g = E.sm_count * 4;
    EGTB_LAUNCH(E, book_count_all_kernel<T><<<g, kSortThreads, 0, s>>>((const T *)E.rates, E.layer_off + l0,
                                                                   E.layer_len + l0, E.first_tile, nl, n_tiles, zero,
                                                                   E.tile_cnt, E.layer_max + l0));
    EGTB_LAUNCH(E, scan_tiles_kernel<<<1, 1024, 0, s>>>(E.tile_cnt, n_tiles, E.tile_off, &E.ctl->n_unique));
    EGTB_LAUNCH(E, book_lens_kernel<<<(nl + 255) / 256, 256, 0, s>>>(E.first_tile, nl, n_tiles, E.tile_off,
                                                                    &E.ctl->n_unique, E.book_len + l0));
    EGTB_LAUNCH(E, book_write_all_kernel<T><<<g, kSortThreads, 0, s>>>(E.arena, (const T *)E.rates, E.layer_off + l0,
                                                                   E.layer_len + l0, E.first_tile, nl, n_tiles, zero,
                                                                   E.tile_off, E.book, E.book_cap_bytes, E.ctl));
}

// Solve every layer on the device-resident arena (layers 0..steps-1 present)
// and pack all books.
template <typename T>
static void enqueue_backward(Engine &E, const BackwardPlan &B, const std::vector<unsigned long long> &len,
                             unsigned *progress) {
    cudaStream_t s = E.stream;
    const T zero = (T)dtype_zero(B.dtype), maxv = (T)dtype_max(B.dtype);
    const int g = E.sm_count * 8;
    T *rates = (T *)E.rates;
    const uint32_t total = (uint32_t)(B.steps * 2);
    unsigned long long biggest = 0;
    for (int L = 0; L < B.steps; ++L) biggest = std::max(biggest, len[L]);
    E.ensure_index(index_slots(biggest));
    const int pf = E.prof_begin(K_FINAL);
    for (int t = B.steps - 2; t < B.steps; ++t)
        if (t >= 0) EGTB_LAUNCH(E, final_layer_kernel<T><<<g, 256, 0, s>>>(E.arena, rates, E.layer_off, E.layer_len, t, B.spec, zero, maxv));
    for (int t = B.steps - 1; t >= B.steps - 2 && t >= 1; --t) enqueue_index<T>(E, t, len[t], zero);
    // the solve of layer t reads the indexes of t+1 and t+2, fills layer t's
    // (L % 4, cleared by the launch before) and clears the one of layer t-1
    if (B.steps - 3 >= 1)
        EGTB_CUDA(cudaMemsetAsync(E.index[(B.steps - 3) % 4], 0, sizeof(ulonglong2) * index_slots(len[B.steps - 3]), s));
    E.prof_end(pf);
    const int ps = E.prof_begin(K_SOLVE, (unsigned long long)std::max(0, B.steps - 2));
    for (int t = B.steps - 3; t >= 0; --t) {
        ulonglong2 *idx0 = t >= 1 ? E.index[t % 4] : nullptr;
        ulonglong2 *clear = t >= 2 ? E.index[(t - 1) % 4] : nullptr;
        // consecutive solves overlap: each launch starts as the one before finishes
        launch_dependent(E, solve_kernel_for<T>(B.spec), g, 256, 0, s, (const uint64_t *)E.arena, rates,
                         (const unsigned long long *)E.layer_off, (const unsigned long long *)E.layer_len, t, B.spec,
                         t > B.docheck ? 1 : 0, (const uint32_t *)E.tab, B.p4, zero, maxv,
                         (const ulonglong2 *)E.index[(t + 1) % 4], index_slots(len[t + 1]) - 1,
                         (const ulonglong2 *)E.index[(t + 2) % 4], index_slots(len[t + 2]) - 1, E.ctl, idx0,
                         index_slots(len[t]) - 1, clear, t >= 2 ? index_slots(len[t - 1]) : 0ull, progress,
                         total - (unsigned)t - 2u);
    }
    E.prof_end(ps);
    const int pp = E.prof_begin(K_PACK);
    enqueue_pack_all<T>(E, B.steps, len, zero);
    E.prof_end(pp);
}

static int writer_threads(const egtb_run_options &o);

// The same solve, with the books packed in groups of layers as the solve
// finishes them: while the device solves the next layers, a pack stream packs
// each finished group, the host copies it (copy stream) into pinned memory and
// writer threads write its .book files. Returns the book lengths and rate
// maxima.
template <typename T>
static void backward_write_books(Engine &E, const BackwardPlan &B, const std::vector<unsigned long long> &len,
                                 const std::vector<unsigned long long> &off, const egtb_run_options &o,
                                 std::vector<unsigned long long> &blen, std::vector<unsigned long long> &maxb,
                                 float *bwd_ms) {
    cudaStream_t s = E.stream;
    const int steps = B.steps;
    const T zero = (T)dtype_zero(B.dtype), maxv = (T)dtype_max(B.dtype);
    const int g = E.sm_count * 8;
    T *rates = (T *)E.rates;
    const uint32_t total = (uint32_t)(steps * 2);
    unsigned *progress = progress_device_ptr();
    const size_t rec = 8 + sizeof(T);
    unsigned long long biggest = 0, raw_total = 0;
    for (int L = 0; L < steps; ++L) {
        biggest = std::max(biggest, len[L]);
        raw_total += len[L];
    }
    E.ensure_index(index_slots(biggest));
    E.ensure_copy_stream();
    struct Group {
        int l0, l1;
        cudaEvent_t solved, packed;
    };
    std::vector<Group> groups;
    struct GroupGuard {
        std::vector<Group> &v;
        ~GroupGuard() {
            for (auto &q : v) {
                cudaEventDestroy(q.solved);
                cudaEventDestroy(q.packed);
            }
        }
    } gguard{groups};
    // a group's layers are solved once the build stream reaches this point;
    // they are packed on the pack stream while the solve goes on (the packing
    // reads only their rates and writes only their book regions)
    auto close_group = [&](int l0, int l1) {
        Group q{l0, l1, nullptr, nullptr};
        EGTB_CUDA(cudaEventCreateWithFlags(&q.solved, cudaEventDisableTiming));
        EGTB_CUDA(cudaEventCreateWithFlags(&q.packed, cudaEventDisableTiming));
        groups.push_back(q);
        EGTB_CUDA(cudaEventRecord(q.solved, s));
        EGTB_CUDA(cudaStreamWaitEvent(E.pack_stream, q.solved, 0));
        enqueue_pack_range<T>(E, l0, l1, len, zero, E.pack_stream);
        EGTB_CUDA(cudaEventRecord(q.packed, E.pack_stream));
    };
    EGTB_CUDA(cudaEventRecord(E.ev[2], s));
    EGTB_CUDA(cudaMemsetAsync(E.layer_max, 0, sizeof(unsigned long long) * steps, s));
    const int pf = E.prof_begin(K_FINAL);
    for (int t = steps - 2; t < steps; ++t)
        if (t >= 0) EGTB_LAUNCH(E, final_layer_kernel<T><<<g, 256, 0, s>>>(E.arena, rates, E.layer_off, E.layer_len, t, B.spec, zero, maxv));
    for (int t = steps - 1; t >= steps - 2 && t >= 1; --t) enqueue_index<T>(E, t, len[t], zero);
    if (steps - 3 >= 1)
        EGTB_CUDA(cudaMemsetAsync(E.index[(steps - 3) % 4], 0, sizeof(ulonglong2) * index_slots(len[steps - 3]), s));
    E.prof_end(pf);
    close_group(std::max(0, steps - 2), steps);
    constexpr int kGroup = 16;  // layers per packed group
    int hi = steps - 2;         // the current group is [t, hi)
    for (int t = steps - 3; t >= 0; --t) {
        const int ps = E.prof_begin(K_SOLVE);
        ulonglong2 *idx0 = t >= 1 ? E.index[t % 4] : nullptr;
        ulonglong2 *clear = t >= 2 ? E.index[(t - 1) % 4] : nullptr;
        // consecutive solves overlap: each launch starts as the one before finishes
        launch_dependent(E, solve_kernel_for<T>(B.spec), g, 256, 0, s, (const uint64_t *)E.arena, rates,
                         (const unsigned long long *)E.layer_off, (const unsigned long long *)E.layer_len, t, B.spec,
                         t > B.docheck ? 1 : 0, (const uint32_t *)E.tab, B.p4, zero, maxv,
                         (const ulonglong2 *)E.index[(t + 1) % 4], index_slots(len[t + 1]) - 1,
                         (const ulonglong2 *)E.index[(t + 2) % 4], index_slots(len[t + 2]) - 1, E.ctl, idx0,
                         index_slots(len[t]) - 1, clear, t >= 2 ? index_slots(len[t - 1]) : 0ull, progress,
                         total - (unsigned)t - 2u);
        E.prof_end(ps);
        if (hi - t == kGroup || t == 0) {
            close_group(t, hi);
            hi = t;
        }
    }
    EGTB_CUDA(cudaEventRecord(E.ev[3], s));
    // copy and write each group as soon as it is packed
    blen.assign(steps, 0);
    maxb.assign(steps, 0);
    unsigned char *pin = E.ensure_pinned(std::max<unsigned long long>(raw_total * rec, 1));
    std::vector<cudaEvent_t> copied;
    struct EventGuard {
        std::vector<cudaEvent_t> &v;
        ~EventGuard() {
            for (auto e : v) cudaEventDestroy(e);
        }
    } cguard{copied};
    WriterPool pool(writer_threads(o));
    unsigned long long pos = 0;
    for (const Group &q : groups) {
        const int nl = q.l1 - q.l0;
        EGTB_CUDA(cudaStreamWaitEvent(E.copy_stream, q.packed, 0));
        EGTB_CUDA(cudaMemcpyAsync(blen.data() + q.l0, E.book_len + q.l0, sizeof(unsigned long long) * nl,
                                  cudaMemcpyDeviceToHost, E.copy_stream));
        EGTB_CUDA(cudaMemcpyAsync(maxb.data() + q.l0, E.layer_max + q.l0, sizeof(unsigned long long) * nl,
                                  cudaMemcpyDeviceToHost, E.copy_stream));
        EGTB_CUDA(cudaStreamSynchronize(E.copy_stream));
        cudaEvent_t ev;
        EGTB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        copied.push_back(ev);
        std::vector<std::pair<int, unsigned long long>> at;
        for (int L = q.l0; L < q.l1; ++L) {
            const unsigned long long bytes = blen[L] * rec;
            if (pos + bytes > E.pinned_cap) throw Error(EGTB_ERR_CAPACITY, "book larger than its raw layer");
            if (bytes)
                EGTB_CUDA(cudaMemcpyAsync(pin + pos, E.book + off[L] * rec, bytes, cudaMemcpyDeviceToHost,
                                          E.copy_stream));
            at.push_back({L, pos});
            pos += bytes;
        }
        EGTB_CUDA(cudaEventRecord(ev, E.copy_stream));
        for (const auto &a : at)
            pool.submit(std::string(o.pathname) + std::to_string(a.first) + ".book", pin + a.second,
                        blen[a.first] * rec, ev, E.device);
    }
    pool.wait();
    EGTB_CUDA(cudaStreamSynchronize(E.copy_stream));
    EGTB_CUDA(cudaStreamSynchronize(E.pack_stream));
    EGTB_CUDA(cudaStreamSynchronize(s));
    EGTB_CUDA(cudaGetLastError());
    EGTB_CUDA(cudaEventElapsedTime(bwd_ms, E.ev[2], E.ev[3]));
}

// ---------------------------------------------------------------- output --

static std::vector<unsigned long long> d2h_u64(Engine &E, const unsigned long long *d, int n) {
    std::vector<unsigned long long> h(n);
    EGTB_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, E.stream));
    EGTB_CUDA(cudaStreamSynchronize(E.stream));
    return h;
}

// stats.txt lines, ensure_stats_header + recalculate_process_impl,
// native_core/src/BookSolver.cpp:286-293,569-581 (layers in solve order).
static void write_stats(const egtb_run_options &o, int dtype, const std::vector<int> &layers,
                        const std::vector<unsigned long long> &raw_len, const std::vector<unsigned long long> &book_len,
                        const std::vector<unsigned long long> &maxbits, double seconds_per_layer) {
    const std::string path = std::string(o.pathname) + "stats.txt";
    const bool exists = file_exists(path);
    std::ofstream f(path, std::ios::app);
    if (!f) throw Error(EGTB_ERR_IO, "cannot open " + path);
    if (!exists) f << "layer,length,max success rate,speed,deletion_threshold,time\n";
    const double zero = dtype_zero(dtype), maxs = dtype_max(dtype);
    for (int t : layers) {
        if (book_len[t] == 0) continue;
        const double m = maxbits[t] ? ordered_to_double(maxbits[t]) : zero;
        const double max_success = (m - zero) / (maxs - zero);
        f << t << "," << raw_len[t] << "," << max_success << ","
          << round_to_2((double)raw_len[t] / std::max(seconds_per_layer, 0.01) / 1e6) << " mbps,"
          << o.deletion_threshold << "," << now_string() << "\n";
    }
}

static int writer_threads(const egtb_run_options &o) {
    if (o.num_threads > 0) return std::min(o.num_threads, 32);
    return 8;
}

// Copy byte ranges [dev_off[i], +bytes[i]) of a device buffer to pinned host
// memory and write them to files with a thread pool; the copies go out in
// groups of about 16 MB, and a group's files are written as soon as its copy
// has landed, while the next groups are still crossing PCIe.
static void write_ranges(Engine &E, const unsigned char *dev, const std::vector<std::string> &paths,
                         const std::vector<unsigned long long> &dev_off, const std::vector<unsigned long long> &bytes,
                         int threads) {
    unsigned long long total = 0;
    for (auto b : bytes) total += b;
    unsigned char *h = E.ensure_pinned(std::max<unsigned long long>(total, 1));
    std::vector<cudaEvent_t> events;
    struct EventGuard {
        std::vector<cudaEvent_t> &v;
        ~EventGuard() {
            for (auto e : v) cudaEventDestroy(e);
        }
    } guard{events};
    WriterPool pool(threads);
    unsigned long long pos = 0, group = 0;
    size_t first = 0;
    for (size_t i = 0; i < paths.size(); ++i) {
        if (bytes[i])
            EGTB_CUDA(cudaMemcpyAsync(h + pos, dev + dev_off[i], bytes[i], cudaMemcpyDeviceToHost, E.stream));
        pos += bytes[i];
        group += bytes[i];
        if (group >= (16ull << 20) || i + 1 == paths.size()) {
            cudaEvent_t ev;
            EGTB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            events.push_back(ev);
            EGTB_CUDA(cudaEventRecord(ev, E.stream));
            unsigned long long at = pos - group;
            for (size_t k = first; k <= i; ++k) {
                pool.submit(paths[k], h + at, bytes[k], ev, E.device);
                at += bytes[k];
            }
            first = i + 1;
            group = 0;
        }
    }
    pool.wait();
    EGTB_CUDA(cudaStreamSynchronize(E.stream));
}

// ------------------------------------------------------------- restart ----

static bool any_layer_file(const egtb_run_options &o) {
    // one pass over the directory instead of five stat() calls per layer (a
    // fresh 304-step build otherwise spends ~2 ms in 1525 failed lookups)
    const std::string p = o.pathname;
    const size_t slash = p.find_last_of('/');
    const std::string dir = slash == std::string::npos ? "." : (slash == 0 ? "/" : p.substr(0, slash));
    const std::string stem = slash == std::string::npos ? p : p.substr(slash + 1);
    DIR *dp = opendir(dir.c_str());
    if (!dp) return false;
    bool found = false;
    for (struct dirent *e = readdir(dp); e && !found; e = readdir(dp)) {
        const char *name = e->d_name;
        if (std::strncmp(name, stem.c_str(), stem.size()) != 0) continue;
        // <stem><i> with i in 0..steps, alone or with one of the suffixes
        const char *q = name + stem.size();
        if (*q < '0' || *q > '9') continue;
        char *end = nullptr;
        const unsigned long long i = std::strtoull(q, &end, 10);
        if (i > (unsigned long long)o.steps || (q[0] == '0' && end != q + 1)) continue;
        const std::string suffix = end;
        found = suffix.empty() || suffix == ".book" || suffix == ".z" || suffix == ".book.7z" || suffix == ".7z";
    }
    closedir(dp);
    return found;
}

// handle_restart, native_core/src/BookGenerator.cpp:384-430: the first step
// that is not already on disk. Invalid files (empty or misaligned) are removed
// on the way, as the reference does.
static int first_step_to_run(const egtb_run_options &o, int rec) {
    const std::string p = o.pathname;
    for (int i = 1; i < o.steps - 1; ++i) {
        const std::string pi = p + std::to_string(i), pi1 = p + std::to_string(i + 1);
        remove_invalid(pi, 8);
        remove_invalid(pi1, 8);
        remove_invalid(pi + ".book", rec);
        remove_invalid(pi1 + ".book", rec);
        remove_invalid(pi + ".z", 0);
        remove_invalid(pi + ".book.7z", 0);
        remove_invalid(pi + ".7z", 0);
        remove_invalid(pi1 + ".z", 0);
        const bool skip = (file_valid(pi1, 8) && file_valid(pi, 8)) || (file_valid(pi1 + ".book", rec) && file_valid(pi, 8)) ||
                          (file_valid(pi1 + ".z", 0) && file_valid(pi, 8)) || file_valid(pi + ".book", rec) ||
                          file_valid(pi + ".z", 0) || file_valid(pi + ".book.7z", 0) || file_valid(pi + ".7z", 0);
        if (!skip) return i;
    }
    return o.steps - 1;  // every step on disk
}

// compress: the books the reference's solve compresses (CompressionBridge.cpp:41-59,
// called for layer i+2 after layer i is solved, BookSolver.cpp:596-597, and by
// the optimal-branch pass, :720-728) become trie + xz directories, once every
// pass that rewrites books (deletion threshold, optimal branches) is done.
static void compress_books_if_asked(const egtb_run_options &o) {
    if (!o.compress || !o.write_files) return;
    compress_table_books(o.pathname, o.steps, dtype_size(o.success_rate_dtype), writer_threads(o));
}

static std::vector<uint64_t> read_u64_file(const std::string &path) {
    const uint64_t sz = file_size(path);
    std::vector<uint64_t> v(sz / 8);
    if (!v.empty()) read_file_into(path, v.data(), v.size() * 8);
    return v;
}

static void check_common(const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec *spec,
                         const egtb_run_options *o) {
    if (!spec || !o) throw Error(EGTB_ERR_ARG, "spec and options are required");
    if (n_seeds && !seeds) throw Error(EGTB_ERR_ARG, "seeds pointer is NULL");
    if (o->compress) {
        if (!o->write_files) throw Error(EGTB_ERR_UNSUPPORTED, "compressed books (compress) are files: build with write_files");
        std::string why;
        if (!xz_available(&why)) throw Error(EGTB_ERR_UNSUPPORTED, "compressed books need liblzma: " + why);
    }
    dtype_size(o->success_rate_dtype);
    if (o->steps > (1 << 20)) throw Error(EGTB_ERR_ARG, "steps out of range");
}

static long long seed_tile_sum(uint64_t b) {
    long long s = 0;
    for (int k = 0; k < 16; ++k) {
        const int v = (int)((b >> (4 * k)) & 0xF);
        s += v ? (1ll << v) : 0ll;
    }
    return s;
}

// Tile sum of layer 0. The layer sets rely on every layer having one tile
// sum, which the reference's pattern catalog guarantees by keeping only the
// seeds of the first seed's sum (Config.py:241-248).
static long long layer0_tile_sum(const uint64_t *seeds, size_t n) {
    if (n == 0) return 0;
    const long long s0 = seed_tile_sum(seeds[0]);
    for (size_t i = 1; i < n; ++i)
        if (seed_tile_sum(seeds[i]) != s0)
            throw Error(EGTB_ERR_ARG, "seed boards must share one tile sum (as the pattern catalog keeps them)");
    return s0;
}

static ForwardPlan make_forward_plan(const egtb_pattern_spec &spec, const egtb_run_options &o, int first_step) {
    ForwardPlan P;
    P.steps = o.steps;
    P.docheck = o.docheck_step;
    P.first_step = first_step;
    P.spec = make_dev_spec(spec, o.target);
    P.sort = sort_plan(spec);
    P.s0 = 0;
    const uint64_t pinned = pinned_nibbles(spec);
    std::memset(&P.free, 0, sizeof P.free);
    P.free.pinned = pinned;
    for (int k = 0; k < 16; ++k)
        if (((pinned >> (4 * k)) & 0xF) != 0xF) P.free.idx[P.free.count++] = k;
    return P;
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// --------------------------------------------------------- fused build ----

template <typename T>
static void fused_build(Engine &E, const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec &spec,
                        const egtb_run_options &o, egtb_build_stats *st) {
    const auto t_start = std::chrono::steady_clock::now();
    const unsigned long long launches0 = E.launches;
    const int steps = o.steps;
    const uint32_t total = (uint32_t)(steps * 2);
    set_progress(0, total);
    ForwardPlan P = make_forward_plan(spec, o, 1);
    P.s0 = layer0_tile_sum(seeds, n_seeds);
    float fwd_ms = 0.f, bwd_ms = 0.f;
    const int retries = run_forward(E, P, seeds, n_seeds, nullptr, 0, &fwd_ms);
    std::vector<unsigned long long> off = d2h_u64(E, E.layer_off, steps + 1);
    std::vector<unsigned long long> len = d2h_u64(E, E.layer_len, steps + 1);
    BackwardPlan B{steps, o.docheck_step, o.success_rate_dtype, o.spawn_rate4, P.spec};
    E.ensure_rates(sizeof(T));
    std::vector<unsigned long long> blen, maxb;
    if (o.write_files) {
        backward_write_books<T>(E, B, len, off, o, blen, maxb, &bwd_ms);
    } else {
        EGTB_CUDA(cudaEventRecord(E.ev[2], E.stream));
        enqueue_backward<T>(E, B, len, progress_device_ptr());
        EGTB_CUDA(cudaEventRecord(E.ev[3], E.stream));
        EGTB_CUDA(cudaStreamSynchronize(E.stream));
        EGTB_CUDA(cudaGetLastError());
        EGTB_CUDA(cudaEventElapsedTime(&bwd_ms, E.ev[2], E.ev[3]));
    }
    E.prof_resolve();
    DevCtl c = read_ctl(E);
    if (c.err & kErrIndexOverflow) throw Error(EGTB_ERR_CAPACITY, "rate index probe chain too long");
    if (c.err) throw Error(EGTB_ERR_CAPACITY, "book buffer overflow");
    if (!o.write_files) {
        blen = d2h_u64(E, E.book_len, steps);
        maxb = d2h_u64(E, E.layer_max, steps);
    }
    const size_t rec = 8 + sizeof(T);
    E.last_steps = steps;
    E.last_rec = rec;
    E.last_off = off;
    E.last_blen = blen;
    if (o.write_files) {
        std::vector<int> order;
        for (int t = steps - 3; t >= 0; --t) order.push_back(t);
        write_stats(o, o.success_rate_dtype, order, len, blen, maxb,
                    (fwd_ms + bwd_ms) * 1e-3 / std::max(1, steps));
    }
    set_progress(total, total);
    if (st) {
        std::memset(st, 0, sizeof *st);
        // raw boards of layers 0..steps-3: the layers the solve computes and
        // stats.txt lists (the last two layers keep only their successes)
        for (int t = 0; t < steps; ++t) {
            if (t <= steps - 3) st->raw_boards += len[t];
            st->book_entries += blen[t];
            st->max_layer = std::max<uint64_t>(st->max_layer, len[t]);
        }
        st->candidates = E.candidates;
        st->lookups = c.lookups;
        st->layers = steps;
        st->retries = retries;
        st->forward_ms = fwd_ms;
        st->backward_ms = bwd_ms;
        st->total_ms = ms_since(t_start);
        st->kernel_launches = E.launches - launches0;
    }
}

// ------------------------------------------------- generate (files) -------

template <typename T>
static void generate_files(Engine &E, const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec &spec,
                           const egtb_run_options &o, int *started, egtb_build_stats *st, bool force_stream = false) {
    const auto t_start = std::chrono::steady_clock::now();
    const int steps = o.steps;
    const size_t rec = 8 + sizeof(T);
    const std::string p = o.pathname;
    *started = 0;
    const uint32_t total = (uint32_t)(steps * 2);
    set_progress(0, total);
    if (steps < 3) {
        remove_file(p + std::to_string(steps - 2));
        return;
    }
    const int i0 = first_step_to_run(o, (int)rec);
    float fwd_ms = 0.f;
    int retries = 0;
    std::vector<unsigned long long> off, len;
    if (i0 <= steps - 2) {
        *started = 1;
        std::vector<uint64_t> base, partial;
        if (i0 == 1) {
            write_file(p + "0", seeds, n_seeds * 8);  // BookGenerator.cpp:417-419
            base.assign(seeds, seeds + n_seeds);
        } else {
            base = read_u64_file(p + std::to_string(i0 - 1));
            partial = read_u64_file(p + std::to_string(i0));
        }
        ForwardPlan P = make_forward_plan(spec, o, i0);
        P.s0 = n_seeds ? layer0_tile_sum(seeds, n_seeds)
                       : (base.empty() ? 0 : seed_tile_sum(base[0]) - 2ll * (i0 - 1));
        // the whole table in device memory when it fits, else layers streamed to their files
        bool streamed = force_stream || stream_layers_forced();
        if (!streamed) {
            try {
                retries = run_forward(E, P, base.data(), base.size(), partial.data(), partial.size(), &fwd_ms);
            } catch (const Error &e) {
                if (e.code != EGTB_ERR_CAPACITY) throw;
                streamed = true;
            }
        }
        if (streamed)
            retries += run_forward_streamed(E, P, base.data(), base.size(), partial.data(), partial.size(), p,
                                            &fwd_ms, off, len);
        else {
            off = d2h_u64(E, E.layer_off, steps + 1);
            len = d2h_u64(E, E.layer_len, steps + 1);
        }
        // raw layers i0 .. steps-3 (written already when streamed)
        std::vector<std::string> paths;
        std::vector<unsigned long long> doff, bytes;
        for (int t = i0; t <= steps - 3 && !streamed; ++t) {
            paths.push_back(p + std::to_string(t));
            doff.push_back(off[t] * 8);
            bytes.push_back(len[t] * 8);
        }
        // final_steps: success-only books of layers steps-2 and steps-1
        const T zero = (T)dtype_zero(o.success_rate_dtype), maxv = (T)dtype_max(o.success_rate_dtype);
        DevSpec ds = make_dev_spec(spec, o.target);
        E.ensure_rates(sizeof(T));
        EGTB_CUDA(cudaMemsetAsync(E.ctl, 0, sizeof(DevCtl), E.stream));
        for (int t = steps - 2; t < steps; ++t) {
            EGTB_LAUNCH(E, final_layer_kernel<T><<<E.sm_count * 4, 256, 0, E.stream>>>(E.arena, (T *)E.rates, E.layer_off, E.layer_len, t, ds, zero, maxv));
            enqueue_pack<T>(E, t, zero);
            enqueue_pack_write<T>(E, t, zero, off[t] * rec);
        }
        std::vector<unsigned long long> blen = d2h_u64(E, E.book_len, steps);
        write_ranges(E, (const unsigned char *)E.arena, paths, doff, bytes, writer_threads(o));
        std::vector<std::string> bpaths = {p + std::to_string(steps - 2) + ".book", p + std::to_string(steps - 1) + ".book"};
        std::vector<unsigned long long> boff = {off[steps - 2] * rec, off[steps - 1] * rec};
        std::vector<unsigned long long> bbytes = {blen[steps - 2] * rec, blen[steps - 1] * rec};
        write_ranges(E, E.book, bpaths, boff, bbytes, writer_threads(o));
        if (st) {
            std::memset(st, 0, sizeof *st);
            for (int t = i0; t <= steps - 3; ++t) {
                st->raw_boards += len[t];
                st->max_layer = std::max<uint64_t>(st->max_layer, len[t]);
            }
            st->book_entries = blen[steps - 2] + blen[steps - 1];
            st->candidates = E.candidates;
        }
    }
    remove_file(p + std::to_string(steps - 2));  // final_steps, BookSolver.cpp:279-282
    if (st) {
        st->layers = steps;
        st->retries = retries;
        st->forward_ms = fwd_ms;
        st->total_ms = ms_since(t_start);
    }
}

// ---------------------------------------------------- solve (files) -------

// Split packed records into the arena slot (keys) and rates.
template <typename T>
__global__ void unpack_records_kernel(const unsigned char *__restrict__ recs, unsigned long long n,
                                      uint64_t *__restrict__ keys, T *__restrict__ rates) {
    constexpr int rec = 8 + (int)sizeof(T);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(recs + i * rec);
        keys[i] = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
        T r;
        std::memcpy(&r, recs + i * rec + 8, sizeof(T));
        rates[i] = r;
    }
}

__global__ void splitters_kernel(const uint64_t *__restrict__ keys, unsigned long long n, uint64_t *__restrict__ split) {
    const unsigned long long ns = (n + kSplitStride - 1) / kSplitStride;
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < ns;
         j += (unsigned long long)gridDim.x * blockDim.x)
        split[j] = keys[j * kSplitStride];
}

// recalculate_process_impl, native_core/src/BookSolver.cpp:513-605, with the
// three live layers (i, i+1, i+2) in rotating arena slots.
template <typename T>
static void solve_files(Engine &E, const void *d1_recs, size_t n1, const void *d2_recs, size_t n2,
                        const egtb_pattern_spec &spec, const egtb_run_options &o, egtb_build_stats *st) {
    const auto t_start = std::chrono::steady_clock::now();
    const int steps = o.steps;
    const size_t rec = 8 + sizeof(T);
    const std::string p = o.pathname;
    const T zero = (T)dtype_zero(o.success_rate_dtype), maxv = (T)dtype_max(o.success_rate_dtype);
    const uint32_t total = (uint32_t)(steps * 2);
    DevSpec ds = make_dev_spec(spec, o.target);
    cudaStream_t s = E.stream;
    E.ensure_steps(4);

    // the largest layer decides the slot size
    unsigned long long slot = 16;
    for (int i = 0; i < steps; ++i) {
        slot = std::max<unsigned long long>(slot, file_size(p + std::to_string(i)) / 8);
        slot = std::max<unsigned long long>(slot, file_size(p + std::to_string(i) + ".book") / rec);
    }
    slot = std::max<unsigned long long>(slot, std::max(n1, n2));
    slot = align16(slot);
    E.ensure_arena(slot * 3);
    E.ensure_rates(sizeof(T));
    E.ensure_cand(std::max<unsigned long long>(E.cand_cap, 1ull << 22));
    E.ensure_index(index_slots(slot));
    int idx_of[3] = {0, 1, 2};  // rate index of layer i, i+1, i+2
    bool index_fresh = false;   // indexes of i+1, i+2 match the resident layers

    // host copies of the two successor layers (packed records)
    std::vector<unsigned char> h1((const unsigned char *)d1_recs, (const unsigned char *)d1_recs + n1 * rec);
    std::vector<unsigned char> h2((const unsigned char *)d2_recs, (const unsigned char *)d2_recs + n2 * rec);
    bool started = false;
    int slot_of[3] = {0, 1, 2};  // slot of layer i, i+1, i+2
    bool resident = false;       // layers i+1, i+2 already on the device
    bool skipped_since_start = false;
    write_stats(o, o.success_rate_dtype, {}, {}, {}, {}, 0.0);  // header first (ensure_stats_header)
    unsigned long long dlen1 = 0, dlen2 = 0;
    unsigned char *d_stage = nullptr;
    EGTB_CUDA(cudaMalloc(&d_stage, std::max<size_t>(slot * rec, 16)));
    std::unique_ptr<unsigned char, void (*)(unsigned char *)> stage_guard(d_stage, [](unsigned char *q) { cudaFree(q); });
    T *rates = (T *)E.rates;

    auto upload_layer = [&](const std::vector<unsigned char> &recs, int sl) -> unsigned long long {
        const unsigned long long n = recs.size() / rec;
        if (n > slot) throw Error(EGTB_ERR_CAPACITY, "layer larger than its slot");
        if (n) {
            EGTB_CUDA(cudaMemcpyAsync(d_stage, recs.data(), n * rec, cudaMemcpyHostToDevice, s));
            EGTB_LAUNCH(E, unpack_records_kernel<T><<<E.sm_count * 4, 256, 0, s>>>(d_stage, n, E.arena + sl * slot, rates + sl * slot));
            EGTB_LAUNCH(E, splitters_kernel<<<E.sm_count, 256, 0, s>>>(E.arena + sl * slot, n, E.split + sl * slot / kSplitStride));
            EGTB_CUDA(cudaStreamSynchronize(s));
        }
        return n;
    };

    for (int i = steps - 3; i >= 0; --i) {
        set_progress(total - (uint32_t)i - 2u, total);
        const std::string pi = p + std::to_string(i);
        remove_invalid(pi + ".book", rec);
        remove_invalid(pi + ".z", 0);
        remove_invalid(pi + ".book.7z", 0);
        if (file_valid(pi + ".book", rec) || file_valid(pi + ".z", 0) || file_valid(pi + ".book.7z", 0)) {
            resident = false;
            if (started) skipped_since_start = true;
            continue;
        }
        if (!started) {
            started = true;
            if (i != steps - 3 || h1.empty() || h2.empty()) {
                h1 = read_file(p + std::to_string(i + 1) + ".book");
                h2 = read_file(p + std::to_string(i + 2) + ".book");
            }
        }
        if (!resident) {
            if (skipped_since_start) {
                // resuming after a layer that was already on disk
                h1 = read_file(p + std::to_string(i + 1) + ".book");
                h2 = read_file(p + std::to_string(i + 2) + ".book");
                skipped_since_start = false;
            }
            dlen1 = upload_layer(h1, slot_of[1]);
            dlen2 = upload_layer(h2, slot_of[2]);
            resident = true;
            index_fresh = false;
        }
        std::vector<uint64_t> raw = read_u64_file(pi);
        const unsigned long long n0 = raw.size();
        if (n0 > slot) throw Error(EGTB_ERR_CAPACITY, "raw layer larger than its slot");
        uint64_t *k0 = E.arena + slot_of[0] * slot;
        if (n0) EGTB_CUDA(cudaMemcpyAsync(k0, raw.data(), n0 * 8, cudaMemcpyHostToDevice, s));
        unsigned long long off_h[3] = {slot_of[0] * slot, slot_of[1] * slot, slot_of[2] * slot};
        unsigned long long len_h[3] = {n0, dlen1, dlen2};
        EGTB_CUDA(cudaMemcpyAsync(E.layer_off, off_h, sizeof off_h, cudaMemcpyHostToDevice, s));
        EGTB_CUDA(cudaMemcpyAsync(E.layer_len, len_h, sizeof len_h, cudaMemcpyHostToDevice, s));
        EGTB_CUDA(cudaMemsetAsync(E.ctl, 0, sizeof(DevCtl), s));
        EGTB_CUDA(cudaMemsetAsync(E.layer_max, 0, sizeof(unsigned long long) * 4, s));
        const auto t0 = std::chrono::steady_clock::now();
        if (!index_fresh) {
            enqueue_index_at<T>(E, 1, dlen1, zero, E.index[idx_of[1]]);
            enqueue_index_at<T>(E, 2, dlen2, zero, E.index[idx_of[2]]);
            index_fresh = true;
        }
        EGTB_LAUNCH(E, solve_kernel_for<T>(ds)<<<E.sm_count * 8, 256, 0, s>>>(
                           E.arena, rates, E.layer_off, E.layer_len, 0, ds, i > o.docheck_step ? 1 : 0, E.tab,
                           o.spawn_rate4, zero, maxv, E.index[idx_of[1]], index_slots(dlen1) - 1, E.index[idx_of[2]],
                           index_slots(dlen2) - 1, E.ctl, nullptr, 0, nullptr, 0, nullptr, 0));
        if (i > 0) enqueue_index_at<T>(E, 0, n0, zero, E.index[idx_of[0]]);
        EGTB_LAUNCH(E, splitters_kernel<<<E.sm_count, 256, 0, s>>>(k0, n0, E.split + slot_of[0] * slot / kSplitStride));
        enqueue_pack<T>(E, 0, zero);
        enqueue_pack_write<T>(E, 0, zero, 0);
        EGTB_LAUNCH(E, layer_max_kernel<T><<<E.sm_count, 256, 0, s>>>(rates, E.layer_off, E.layer_len, 0, zero, E.layer_max));
        unsigned long long nb = 0, mb = 0;
        EGTB_CUDA(cudaMemcpyAsync(&nb, E.book_len, 8, cudaMemcpyDeviceToHost, s));
        EGTB_CUDA(cudaMemcpyAsync(&mb, E.layer_max, 8, cudaMemcpyDeviceToHost, s));
        EGTB_CUDA(cudaStreamSynchronize(s));
        EGTB_CUDA(cudaGetLastError());
        if (read_ctl(E).err) throw Error(EGTB_ERR_CAPACITY, "rate index or book buffer overflow in the solve");
        std::vector<unsigned char> book(nb * rec);
        if (nb) EGTB_CUDA(cudaMemcpy(book.data(), E.book, nb * rec, cudaMemcpyDeviceToHost));
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (nb) {
            std::vector<int> lay = {i};
            std::vector<unsigned long long> rl(i + 1, 0), bl(i + 1, 0), mx(i + 1, 0);
            rl[i] = n0;
            bl[i] = nb;
            mx[i] = mb;
            write_stats(o, o.success_rate_dtype, lay, rl, bl, mx, secs);
        }
        write_file(pi + ".book", book.data(), book.size());
        remove_file(pi);
        if (o.deletion_threshold > 0.0) {
            // compact layer i+2 with the threshold and rewrite its book
            // (BookSolver.cpp:589-593); computation is unaffected.
            const double thr_d = o.deletion_threshold * (dtype_max(o.success_rate_dtype) - dtype_zero(o.success_rate_dtype)) +
                                 dtype_zero(o.success_rate_dtype);
            const T thr = (T)thr_d;
            std::vector<unsigned char> kept;
            for (size_t r = 0; r < h2.size() / rec; ++r) {
                T v;
                std::memcpy(&v, h2.data() + r * rec + 8, sizeof(T));
                if (v > thr) kept.insert(kept.end(), h2.begin() + r * rec, h2.begin() + (r + 1) * rec);
            }
            write_file(p + std::to_string(i + 2) + ".book", kept.data(), kept.size());
        }
        if (i > 0) {
            // rotate: layer i becomes i+1, i+1 becomes i+2
            const int old2 = slot_of[2];
            slot_of[2] = slot_of[1];
            slot_of[1] = slot_of[0];
            slot_of[0] = old2;
            const int oldi = idx_of[2];
            idx_of[2] = idx_of[1];
            idx_of[1] = idx_of[0];
            idx_of[0] = oldi;
            dlen2 = dlen1;
            dlen1 = n0;
            h2.swap(h1);
            h1.swap(book);
            resident = true;
        }
        if (st) {
            st->raw_boards += n0;
            st->book_entries += nb;
            st->max_layer = std::max<uint64_t>(st->max_layer, n0);
        }
    }
    if (st) {
        st->layers = steps;
        st->total_ms = ms_since(t_start);
    }
}

// ---------------------------------------------- optimal-branch pass --------

// keep_only_optimal_branches_impl (native_core/src/BookSolver.cpp:688-735) on
// the book files the solve wrote: for i = 21 .. steps-1, book i keeps only
// the entries that are the best move of a position of the thinned book i-2
// plus a 4 or of the thinned book i-1 plus a 2 (optimal_mark_kernel), in
// order, and is rewritten. Three layers live on the device (keys + rates),
// with a {key, position} index and a mark byte per entry of book i.
template <typename T>
static void optimal_branch_files(Engine &E, const egtb_pattern_spec &spec, const egtb_run_options &o) {
    const int steps = o.steps;
    const std::string p = o.pathname;
    const size_t rec = 8 + sizeof(T);
    const T zero = (T)dtype_zero(o.success_rate_dtype);
    cudaStream_t s = E.stream;
    const uint32_t total = (uint32_t)(steps * 3);
    if (steps <= 21) {  // the pass thins layers 21 and up only
        if (file_exists(p + "optlayer")) std::remove((p + "optlayer").c_str());
        set_progress(total, total);
        return;
    }
    const DevSpec ds = make_dev_spec(spec, o.target);
    unsigned long long cap = 16;
    for (int i = 19; i < steps; ++i) cap = std::max<unsigned long long>(cap, file_size(p + std::to_string(i) + ".book") / rec);
    unsigned long long slots = 64;
    while (slots < 2 * cap) slots <<= 1;
    const unsigned long long tiles = cap / kTileKeys + 2;
    // one block: keys[3] | rates[3] | index | marks | records | tile counts |
    // tile offsets | total, every part starting on a 256-byte boundary
    auto r256 = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t part[7] = {r256(cap * 8),  r256(cap * sizeof(T)), r256(slots * sizeof(ulonglong2)), r256(cap),
                            r256(cap * rec), r256(tiles * 4),       r256(tiles * 8)};
    const size_t bytes = 3 * part[0] + 3 * part[1] + part[2] + part[3] + part[4] + part[5] + part[6] + 256;
    unsigned char *base = nullptr;
    E.alloc_or_throw((void **)&base, bytes, "optimal-branch pass");
    std::unique_ptr<unsigned char, void (*)(unsigned char *)> guard(base, [](unsigned char *q) { cudaFree(q); });
    size_t at = 0;
    auto take = [&](size_t n) {
        unsigned char *q = base + at;
        at += n;
        return q;
    };
    uint64_t *keys[3];
    T *rates[3];
    for (int k = 0; k < 3; ++k) keys[k] = (uint64_t *)take(part[0]);
    for (int k = 0; k < 3; ++k) rates[k] = (T *)take(part[1]);
    ulonglong2 *index = (ulonglong2 *)take(part[2]);
    uint8_t *marks = take(part[3]);
    unsigned char *recs = take(part[4]);
    unsigned *tile_cnt = (unsigned *)take(part[5]);
    unsigned long long *tile_off = (unsigned long long *)take(part[6]);
    unsigned long long *d_total = (unsigned long long *)take(256);
    const int g = E.sm_count * 4;
    // book L's records -> keys[slot], rates[slot] (staged through `recs`)
    auto load = [&](int L, int slot) -> unsigned long long {
        std::vector<unsigned char> h = read_file(p + std::to_string(L) + ".book");
        const unsigned long long n = h.size() / rec;
        if (n > cap) throw Error(EGTB_ERR_CAPACITY, "book larger than measured");
        if (n) {
            EGTB_CUDA(cudaMemcpyAsync(recs, h.data(), n * rec, cudaMemcpyHostToDevice, s));
            EGTB_LAUNCH(E, unpack_records_kernel<T><<<g, 256, 0, s>>>(recs, n, keys[slot], rates[slot]));
        }
        EGTB_CUDA(cudaStreamSynchronize(s));
        return n;
    };
    int s0 = 0, s1 = 1, s2 = 2;  // slots of books i-2, i-1 (thinned) and i
    unsigned long long n0 = 0, n1 = 0;
    // handle_restart_opt_only (BookSolver.cpp:648-683): "<path>optlayer" holds
    // the last layer already thinned; the pass starts after it, from books
    // i-2 and i-1 as they are on disk, and rewrites the marker before each
    // later layer.
    const std::string marker = p + "optlayer";
    bool started = false;
    for (int i = 0; i < steps; ++i) {
        set_progress((uint32_t)(2 * steps + i + 1), total);
        if (started) {
            const std::string last = std::to_string(i - 1);
            write_file(marker, last.data(), last.size());
        } else {
            int current = i - 1;
            if (file_exists(marker)) {
                const std::vector<unsigned char> text = read_file(marker);
                std::istringstream in(std::string(text.begin(), text.end()));
                in >> current;
            }
            const std::string b0 = p + std::to_string(i - 2) + ".book", b1 = p + std::to_string(i - 1) + ".book";
            if (current >= i || i <= 20 || !file_exists(b0) || !file_exists(b1)) continue;
            n0 = load(i - 2, s0);
            n1 = load(i - 1, s1);
            started = true;
        }
        const unsigned long long n2 = load(i, s2);
        unsigned long long kept = 0;
        if (n2) {
            unsigned long long sl = 64;
            while (sl < 2 * n2) sl <<= 1;
            EGTB_CUDA(cudaMemsetAsync(index, 0, sl * sizeof(ulonglong2), s));
            EGTB_LAUNCH(E, pos_index_kernel<<<g, 256, 0, s>>>(keys[s2], n2, index, sl - 1));
            EGTB_CUDA(cudaMemsetAsync(marks, 0, n2, s));
            if (n0)
                EGTB_LAUNCH(E, optimal_mark_kernel<T><<<g, 256, 0, s>>>(keys[s0], n0, 2ull, ds, E.tab, index, sl - 1,
                                                                      rates[s2], n2, zero, marks));
            if (n1)
                EGTB_LAUNCH(E, optimal_mark_kernel<T><<<g, 256, 0, s>>>(keys[s1], n1, 1ull, ds, E.tab, index, sl - 1,
                                                                      rates[s2], n2, zero, marks));
            const unsigned long long nt = (n2 + kTileKeys - 1) / kTileKeys;
            EGTB_LAUNCH(E, mark_count_kernel<<<g, kSortThreads, 0, s>>>(marks, n2, tile_cnt));
            EGTB_LAUNCH(E, scan_tiles_kernel<<<1, 1024, 0, s>>>(tile_cnt, nt, tile_off, d_total));
            // the thinned book i goes to the slot of book i-2, which is no longer needed
            EGTB_LAUNCH(E, mark_write_kernel<T><<<g, kSortThreads, 0, s>>>(keys[s2], rates[s2], marks, n2, tile_off,
                                                                        keys[s0], rates[s0], recs));
            EGTB_CUDA(cudaMemcpyAsync(&kept, d_total, 8, cudaMemcpyDeviceToHost, s));
            EGTB_CUDA(cudaStreamSynchronize(s));
            EGTB_CUDA(cudaGetLastError());
        }
        std::vector<unsigned char> out(kept * rec);
        if (kept) EGTB_CUDA(cudaMemcpy(out.data(), recs, kept * rec, cudaMemcpyDeviceToHost));
        write_file(p + std::to_string(i) + ".book", out.data(), out.size());
        // books i-1 and i (thinned) are the parents of book i+1
        const int thinned = s0;
        s0 = s1;
        s1 = thinned;
        n0 = n1;
        n1 = kept;
    }
    if (file_exists(marker)) std::remove(marker.c_str());
    set_progress(total, total);
}

// ------------------------------------------------------ primitives -------

__global__ void prim_moves_kernel(const uint32_t *tab, const uint64_t *in, size_t n, uint64_t *out4) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t m[4];
        move_all_dir(tab, in[i], m);
        for (int d = 0; d < 4; ++d) out4[4 * i + d] = m[d];
    }
}

__global__ void prim_canonical_kernel(const uint64_t *in, size_t n, int mode, uint64_t *out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = canonical(in[i], mode);
}

__global__ void prim_sym_kernel(const uint64_t *in, size_t n, int idx, uint64_t *out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = apply_sym(in[i], idx);
}

template <typename Launch>
static void run_prim(int device, const uint64_t *boards, size_t n, size_t out_per, uint64_t *out, Launch launch) {
    if (n == 0) return;
    if (!boards || !out) throw Error(EGTB_ERR_ARG, "NULL buffer");
    Engine &E = engine_for(device);
    std::lock_guard<std::mutex> lk(E.mu);
    uint64_t *din = nullptr, *dout = nullptr;
    EGTB_CUDA(cudaMalloc(&din, n * 8));
    std::unique_ptr<uint64_t, void (*)(uint64_t *)> g1(din, [](uint64_t *q) { cudaFree(q); });
    EGTB_CUDA(cudaMalloc(&dout, n * 8 * out_per));
    std::unique_ptr<uint64_t, void (*)(uint64_t *)> g2(dout, [](uint64_t *q) { cudaFree(q); });
    EGTB_CUDA(cudaMemcpyAsync(din, boards, n * 8, cudaMemcpyHostToDevice, E.stream));
    launch(E, din, dout);
    EGTB_CUDA(cudaGetLastError());
    EGTB_CUDA(cudaMemcpyAsync(out, dout, n * 8 * out_per, cudaMemcpyDeviceToHost, E.stream));
    EGTB_CUDA(cudaStreamSynchronize(E.stream));
}

// ------------------------------------------- access for the batched build --

EngineRef engine_ref(int device) {
    Engine &E = engine_for(device);
    // the batched build moves every table with the classic rule
    return EngineRef{&E.mu, E.device, &E.stream, E.classic_tab, E.sm_count, E.sweep_grid, E.seg_grid};
}

uint64_t pattern_pinned_nibbles(const egtb_pattern_spec &s) { return pinned_nibbles(s); }

unsigned *build_progress_ptr() { return progress_device_ptr(); }

void build_progress_set(uint32_t cur, uint32_t total) { set_progress(cur, total); }

void write_stats_file(const egtb_run_options &o, int dtype, const std::vector<int> &layers,
                      const std::vector<unsigned long long> &raw_len, const std::vector<unsigned long long> &book_len,
                      const std::vector<unsigned long long> &maxbits, double seconds_per_layer) {
    write_stats(o, dtype, layers, raw_len, book_len, maxbits, seconds_per_layer);
}

}  // namespace egtb

// =================================================================== C ABI ===

using namespace egtb;

extern "C" const char *egtb_version(void) { return "egtb_gpu 0.1 sm_100a"; }

extern "C" int egtb_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" int egtb_set_stream(int device, void *stream) {
    return guarded([&] {
        Engine &E = engine_for(device);
        std::lock_guard<std::mutex> lk(E.mu);
        EGTB_CUDA(cudaStreamSynchronize(E.stream));
        E.stream = stream ? (cudaStream_t)stream : E.own_stream;
    });
}

extern "C" int egtb_profile(int device, int enable) {
    return guarded([&] {
        Engine &E = engine_for(device);
        std::lock_guard<std::mutex> lk(E.mu);
        E.prof_resolve();
        E.prof = enable != 0;
        for (int k = 0; k < K_NKINDS; ++k) {
            E.prof_launches[k] = 0;
            E.prof_ms[k] = 0.0;
        }
    });
}

extern "C" int egtb_profile_read(int device, egtb_kernel_time *out, int max_kinds, int *n_kinds) {
    return guarded([&] {
        if (!out || !n_kinds) throw Error(EGTB_ERR_ARG, "NULL argument");
        Engine &E = engine_for(device);
        std::lock_guard<std::mutex> lk(E.mu);
        E.prof_resolve();
        int n = 0;
        for (int k = 0; k < K_NKINDS && n < max_kinds; ++k) {
            std::memset(&out[n], 0, sizeof out[n]);
            std::strncpy(out[n].name, kKindNames[k], sizeof out[n].name - 1);
            out[n].launches = E.prof_launches[k];
            out[n].total_ms = E.prof_ms[k];
            ++n;
        }
        *n_kinds = n;
    });
}

extern "C" int egtb_get_build_progress(uint32_t *current, uint32_t *total) {
    if (!current || !total) return EGTB_ERR_ARG;
    // get_build_progress, native_core/include/FormationRuntime.h:73-82
    uint32_t t = g_progress_total.load(std::memory_order_relaxed);
    uint32_t c = read_progress();
    if (c > t) t = c;
    *current = c;
    *total = t;
    return EGTB_OK;
}

extern "C" int egtb_reset_build_progress(uint32_t total) {
    g_progress_total.store(total, std::memory_order_relaxed);
    g_progress_host.store(0, std::memory_order_relaxed);
    if (g_progress_mapped) *(volatile unsigned *)g_progress_mapped = 0;
    return EGTB_OK;
}

template <typename F>
static int dispatch_dtype(int dtype, F &&f) {
    switch (dtype) {
        case EGTB_DTYPE_UINT32: f((uint32_t)0); break;
        case EGTB_DTYPE_UINT64: f((uint64_t)0); break;
        case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32: f(0.0f); break;
        case EGTB_DTYPE_FLOAT64: case EGTB_DTYPE_1_FLOAT64: f(0.0); break;
        default: throw Error(EGTB_ERR_ARG, "unknown success_rate_dtype");
    }
    return 0;
}

extern "C" int egtb_generate(const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec *spec,
                             const egtb_run_options *options, int32_t *started, egtb_build_stats *stats) {
    return guarded([&] {
        check_common(seeds, n_seeds, spec, options);
        Engine &E = engine_for(options->device);
        std::lock_guard<std::mutex> lk(E.mu);
        E.use_mover(options->is_variant != 0);  // VBoardMover for variant boards (BookSolver.cpp:792-819)
        int st = 0;
        if (stats) std::memset(stats, 0, sizeof *stats);
        dispatch_dtype(options->success_rate_dtype, [&](auto z) {
            using T = decltype(z);
            generate_files<T>(E, seeds, n_seeds, *spec, *options, &st, stats);
        });
        if (started) *started = st;
    });
}

extern "C" int egtb_solve(const void *d1_records, size_t n1, const void *d2_records, size_t n2,
                          const egtb_pattern_spec *spec, const egtb_run_options *options, egtb_build_stats *stats) {
    return guarded([&] {
        check_common(nullptr, 0, spec, options);
        if ((n1 && !d1_records) || (n2 && !d2_records)) throw Error(EGTB_ERR_ARG, "NULL record buffer");
        Engine &E = engine_for(options->device);
        std::lock_guard<std::mutex> lk(E.mu);
        E.use_mover(options->is_variant != 0);  // VBoardMover for variant boards (BookSolver.cpp:792-819)
        if (stats) std::memset(stats, 0, sizeof *stats);
        dispatch_dtype(options->success_rate_dtype, [&](auto z) {
            using T = decltype(z);
            solve_files<T>(E, d1_records, n1, d2_records, n2, *spec, *options, stats);
            if (options->optimal_branch_only) optimal_branch_files<T>(E, *spec, *options);  // run_pattern_solve_impl
            compress_books_if_asked(*options);
        });
    });
}

extern "C" int egtb_build(const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec *spec,
                          const egtb_run_options *options, egtb_build_stats *stats) {
    return guarded([&] {
        check_common(seeds, n_seeds, spec, options);
        // run_pattern_build_cpp resets the progress first (BookSolver.cpp:828)
        // classic_build_progress_total (FormationRuntime.h:48-54)
        egtb_reset_build_progress((uint32_t)(options->steps > 0 ? options->steps * (options->optimal_branch_only ? 3 : 2)
                                                                : 0));
        Engine &E = engine_for(options->device);
        std::lock_guard<std::mutex> lk(E.mu);
        E.use_mover(options->is_variant != 0);  // VBoardMover for variant boards (BookSolver.cpp:792-819)
        if (stats) std::memset(stats, 0, sizeof *stats);
        const bool resume = options->write_files && any_layer_file(*options);
        dispatch_dtype(options->success_rate_dtype, [&](auto z) {
            using T = decltype(z);
            if (options->steps < 3) {
                int st = 0;
                generate_files<T>(E, seeds, n_seeds, *spec, *options, &st, stats);
                return;
            }
            bool streamed = false;
            // a deletion threshold rewrites the book of layer i+2 after solving
            // layer i (BookSolver.cpp:589-593): the layer-by-layer solve does that
            const bool layered = options->deletion_threshold > 0.0;
            if ((layered || options->optimal_branch_only) && !options->write_files)
                throw Error(EGTB_ERR_UNSUPPORTED,
                            "deletion_threshold and optimal_branch_only rewrite book files: build with write_files");
            if (!resume && !layered && !(options->write_files && stream_layers_forced())) {
                try {
                    fused_build<T>(E, seeds, n_seeds, *spec, *options, stats);
                    if (options->optimal_branch_only) optimal_branch_files<T>(E, *spec, *options);
                    compress_books_if_asked(*options);
                    return;
                } catch (const Error &e) {
                    // the table does not fit in device memory: with files, build it
                    // as the reference does (generate, then solve) with streamed layers
                    if (e.code != EGTB_ERR_CAPACITY || !options->write_files) throw;
                    streamed = true;
                }
            } else if (!resume && !layered) {
                streamed = true;  // EGTB_STREAM_LAYERS
            }
            {
                int st = 0;
                egtb_build_stats g;
                std::memset(&g, 0, sizeof g);
                generate_files<T>(E, seeds, n_seeds, *spec, *options, &st, &g, streamed);
                solve_files<T>(E, nullptr, 0, nullptr, 0, *spec, *options, stats);
                if (options->optimal_branch_only) optimal_branch_files<T>(E, *spec, *options);
                compress_books_if_asked(*options);
                if (stats) {
                    stats->forward_ms = g.forward_ms;
                    stats->candidates = g.candidates;
                }
            }
        });
    });
}

extern "C" int egtb_release(int32_t device) {
    return guarded([&] {
        Engine &E = engine_for(device);
        std::lock_guard<std::mutex> lk(E.mu);
        EGTB_CUDA(cudaSetDevice(E.device));
        EGTB_CUDA(cudaStreamSynchronize(E.stream));
        if (E.copy_stream) EGTB_CUDA(cudaStreamSynchronize(E.copy_stream));
        E.release_buffers();
        batch_release_buffers(E.device);
    });
}

extern "C" int egtb_book_layer_copy(int device, int32_t layer, void *dst, size_t dst_bytes, uint64_t *bytes) {
    return guarded([&] {
        if (!bytes) throw Error(EGTB_ERR_ARG, "NULL size pointer");
        Engine &E = engine_for(device);
        std::lock_guard<std::mutex> lk(E.mu);
        if (layer < 0 || layer >= E.last_steps) throw Error(EGTB_ERR_ARG, "no such layer in the last in-memory build");
        const unsigned long long nb = E.last_blen[layer] * E.last_rec;
        *bytes = nb;
        if (!dst) return;  // size query
        if (dst_bytes < nb) throw Error(EGTB_ERR_ARG, "destination buffer too small");
        if (nb)
            EGTB_CUDA(cudaMemcpy(dst, E.book + E.last_off[layer] * E.last_rec, nb, cudaMemcpyDeviceToHost));
    });
}

extern "C" int egtb_move_all_dir(int device, const uint64_t *boards, size_t n, uint64_t *out4) {
    return guarded([&] {
        run_prim(device, boards, n, 4, out4, [&](Engine &E, uint64_t *din, uint64_t *dout) {
            EGTB_LAUNCH(E, prim_moves_kernel<<<E.sm_count * 4, 256, 0, E.stream>>>(E.classic_tab, din, n, dout));
        });
    });
}

extern "C" int egtb_move_all_dir_variant(int device, const uint64_t *boards, size_t n, uint64_t *out4) {
    return guarded([&] {
        run_prim(device, boards, n, 4, out4, [&](Engine &E, uint64_t *din, uint64_t *dout) {
            EGTB_LAUNCH(E, prim_moves_kernel<<<E.sm_count * 4, 256, 0, E.stream>>>(E.variant_tab, din, n, dout));
        });
    });
}

extern "C" int egtb_canonical(int device, const uint64_t *boards, size_t n, int32_t symm_mode, uint64_t *out) {
    return guarded([&] {
        if (symm_mode < 0 || symm_mode > 6) throw Error(EGTB_ERR_ARG, "symmetry mode out of range");
        run_prim(device, boards, n, 1, out, [&](Engine &E, uint64_t *din, uint64_t *dout) {
            EGTB_LAUNCH(E, prim_canonical_kernel<<<E.sm_count * 4, 256, 0, E.stream>>>(din, n, symm_mode, dout));
        });
    });
}

extern "C" int egtb_apply_sym(int device, const uint64_t *boards, size_t n, int32_t symm_index, uint64_t *out) {
    return guarded([&] {
        run_prim(device, boards, n, 1, out, [&](Engine &E, uint64_t *din, uint64_t *dout) {
            EGTB_LAUNCH(E, prim_sym_kernel<<<E.sm_count * 4, 256, 0, E.stream>>>(din, n, symm_index, dout));
        });
    });
}
