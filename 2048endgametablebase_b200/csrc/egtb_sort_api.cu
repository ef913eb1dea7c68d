// egtb_sort_unique_u64: the layer sort of the build (onesweep LSD radix sort
// over all 16 nibbles + single-pass unique) on caller-owned device memory.
// It takes the place of the reference's CPU sort/unique plug-in seam
// (bookgen_native.so: sort_uint64, native_core/xss_wrapper.cpp:14-31, and
// unique_sorted_u64_inplace, native_core/src/unique_wrapper.cpp:12-14),
// on the device. Scratch is stream-ordered (cudaMallocAsync on the caller's
// stream) and released before the call returns to the stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "egtb_host.h"
#include "egtb_sort.cuh"

namespace egtb {

// All 16 nibbles, two per pass, least significant first.
static SortPlan full_key_plan() {
    SortPlan sp;
    std::memset(&sp, 0, sizeof sp);
    sp.passes = 8;
    for (int p = 0; p < 8; ++p) {
        sp.lo[p] = 2 * p;
        sp.hi[p] = 2 * p + 1;
    }
    return sp;
}

// Scratch of one sort of up to n keys, carved from one block of device memory.
struct SortScratch {
    uint64_t *tmp;                 // n keys
    unsigned long long *status;    // tiles x 256
    unsigned long long *ustatus;   // tiles
    unsigned *hist;                // kMaxPasses x 256
    unsigned *counters;            // 16
    DevCtl *ctl;
    unsigned long long *layer_off; // 2
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t scratch_bytes(size_t n) {
    const size_t tiles = n / kTileKeys + 2;
    return align256(n * 8 + 8) + align256(tiles * 256 * 8) + align256(tiles * 8) +
           align256(kMaxPasses * 256 * 4) + align256(16 * 4) + align256(sizeof(DevCtl)) + align256(16);
}

static SortScratch carve(unsigned char *base, size_t n) {
    const size_t tiles = n / kTileKeys + 2;
    SortScratch s;
    size_t o = 0;
    s.tmp = (uint64_t *)(base + o);
    o += align256(n * 8 + 8);
    s.status = (unsigned long long *)(base + o);
    o += align256(tiles * 256 * 8);
    s.ustatus = (unsigned long long *)(base + o);
    o += align256(tiles * 8);
    s.hist = (unsigned *)(base + o);
    o += align256(kMaxPasses * 256 * 4);
    s.counters = (unsigned *)(base + o);
    o += align256(16 * 4);
    s.ctl = (DevCtl *)(base + o);
    o += align256(sizeof(DevCtl));
    s.layer_off = (unsigned long long *)(base + o);
    return s;
}

static __global__ void set_count_kernel(unsigned long long *p, unsigned long long v) { *p = v; }

// Enqueue the sort of d_in[0..n) into d_out (unique keys, ascending) and the
// unique count into *d_n_out, using scratch s whose look-back words carry
// epochs first_epoch .. first_epoch+8. The scratch's look-back words, the
// histograms and the control block are cleared first.
static void enqueue_sort_unique_u64(const uint64_t *d_in, size_t n, uint64_t *d_out, unsigned long long *d_n_out,
                                    const SortScratch &s, int grid, cudaStream_t st, bool count_by_kernel = false) {
    const size_t tiles = n / kTileKeys + 2;
    EGTB_CUDA(cudaMemsetAsync(s.status, 0, tiles * 256 * 8, st));
    EGTB_CUDA(cudaMemsetAsync(s.ustatus, 0, tiles * 8, st));
    EGTB_CUDA(cudaMemsetAsync(s.hist, 0, kMaxPasses * 256 * 4, st));
    EGTB_CUDA(cudaMemsetAsync(s.ctl, 0, sizeof(DevCtl), st));
    EGTB_CUDA(cudaMemsetAsync(s.layer_off, 0, 16, st));
    // the key count goes through the control block, like a layer's candidate count
    const unsigned long long nn = n;
    if (count_by_kernel)
        set_count_kernel<<<1, 1, 0, st>>>(&s.ctl->cand_count[0], nn);
    else
        EGTB_CUDA(cudaMemcpyAsync(&s.ctl->cand_count[0], &nn, sizeof nn, cudaMemcpyHostToDevice, st));
    const SortPlan sp = full_key_plan();
    const unsigned spin_limit = look_back_spin_limit();
    sort_hist_kernel<<<grid, kHistThreads, 0, st>>>(d_in, &s.ctl->cand_count[0], n, sp, s.hist, s.counters, s.ctl);
    // 8 passes: in -> out -> tmp -> out ... -> tmp, then unique tmp -> out
    const uint64_t *src = d_in;
    for (int p = 0; p < sp.passes; ++p) {
        uint64_t *dst = (p % 2 == 0) ? d_out : s.tmp;
        onesweep_kernel<<<grid, kSweepThreads, 0, st>>>(src, dst, &s.ctl->cand_count[0], n, sp, p, s.hist, s.counters,
                                                       s.status, (unsigned)(p + 1), s.ctl, spin_limit);
        src = dst;
    }
    // the output "arena" is d_out; its capacity check rounds up to a 16-key line
    const unsigned long long cap16 = (n + 15) & ~15ull;
    unique_layer_kernel<<<grid, kSortThreads, 0, st>>>(src, 0, n, d_out, s.layer_off, d_n_out, 0, cap16, s.counters,
                                                       s.ustatus, 9u, s.hist, s.ctl, nullptr, spin_limit);
    EGTB_CUDA(cudaGetLastError());
}

static int sweep_grid_for_device() {
    int dev = 0, sms = 0, per_sm = 0;
    EGTB_CUDA(cudaGetDevice(&dev));
    EGTB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EGTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_kernel, kSweepThreads, 0));
    return sms * std::max(1, per_sm);
}

}  // namespace egtb

using namespace egtb;

extern "C" int egtb_sort_unique_u64(int device, const uint64_t *d_keys, size_t n, uint64_t *d_out,
                                    uint64_t *d_n_out, void *stream) {
    return guarded([&] {
        if (n && (!d_keys || !d_out)) throw Error(EGTB_ERR_ARG, "NULL key buffer");
        if (!d_n_out) throw Error(EGTB_ERR_ARG, "NULL count pointer");
        if ((const void *)d_keys == (const void *)d_out && n) throw Error(EGTB_ERR_ARG, "d_out must not alias d_keys");
        if (n >= (1ull << 32)) throw Error(EGTB_ERR_ARG, "at most 2^32-1 keys");
        EGTB_CUDA(cudaSetDevice(device));
        cudaStream_t st = (cudaStream_t)stream;
        unsigned char *base = nullptr;
        EGTB_CUDA(cudaMallocAsync((void **)&base, scratch_bytes(n), st));
        const SortScratch s = carve(base, n);
        enqueue_sort_unique_u64(d_keys, n, d_out, (unsigned long long *)d_n_out, s, sweep_grid_for_device(), st);
        EGTB_CUDA(cudaFreeAsync(base, st));
    });
}

// ------------------------------------------------ allocation-free variant ---
//
// Some callers cannot let a library allocate device memory: processes whose
// device memory is all held by their own pool (a cudaMalloc would fail, or
// force the pool to give memory back), and latency-critical paths that cannot
// afford cudaMalloc/cudaFree, which may synchronise the device. For them,
// egtb_sort_unique_u64_noalloc runs the same sort with its scratch in the
// file-scope array below: kNoAllocMaxKeys keys at most, about 8.6 MB that
// every GPU loading this library holds until the process exits.

namespace egtb {

constexpr size_t kNoAllocMaxKeys = size_t(1) << 20;

// the largest scratch_bytes() the limit needs, rounded to 256 bytes
constexpr size_t kNoAllocTiles = kNoAllocMaxKeys / kTileKeys + 2;
constexpr size_t kNoAllocBytes = ((kNoAllocMaxKeys * 8 + 8 + 255) & ~size_t(255)) +
                                 ((kNoAllocTiles * 256 * 8 + 255) & ~size_t(255)) +
                                 ((kNoAllocTiles * 8 + 255) & ~size_t(255)) +
                                 ((kMaxPasses * 256 * 4 + 255) & ~size_t(255)) + 256 +
                                 ((sizeof(DevCtl) + 255) & ~size_t(255)) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device. In host code the array's
// name only stands in for the symbol, so the address is asked for once per
// device, with that device current. It stays valid while the device's
// context lives: a cudaDeviceReset ends that, and the entry point is not to
// be called on that device afterwards (documented in egtb_gpu.h).
static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[64] = {};
static int g_noalloc_grid[64] = {};

static unsigned char *noalloc_scratch(int device, int *grid) {
    if (device < 0 || device >= 64) throw Error(EGTB_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            throw Error(EGTB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_noalloc_grid[device] = sweep_grid_for_device();
        g_noalloc_ptr[device] = (unsigned char *)ptr;
    }
    *grid = g_noalloc_grid[device];
    return g_noalloc_ptr[device];
}

}  // namespace egtb

extern "C" int egtb_sort_unique_u64_noalloc(int device, const uint64_t *d_keys, size_t n, uint64_t *d_out,
                                            uint64_t *d_n_out, void *stream) {
    return guarded([&] {
        if (n > kNoAllocMaxKeys)
            throw Error(EGTB_ERR_ARG, "n = " + std::to_string(n) + " exceeds the " + std::to_string(kNoAllocMaxKeys) +
                                          "-key limit of egtb_sort_unique_u64_noalloc (use egtb_sort_unique_u64)");
        if (n && (!d_keys || !d_out)) throw Error(EGTB_ERR_ARG, "NULL key buffer");
        if (!d_n_out) throw Error(EGTB_ERR_ARG, "NULL count pointer");
        if ((const void *)d_keys == (const void *)d_out && n) throw Error(EGTB_ERR_ARG, "d_out must not alias d_keys");
        EGTB_CUDA(cudaSetDevice(device));
        int grid = 0;
        unsigned char *base = noalloc_scratch(device, &grid);
        // the look-back words, histograms and control block are cleared by
        // enqueue_sort_unique_u64 itself: the array keeps the last call's contents
        enqueue_sort_unique_u64(d_keys, n, d_out, (unsigned long long *)d_n_out, carve(base, n), grid,
                                (cudaStream_t)stream, /*count_by_kernel=*/true);
    });
}
