// Onesweep LSD radix sort + single-pass unique of a layer's candidates.
//
// Digits are 8 bits made of two free nibbles (nibbles pinned to 0xF in every
// canonical key never vary, so they are not sorted). One kernel computes the
// digit histograms of every pass; each pass is then ONE kernel: a block claims
// the next tile (4096 keys) with an atomic, ranks its keys per digit
// (warp-striped, __match_any_sync), publishes its per-digit counts, looks back
// over the previous tiles' counts (decoupled look-back) for its global digit
// offsets, and scatters through shared memory so global writes run along digit
// runs. The unique kernel keeps the first of every run of equal keys, writes
// them as layer L of the arena (same look-back scheme for the output offset)
// and closes the layer (length, next offset, capacity check).
//
// Every wait on another block is bounded: after spin_limit polls (a kernel
// argument; kSpinLimit unless the host set another limit) the kernel flags
// kErrTimeout and carries on with the counts it has seen, which only moves
// its writes to lower positions inside the same layer (the host reports
// EGTB_ERR_TIMEOUT and the result is not used). A tile
// id is only ever held by a running block, which publishes its own counts
// before it waits, so the waits always end.
#pragma once

#include <cstdint>

#include "egtb_kernels.cuh"

namespace egtb {

constexpr unsigned kErrTimeout = 8u;
constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagPrefix = 2ull << 32;
constexpr unsigned long long kFlagMask = 3ull << 32;
constexpr int kMaxPasses = 8;
constexpr int kCounterUnique = 15;  // tile counter slot of the unique kernel

// Digit layout of every pass: digit = nibble lo | nibble hi << 4 (hi < 0: none).
struct SortPlan {
    int passes;
    int lo[kMaxPasses];
    int hi[kMaxPasses];
};

// status word: [63:34] epoch, [33:32] flag, [31:0] count
__device__ __forceinline__ unsigned long long status_word(unsigned epoch, unsigned long long flag, unsigned count) {
    return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | flag | (unsigned long long)count;
}

__device__ __forceinline__ unsigned sort_digit(uint64_t key, const SortPlan &sp, int p) {
    unsigned d = (unsigned)(key >> (4 * sp.lo[p])) & 0xFu;
    if (sp.hi[p] >= 0) d |= ((unsigned)(key >> (4 * sp.hi[p])) & 0xFu) << 4;
    return d;
}

__device__ __forceinline__ void publish_status(unsigned long long *p, unsigned long long w) {
    *(volatile unsigned long long *)p = w;
}

constexpr int kLookWindow = 4;

// Sum of the counts of tiles tile-1, tile-2, ... back to (and including) the
// nearest one that published its inclusive prefix. Words are at
// base[j * stride]; kLookWindow predecessors are read at once, so a chain of
// tiles that all started together is walked kLookWindow tiles per round trip.
__device__ __forceinline__ unsigned long long look_back(const unsigned long long *base, unsigned long long stride,
                                                        long long tile, unsigned epoch, unsigned spin_limit,
                                                        DevCtl *ctl) {
    const unsigned long long want = (unsigned long long)(epoch & 0x3FFFFFFFu);
    unsigned long long excl = 0;
    long long j = tile - 1;
    unsigned spins = 0;
    while (j >= 0) {
        unsigned long long w[kLookWindow];
#pragma unroll
        for (int q = 0; q < kLookWindow; ++q)
            w[q] = (j - q >= 0) ? *(const volatile unsigned long long *)(base + (unsigned long long)(j - q) * stride) : 0ull;
        int used = 0;
        bool done = false;
#pragma unroll
        for (int q = 0; q < kLookWindow; ++q) {
            if (done || used < q || j - q < 0) continue;
            if ((w[q] >> 34) != want || !(w[q] & kFlagMask)) continue;  // not published yet
            excl += (unsigned)(w[q] & 0xFFFFFFFFull);
            used = q + 1;
            if ((w[q] & kFlagMask) == kFlagPrefix) done = true;
        }
        if (done) return excl;
        j -= used;
        if (used == 0) {
            if (++spins > spin_limit) {
                atomicOr(&ctl->err, kErrTimeout);
                return excl;
            }
            if (spins > 64) __nanosleep(128);
        }
    }
    return excl;
}

// Digit histograms of every pass; also resets the tile counters of the coming
// passes and counts the candidates. Each thread has kHistKeys loads in flight
// (coalesced across the block); a digit shared by the whole warp (common for
// the high nibbles of sorted or clustered keys) is counted with one
// shared-memory atomic, other digits with one atomic per lane.
constexpr int kHistThreads = 512;
constexpr int kHistKeys = 8;

static __global__ void __launch_bounds__(kHistThreads, 2)
sort_hist_kernel(const uint64_t *__restrict__ keys, const unsigned long long *n_ptr, unsigned long long cap, SortPlan sp,
                 unsigned *__restrict__ hist, unsigned *__restrict__ counters, DevCtl *ctl) {
    __shared__ unsigned h[kMaxPasses][256];
    const unsigned long long n = clamp_n(*n_ptr, cap);
    for (int i = threadIdx.x; i < kMaxPasses * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x < 16) counters[threadIdx.x] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->candidates += n;
        ctl->n_sort = n;  // stable copy for the unique kernel, which resets the buffer count
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const unsigned long long span = (unsigned long long)kHistThreads * kHistKeys;
    for (unsigned long long base = (unsigned long long)blockIdx.x * span; base < n; base += (unsigned long long)gridDim.x * span) {
        uint64_t k[kHistKeys];
#pragma unroll
        for (int r = 0; r < kHistKeys; ++r) {
            const unsigned long long i = base + (unsigned long long)r * kHistThreads + threadIdx.x;
            k[r] = i < n ? keys[i] : 0;
        }
#pragma unroll
        for (int r = 0; r < kHistKeys; ++r) {
            const bool valid = base + (unsigned long long)r * kHistThreads + threadIdx.x < n;
            for (int p = 0; p < sp.passes; ++p) {
                const unsigned d = valid ? sort_digit(k[r], sp, p) : 256u;
                const unsigned d0 = __shfl_sync(0xFFFFFFFFu, d, 0);
                if (__all_sync(0xFFFFFFFFu, d == d0)) {
                    if (lane == 0 && d0 < 256u) atomicAdd(&h[p][d0], 32u);
                } else if (valid) {
                    atomicAdd(&h[p][d], 1u);
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < sp.passes * 256; i += blockDim.x) {
        const unsigned c = (&h[0][0])[i];
        if (c) atomicAdd(hist + i, c);
    }
}

// One pass: src -> dst ordered by digit p, stable. 256 threads per 4096-key
// tile (8 warps x 16 rounds of 32 keys), four blocks per SM; each thread owns
// one digit for the look-back. (Two 512-thread blocks per SM measured 4-5 %
// slower: their barriers held more of the SM's warps at once.)
constexpr int kSweepThreads = 256;
constexpr int kSweepWarps = kSweepThreads / 32;
constexpr int kSweepKeys = kTileKeys / kSweepThreads;  // keys per thread

static __global__ void __launch_bounds__(kSweepThreads, 4)
onesweep_kernel(const uint64_t *__restrict__ src, uint64_t *__restrict__ dst, const unsigned long long *n_ptr,
                unsigned long long cap, SortPlan sp, int p, const unsigned *__restrict__ hist,
                unsigned *__restrict__ counters, unsigned long long *__restrict__ status, unsigned epoch, DevCtl *ctl,
                unsigned spin_limit) {
    __shared__ uint64_t tkeys[kTileKeys];
    __shared__ unsigned short wcnt[kSweepWarps][256];
    __shared__ unsigned loff[256];
    __shared__ unsigned long long gbase[256];
    __shared__ unsigned ghist[256];
    __shared__ unsigned long long sm[33];
    __shared__ unsigned tile_sh;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int d = threadIdx.x;  // digit owned by this thread when d < 256
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    {
        // start of every digit in the output (same in every block)
        unsigned long long tot;
        const unsigned long long h = d < 256 ? hist[p * 256 + d] : 0ull;
        const unsigned long long ex = block_excl_scan<unsigned long long>(h, sm, &tot);
        if (d < 256) ghist[d] = (unsigned)ex;
    }
    for (;;) {
        if (threadIdx.x == 0) tile_sh = atomicAdd(&counters[p], 1u);
        for (int i = threadIdx.x; i < kSweepWarps * 256; i += kSweepThreads) (&wcnt[0][0])[i] = 0;
        __syncthreads();
        const unsigned long long tile = tile_sh;
        if (tile >= ntiles) break;
        const unsigned long long base = tile * kTileKeys + (unsigned long long)warp * (kTileKeys / kSweepWarps);
        uint64_t k[kSweepKeys];
        unsigned rd[kSweepKeys];  // rank in the warp (low 16 bits) | digit << 16 (256 = no key)
        // all loads first, so a thread has its reads in flight together
#pragma unroll
        for (int r = 0; r < kSweepKeys; ++r) {
            const unsigned long long idx = base + (unsigned long long)r * 32 + lane;
            k[r] = idx < n ? src[idx] : 0;
        }
#pragma unroll
        for (int r = 0; r < kSweepKeys; ++r) {
            const unsigned long long idx = base + (unsigned long long)r * 32 + lane;
            const bool valid = idx < n;
            const unsigned dg = valid ? sort_digit(k[r], sp, p) : 256u;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, dg);
            const unsigned before = __popc(peers & ((1u << lane) - 1u));
            unsigned c = 0;
            if (valid) c = wcnt[warp][dg];
            rd[r] = (c + before) | (dg << 16);
            __syncwarp();
            if (valid && before == 0) wcnt[warp][dg] = (unsigned short)(c + __popc(peers));
            __syncwarp();
        }
        __syncthreads();
        unsigned cnt = 0;
        unsigned long long excl = 0;
        if (d < 256) {
#pragma unroll
            for (int w = 0; w < kSweepWarps; ++w) {
                const unsigned c = wcnt[w][d];
                wcnt[w][d] = (unsigned short)cnt;
                cnt += c;
            }
            // publish this tile's count, then look back for the counts before it
            unsigned long long *my = status + tile * 256 + d;
            if (tile == 0) {
                publish_status(my, status_word(epoch, kFlagPrefix, cnt));
            } else {
                publish_status(my, status_word(epoch, kFlagAgg, cnt));
                excl = look_back(status + d, 256, (long long)tile, epoch, spin_limit, ctl);
                publish_status(my, status_word(epoch, kFlagPrefix, (unsigned)(excl + cnt)));
            }
            gbase[d] = (unsigned long long)ghist[d] + excl;
        }
        {
            unsigned long long tot;
            const unsigned long long lo = block_excl_scan<unsigned long long>((unsigned long long)cnt, sm, &tot);
            if (d < 256) loff[d] = (unsigned)lo;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kSweepKeys; ++r) {
            const unsigned dg = rd[r] >> 16;
            if (dg < 256u) tkeys[loff[dg] + wcnt[warp][dg] + (rd[r] & 0xFFFFu)] = k[r];
        }
        __syncthreads();
        const unsigned long long rem = n - tile * kTileKeys;
        const unsigned tile_n = rem < (unsigned long long)kTileKeys ? (unsigned)rem : (unsigned)kTileKeys;
        for (unsigned i = threadIdx.x; i < tile_n; i += kSweepThreads) {
            const uint64_t key = tkeys[i];
            const unsigned dg = sort_digit(key, sp, p);
            dst[gbase[dg] + (i - loff[dg])] = key;
        }
        __syncthreads();
    }
}

// ------------------------------------------- per-layer (segmented) sort ----
//
// Every layer of the arena sorted in place of its own region, by its free
// nibbles only (the other nibbles are 0xF in every key of a layer): tiles of
// kTileKeys keys never straddle two layers (tile_layer[j] is tile j's layer,
// layer_tile0[L] the first tile of layer L), each layer has its own digit
// histograms (hist_l[(L * kMaxPasses + p) * 256 + d]) and its own digit
// positions (seg_nib[L * kMaxPasses + p]: the less significant nibble in the
// low byte, the more significant one in the high byte, 0xFF for none, so the
// layers of tables with different free cells sort together), and the
// look-back of a tile stops at its layer's first tile, which publishes its
// counts as a prefix. The layer digits of a composite (layer, key) sort are
// not needed.

__device__ __forceinline__ unsigned seg_digit(uint64_t key, unsigned nib2) {
    const unsigned lo = nib2 & 0xFFu, hi = nib2 >> 8;
    unsigned d = lo != 0xFFu ? (unsigned)(key >> (4 * lo)) & 0xFu : 0u;
    if (hi != 0xFFu) d |= ((unsigned)(key >> (4 * hi)) & 0xFu) << 4;
    return d;
}

// A tile's layer, its first key in the arena and its key count.
struct SegTile {
    int layer;
    unsigned long long first;
    unsigned n;
    bool head;  // first tile of its layer
};

__device__ __forceinline__ SegTile seg_tile(unsigned tile, const int *__restrict__ tile_layer,
                                            const int *__restrict__ layer_tile0,
                                            const unsigned long long *__restrict__ layer_off,
                                            const unsigned long long *__restrict__ layer_len) {
    SegTile t;
    t.layer = tile_layer[tile];
    const unsigned lt = tile - (unsigned)layer_tile0[t.layer];
    const unsigned long long done = (unsigned long long)lt * kTileKeys;
    const unsigned long long rem = layer_len[t.layer] - done;
    t.first = layer_off[t.layer] + done;
    t.n = rem < (unsigned long long)kTileKeys ? (unsigned)rem : (unsigned)kTileKeys;
    t.head = lt == 0;
    return t;
}

// Digit histograms of every pass, per layer. Block b takes a contiguous run
// of tiles (mostly of one layer) and adds its counts to the layer's
// histograms when the layer changes. Also resets the tile counters.
static __global__ void __launch_bounds__(kHistThreads, 2)
seg_hist_kernel(const uint64_t *__restrict__ keys, const int *__restrict__ tile_layer,
                const int *__restrict__ layer_tile0, const unsigned long long *__restrict__ layer_off,
                const unsigned long long *__restrict__ layer_len, unsigned ntiles, int passes,
                const unsigned short *__restrict__ seg_nib, unsigned *__restrict__ hist_l,
                unsigned *__restrict__ counters) {
    __shared__ unsigned h[kMaxPasses][256];
    __shared__ unsigned nib[kMaxPasses];
    for (int i = threadIdx.x; i < kMaxPasses * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x < 16) counters[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const unsigned per = (ntiles + gridDim.x - 1) / gridDim.x;
    const unsigned t0 = blockIdx.x * per;
    const unsigned t1 = t0 + per < ntiles ? t0 + per : ntiles;
    int cur = -1;
    auto flush = [&]() {
        __syncthreads();
        unsigned *out = hist_l + (size_t)cur * kMaxPasses * 256;
        for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
            const unsigned c = (&h[0][0])[i];
            if (c) {
                atomicAdd(out + i, c);
                (&h[0][0])[i] = 0;
            }
        }
        __syncthreads();
    };
    for (unsigned tile = t0; tile < t1; ++tile) {
        const SegTile t = seg_tile(tile, tile_layer, layer_tile0, layer_off, layer_len);
        if (t.layer != cur) {
            if (cur >= 0) flush();
            cur = t.layer;
            if (threadIdx.x < kMaxPasses) nib[threadIdx.x] = seg_nib[(size_t)cur * kMaxPasses + threadIdx.x];
            __syncthreads();
        }
        uint64_t k[kHistKeys];
#pragma unroll
        for (int r = 0; r < kHistKeys; ++r) {
            const unsigned i = (unsigned)r * kHistThreads + threadIdx.x;
            k[r] = i < t.n ? keys[t.first + i] : 0;
        }
#pragma unroll
        for (int r = 0; r < kHistKeys; ++r) {
            const bool valid = (unsigned)r * kHistThreads + threadIdx.x < t.n;
            for (int p = 0; p < passes; ++p) {
                const unsigned d = valid ? seg_digit(k[r], nib[p]) : 256u;
                const unsigned d0 = __shfl_sync(0xFFFFFFFFu, d, 0);
                if (__all_sync(0xFFFFFFFFu, d == d0)) {
                    if (lane == 0 && d0 < 256u) atomicAdd(&h[p][d0], 32u);
                } else if (valid) {
                    atomicAdd(&h[p][d], 1u);
                }
            }
        }
    }
    if (cur >= 0) flush();
}

// ---------------------------------------------- bulk copies into smem ----
//
// The per-layer sort reads each tile with one bulk asynchronous copy
// (cp.async.bulk into this block's own shared memory, no tensor map) completed on an mbarrier, so
// the next tile's keys arrive while the block writes out the current one.

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Orders this thread's shared-memory accesses before later bulk copies (and
// an mbarrier's initialisation before the copies that complete on it).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bytes (a multiple of 16) from global src (16-byte aligned) into shared dst
// (16-byte aligned), counted on bar.
__device__ __forceinline__ void bulk_load_smem(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Polls of an mbarrier wait for a bulk copy; a copy of one tile lands within
// microseconds, so running out means the copy engine failed: kErrTimeout.
constexpr unsigned kBulkWaitPolls = 1u << 24;

__device__ __forceinline__ void mbar_wait_bounded(unsigned long long *bar, unsigned parity, DevCtl *ctl) {
    for (unsigned spins = 0; !mbar_try_wait(bar, parity);) {
        if (++spins == kBulkWaitPolls) atomicOr(&ctl->err, kErrTimeout);
        if (spins >= 2 * kBulkWaitPolls) return;  // the result is not used (the host reports the timeout)
    }
}

// Dynamic shared memory of seg_onesweep_kernel: the tile as read, the tile in
// digit order and the digit of every key of the latter.
constexpr int kSegSweepSmem = 2 * kTileKeys * (int)sizeof(uint64_t) + kTileKeys;

// One pass of the per-layer sort: src -> dst (same layout) ordered by digit p
// within every layer, stable. The same tile work as onesweep_kernel, with
// the keys read into shared memory by a bulk copy that is issued as soon as
// the previous tile's keys are scattered (a tile of n keys reads n rounded up
// to even keys: layer regions start 16-key aligned and are padded to 16 keys,
// so the rounded read stays inside the tile's layer region).
static __global__ void __launch_bounds__(kSweepThreads, 3)
seg_onesweep_kernel(const uint64_t *__restrict__ src, uint64_t *__restrict__ dst, const int *__restrict__ tile_layer,
                    const int *__restrict__ layer_tile0, const unsigned long long *__restrict__ layer_off,
                    const unsigned long long *__restrict__ layer_len, unsigned ntiles,
                    const unsigned short *__restrict__ seg_nib, int p, const unsigned *__restrict__ hist_l,
                    unsigned *__restrict__ counters,
                    unsigned long long *__restrict__ status, unsigned epoch, DevCtl *ctl, unsigned spin_limit) {
    extern __shared__ __align__(128) uint64_t seg_smem[];
    uint64_t *const in = seg_smem, *const tkeys = seg_smem + kTileKeys;
    unsigned char *const tdig = reinterpret_cast<unsigned char *>(seg_smem + 2 * kTileKeys);
    // per warp and digit: the warp's count, then the tile position of its first key of the digit
    __shared__ unsigned short wcnt[kSweepWarps][256];
    __shared__ unsigned long long gdelta[256];  // destination of tile position i (digit d): gdelta[d] + i
    __shared__ unsigned long long sm[33];
    __shared__ unsigned tile_sh;
    __shared__ __align__(8) unsigned long long full;  // completes when a tile's keys are in `in`
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int d = threadIdx.x;  // digit owned by this thread when d < 256
    // thread 0: claim the next tile and start reading its keys
    auto claim = [&]() {
        const unsigned tile = atomicAdd(&counters[p], 1u);
        tile_sh = tile;
        if (tile < ntiles) {
            const SegTile t = seg_tile(tile, tile_layer, layer_tile0, layer_off, layer_len);
            const unsigned bytes = ((t.n + 1u) & ~1u) * (unsigned)sizeof(uint64_t);
            mbar_arrive_expect_tx(&full, bytes);
            bulk_load_smem(in, src + t.first, bytes, &full);
        }
    };
    if (threadIdx.x == 0) {
        mbar_init(&full, 1);
        fence_proxy_async_smem();
        claim();
    }
    unsigned parity = 0;
    for (;;) {
        for (int i = threadIdx.x; i < kSweepWarps * 256; i += kSweepThreads) (&wcnt[0][0])[i] = 0;
        __syncthreads();
        const unsigned tile = tile_sh;
        if (tile >= ntiles) break;
        const SegTile t = seg_tile(tile, tile_layer, layer_tile0, layer_off, layer_len);
        const unsigned nib2 = seg_nib[(size_t)t.layer * kMaxPasses + p];
        // start of every digit of this layer in the layer's region
        unsigned long long ghist_d;
        {
            unsigned long long tot;
            const unsigned long long hd = d < 256 ? hist_l[((size_t)t.layer * kMaxPasses + p) * 256 + d] : 0ull;
            ghist_d = block_excl_scan<unsigned long long>(hd, sm, &tot);
        }
        mbar_wait_bounded(&full, parity, ctl);
        parity ^= 1u;
        const unsigned base = (unsigned)warp * (kTileKeys / kSweepWarps);
        unsigned rd[kSweepKeys];  // rank in the warp (low 16 bits) | digit << 16 (256 = no key)
#pragma unroll
        for (int r = 0; r < kSweepKeys; ++r) {
            const unsigned idx = base + (unsigned)r * 32 + lane;
            const bool valid = idx < t.n;
            const unsigned dg = valid ? seg_digit(in[idx], nib2) : 256u;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, dg);
            const unsigned before = __popc(peers & ((1u << lane) - 1u));
            unsigned c = 0;
            if (valid) c = wcnt[warp][dg];
            rd[r] = (c + before) | (dg << 16);
            __syncwarp();
            if (valid && before == 0) wcnt[warp][dg] = (unsigned short)(c + __popc(peers));
            __syncwarp();
        }
        __syncthreads();
        unsigned cnt = 0;
        unsigned long long excl = 0;
        if (d < 256) {
#pragma unroll
            for (int w = 0; w < kSweepWarps; ++w) {
                const unsigned c = wcnt[w][d];
                wcnt[w][d] = (unsigned short)cnt;
                cnt += c;
            }
            unsigned long long *my = status + (size_t)tile * 256 + d;
            if (t.head) {
                publish_status(my, status_word(epoch, kFlagPrefix, cnt));
            } else {
                publish_status(my, status_word(epoch, kFlagAgg, cnt));
                // stops at the first prefix: at the latest the layer's first tile
                excl = look_back(status + d, 256, (long long)tile, epoch, spin_limit, ctl);
                publish_status(my, status_word(epoch, kFlagPrefix, (unsigned)(excl + cnt)));
            }
        }
        {
            unsigned long long tot;
            const unsigned long long lo = block_excl_scan<unsigned long long>((unsigned long long)cnt, sm, &tot);
            if (d < 256) {
                // modular: gdelta[d] + i for i >= lo is the key's destination
                gdelta[d] = layer_off[t.layer] + ghist_d + excl - lo;
#pragma unroll
                for (int w = 0; w < kSweepWarps; ++w) wcnt[w][d] = (unsigned short)(wcnt[w][d] + lo);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kSweepKeys; ++r) {
            const unsigned dg = rd[r] >> 16;
            if (dg < 256u) {
                const unsigned pos = wcnt[warp][dg] + (rd[r] & 0xFFFFu);
                tkeys[pos] = in[base + (unsigned)r * 32 + lane];
                tdig[pos] = (unsigned char)dg;
            }
        }
        __syncthreads();
        // `in` is free: the next tile's keys load while this one is written out
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            claim();
        }
        for (unsigned i = threadIdx.x; i < t.n; i += kSweepThreads) dst[gdelta[tdig[i]] + i] = tkeys[i];
    }
}

// Copy every layer's keys (tile by tile) from src to dst.
static __global__ void __launch_bounds__(256)
seg_copy_kernel(const uint64_t *__restrict__ src, uint64_t *__restrict__ dst, const int *__restrict__ tile_layer,
                const int *__restrict__ layer_tile0, const unsigned long long *__restrict__ layer_off,
                const unsigned long long *__restrict__ layer_len, unsigned ntiles) {
    for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const SegTile t = seg_tile(tile, tile_layer, layer_tile0, layer_off, layer_len);
        for (unsigned i = threadIdx.x; i < t.n; i += blockDim.x) dst[t.first + i] = src[t.first + i];
    }
}

// Unique + layer write + layer close, single pass. keys: sorted candidates
// of buffer x; layer L goes to arena[layer_off[L] ..]. The last tile records
// layer_len[L] and the next 16-aligned offset, resets the buffer's count and
// the histograms for the next sort, and reports progress.
static __global__ void __launch_bounds__(kSortThreads)
unique_layer_kernel(const uint64_t *__restrict__ keys, int x, unsigned long long cap, uint64_t *__restrict__ arena,
                    unsigned long long *__restrict__ layer_off, unsigned long long *__restrict__ layer_len, int L,
                    unsigned long long arena_cap, unsigned *__restrict__ counters,
                    unsigned long long *__restrict__ ustatus, unsigned epoch, unsigned *__restrict__ hist,
                    DevCtl *ctl, unsigned *progress, unsigned spin_limit) {
    __shared__ unsigned long long sm[33];
    __shared__ unsigned tile_sh;
    __shared__ unsigned long long excl_sh;
    const unsigned long long n = clamp_n(ctl->n_sort, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    const unsigned long long off = layer_off[L];
    auto close = [&](unsigned long long total) {
        const unsigned long long end = off + total;
        const unsigned long long next = (end + kSplitStride - 1) & ~(unsigned long long)(kSplitStride - 1);
        if (next > arena_cap || (ctl->err & kErrArenaOverflow)) {
            atomicOr(&ctl->err, kErrArenaOverflow);
            layer_len[L] = 0;
            layer_off[L + 1] = off;
        } else {
            layer_len[L] = total;
            layer_off[L + 1] = next;
        }
        ctl->cand_count[x] = 0;
        for (int i = 0; i < kMaxPasses * 256; ++i) hist[i] = 0;
        if (progress) *(volatile unsigned *)progress = (unsigned)L;
    };
    if (ntiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) close(0);
        return;
    }
    for (;;) {
        if (threadIdx.x == 0) tile_sh = atomicAdd(&counters[kCounterUnique], 1u);
        __syncthreads();
        const unsigned long long tile = tile_sh;
        if (tile >= ntiles) break;
        const unsigned long long base = tile * kTileKeys + (unsigned long long)threadIdx.x * kKeysPerThread;
        uint64_t k[kKeysPerThread];
        unsigned head = 0, c = 0;
        uint64_t prev = (base > 0 && base < n) ? keys[base - 1] : 0;
#pragma unroll
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + i;
            k[i] = idx < n ? keys[idx] : 0;
            const bool hd = idx < n && (idx == 0 || k[i] != prev);
            prev = k[i];
            head |= (unsigned)hd << i;
            c += hd;
        }
        unsigned long long tile_total;
        const unsigned long long local = block_excl_scan<unsigned long long>((unsigned long long)c, sm, &tile_total);
        if (threadIdx.x == 0) {
            unsigned long long *my = ustatus + tile;
            unsigned long long excl = 0;
            if (tile == 0) {
                publish_status(my, status_word(epoch, kFlagPrefix, (unsigned)tile_total));
            } else {
                publish_status(my, status_word(epoch, kFlagAgg, (unsigned)tile_total));
                excl = look_back(ustatus, 1, (long long)tile, epoch, spin_limit, ctl);
                publish_status(my, status_word(epoch, kFlagPrefix, (unsigned)(excl + tile_total)));
            }
            excl_sh = excl;
            if (tile == ntiles - 1) close(excl + tile_total);
        }
        __syncthreads();
        unsigned long long pos = excl_sh + local;
#pragma unroll
        for (int i = 0; i < kKeysPerThread; ++i) {
            if (head >> i & 1u) {
                const unsigned long long g = off + pos;
                if (g < arena_cap) arena[g] = k[i];
                ++pos;
            }
        }
        __syncthreads();
    }
}

}  // namespace egtb
