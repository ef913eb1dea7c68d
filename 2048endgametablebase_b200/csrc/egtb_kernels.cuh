// Build kernels of the classic tablebase path: forward expand, LSD radix
// sort, unique + compaction into the layer arena, backward solve and book
// packing. Sizes live in device memory (layer offsets/lengths, candidate
// counters), so a whole build can be enqueued without host round trips;
// every kernel runs a fixed grid that loops over its work.
#pragma once

#include <cstdint>

#include "egtb_device.cuh"

namespace egtb {

// error flags (DevCtl::err)
constexpr unsigned kErrCandOverflow = 1u;
constexpr unsigned kErrArenaOverflow = 2u;
constexpr unsigned kErrBookOverflow = 4u;

constexpr int kTileKeys = 4096;     // keys per sort / compaction tile
constexpr int kSortThreads = 256;   // 8 warps x 16 keys x 32 lanes
constexpr int kKeysPerThread = kTileKeys / kSortThreads;

// Control block in device memory.
struct DevCtl {
    unsigned long long cand_count[2];   // keys in the two candidate buffers
    unsigned long long n_sort;          // keys handed to the sort
    unsigned long long n_unique;        // result of the last unique / compaction
    unsigned long long candidates;      // statistics: keys that reached a sort
    unsigned long long lookups;         // statistics: exact searches in the backward pass
    unsigned int err;
    unsigned int pad;
};

__device__ __forceinline__ unsigned long long clamp_n(unsigned long long n, unsigned long long cap) {
    return n < cap ? n : cap;
}

// ----------------------------------------------------------- scans -------

__device__ __forceinline__ unsigned warp_incl_scan(unsigned v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_incl_scan64(unsigned long long v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total in *total.
// smem: at least blockDim.x/32 entries.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *smem, T *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T inc;
    if constexpr (sizeof(T) == 8) inc = warp_incl_scan64(v); else inc = warp_incl_scan(v);
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nw ? smem[lane] : T(0);
        T wi;
        if constexpr (sizeof(T) == 8) wi = warp_incl_scan64(w); else wi = warp_incl_scan(w);
        if (lane < nw) smem[lane] = wi - w;
        if (lane == nw - 1) smem[32] = wi;
    }
    __syncthreads();
    T r = smem[warp] + inc - v;
    *total = smem[32];
    __syncthreads();
    return r;
}

// --------------------------------------------------------- expand --------

constexpr int kExpandThreads = 256;
constexpr int kStage = 64;  // per-warp staging slots per stream

// Flush a warp's staging buffer to its candidate stream.
__device__ __forceinline__ void stage_flush(uint64_t *stage, int &count, uint64_t *__restrict__ out,
                                            unsigned long long *cnt, unsigned long long cap, unsigned *err) {
    const int lane = threadIdx.x & 31;
    if (count == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(cnt, (unsigned long long)count);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base + (unsigned long long)count > cap) {
        if (lane == 0) atomicOr(err, kErrCandOverflow);
    } else {
        for (int i = lane; i < count; i += 32) out[base + i] = stage[i];
    }
    __syncwarp();
    count = 0;
}

// Forward expand of layer t (gen_boards_*, native_core/src/BookGenerator.cpp:
// 472-760): every parent, unless do_check and it is a success, every empty
// nibble k ascending, spawn 2 (v=1) and 4 (v=2), the four moves; a child is
// kept when it moved and matches the pattern, and is emitted canonicalised:
// v=1 children to the stream of layer t+1, v=2 children to the stream of
// layer t+2. A direct-mapped table drops most repeats before they reach the
// sort (its role is the reference's lossy prefilter, BookGenerator.cpp:
// 101-127; results never depend on it). Each warp stages its survivors in
// shared memory and appends them with one atomic per 32+ keys.
__global__ void __launch_bounds__(kExpandThreads)
expand_kernel(const uint64_t *__restrict__ arena, const unsigned long long *__restrict__ layer_off,
              const unsigned long long *__restrict__ layer_len, int t, DevSpec spec, int do_check,
              const uint32_t *__restrict__ tab, uint64_t *__restrict__ out1, uint64_t *__restrict__ out2,
              DevCtl *ctl, int which1, int which2, unsigned long long cap, uint64_t *filter, int filter_bits) {
    __shared__ uint64_t stage[kExpandThreads / 32][2][kStage];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (ctl->err & kErrArenaOverflow) return;
    const unsigned long long n = layer_len[t];
    const uint64_t *par = arena + layer_off[t];
    int cnt[2] = {0, 0};
    uint64_t *outs[2] = {out1, out2};
    unsigned long long *counters[2] = {&ctl->cand_count[which1], &ctl->cand_count[which2]};
    const unsigned long long nwarps = (unsigned long long)gridDim.x * (kExpandThreads / 32);
    for (unsigned long long base = ((unsigned long long)blockIdx.x * (kExpandThreads / 32) + warp) * 32; base < n;
         base += nwarps * 32) {
        const unsigned long long p = base + lane;
        bool active = p < n;
        uint64_t b = active ? par[p] : 0;
        if (active && do_check && is_success(b, spec)) active = false;
        uint64_t empt = active ? empty_nibbles(b) : 0;
        MoveCtx mc;
        move_ctx_init(tab, b, mc);
        unsigned any = __ballot_sync(0xFFFFFFFFu, empt != 0);
        while (any) {
            // next empty nibble of this lane (lanes advance independently; the
            // loop runs while any lane still has one)
            int k = -1;
            if (empt) {
                k = (__ffsll((long long)empt) - 1) >> 2;
                empt &= empt - 1;
            }
#pragma unroll
            for (int v = 1; v <= 2; ++v) {
                uint64_t mv[4], s = 0;
                if (k >= 0) spawn_moves(tab, mc, k, (uint64_t)v, s, mv);
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    bool keep = k >= 0 && mv[d] != s && is_pattern(mv[d], spec);
                    uint64_t key = 0;
                    if (keep) {
                        key = canonical(mv[d], spec.symm);
                        const uint64_t slot = filter_slot(key, filter_bits);
                        if (filter[slot] == key) keep = false;
                        else filter[slot] = key;
                    }
                    const unsigned m = __ballot_sync(0xFFFFFFFFu, keep);
                    if (m) {
                        const int pos = cnt[v - 1] + __popc(m & ((1u << lane) - 1u));
                        if (keep) stage[warp][v - 1][pos] = key;
                        cnt[v - 1] += __popc(m);
                        __syncwarp();
                        if (cnt[v - 1] > kStage - 32)
                            stage_flush(stage[warp][v - 1], cnt[v - 1], outs[v - 1], counters[v - 1], cap, &ctl->err);
                    }
                }
            }
            any = __ballot_sync(0xFFFFFFFFu, empt != 0);
        }
    }
    stage_flush(stage[warp][0], cnt[0], out1, counters[0], cap, &ctl->err);
    stage_flush(stage[warp][1], cnt[1], out2, counters[1], cap, &ctl->err);
}

// -------------------------------------------------- LSD radix sort -------
//
// One 8-bit digit per pass; only the bytes that can differ between keys are
// sorted (bytes made of pinned nibbles are constant). Each pass is three
// kernels: per-tile digit counts, a digit-major scan of those counts, and a
// stable scatter (warp-striped ranking with __match_any_sync, tile staged in
// shared memory so the global writes run along digit runs).

__global__ void __launch_bounds__(kSortThreads)
radix_count_kernel(const uint64_t *__restrict__ keys, const unsigned long long *n_ptr, unsigned long long cap,
                   int shift, unsigned *__restrict__ tile_hist, unsigned long long max_tiles,
                   unsigned *__restrict__ digit_tot) {
    __shared__ unsigned hist[256];
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        hist[threadIdx.x] = 0;
        __syncthreads();
        const unsigned long long base = tile * kTileKeys;
#pragma unroll 4
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + (unsigned long long)i * kSortThreads + threadIdx.x;
            if (idx < n) atomicAdd(&hist[(unsigned)(keys[idx] >> shift) & 0xFFu], 1u);
        }
        __syncthreads();
        const unsigned c = hist[threadIdx.x];
        tile_hist[(unsigned long long)threadIdx.x * max_tiles + tile] = c;
        if (c) atomicAdd(&digit_tot[threadIdx.x], c);
        __syncthreads();
    }
}

// One block per digit: offset of (digit, tile) = keys of smaller digits +
// keys of this digit in earlier tiles.
__global__ void __launch_bounds__(1024)
radix_scan_kernel(const unsigned long long *n_ptr, unsigned long long cap, unsigned *__restrict__ tile_hist,
                  unsigned long long max_tiles, const unsigned *__restrict__ digit_tot) {
    __shared__ unsigned long long sm[33];
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    const int d = blockIdx.x;
    unsigned long long tot = 0;
    unsigned *row = tile_hist + (unsigned long long)d * max_tiles;
    unsigned long long run = 0;
    for (unsigned long long c0 = 0; c0 < ntiles; c0 += blockDim.x) {
        const unsigned long long i = c0 + threadIdx.x;
        unsigned long long x = i < ntiles ? row[i] : 0;
        unsigned long long ex = block_excl_scan<unsigned long long>(x, sm, &tot);
        // offset inside the digit (candidate buffers hold < 2^32 keys); the
        // scatter adds the 64-bit start of the digit
        if (i < ntiles) row[i] = (unsigned)(run + ex);
        run += tot;
    }
}

__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out, const unsigned long long *n_ptr,
                     unsigned long long cap, int shift, const unsigned *__restrict__ tile_off,
                     unsigned long long max_tiles, const unsigned *__restrict__ digit_tot) {
    __shared__ uint64_t tkeys[kTileKeys];
    __shared__ unsigned short wcnt[kSortThreads / 32][256];
    __shared__ unsigned loff[256];
    __shared__ unsigned long long dbase[256];
    __shared__ unsigned long long sm[33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    {
        // 64-bit start of every digit in the output
        unsigned long long tot;
        unsigned long long v = digit_tot[threadIdx.x];
        unsigned long long ex = block_excl_scan<unsigned long long>(v, sm, &tot);
        dbase[threadIdx.x] = ex;
    }
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int i = threadIdx.x; i < (kSortThreads / 32) * 256; i += kSortThreads) (&wcnt[0][0])[i] = 0;
        __syncthreads();
        const unsigned long long base = tile * kTileKeys + (unsigned long long)warp * (kTileKeys / 8);
        uint64_t k[kKeysPerThread];
        unsigned short rank[kKeysPerThread];
        unsigned short dig[kKeysPerThread];
#pragma unroll
        for (int r = 0; r < kKeysPerThread; ++r) {
            const unsigned long long idx = base + (unsigned long long)r * 32 + lane;
            const bool valid = idx < n;
            k[r] = valid ? in[idx] : 0;
            const unsigned d = valid ? (unsigned)(k[r] >> shift) & 0xFFu : 256u;
            dig[r] = (unsigned short)d;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
            const unsigned before = __popc(peers & ((1u << lane) - 1u));
            unsigned short c = 0;
            if (valid) c = wcnt[warp][d];
            rank[r] = (unsigned short)(c + before);
            __syncwarp();
            if (valid && before == 0) wcnt[warp][d] = (unsigned short)(c + __popc(peers));
            __syncwarp();
        }
        __syncthreads();
        // per digit: warp offsets and tile total
        {
            const int d = threadIdx.x;
            unsigned s = 0;
#pragma unroll
            for (int w = 0; w < kSortThreads / 32; ++w) {
                unsigned c = wcnt[w][d];
                wcnt[w][d] = (unsigned short)s;
                s += c;
            }
            unsigned long long tot;
            unsigned long long ex = block_excl_scan<unsigned long long>((unsigned long long)s, sm, &tot);
            loff[d] = (unsigned)ex;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kKeysPerThread; ++r) {
            const unsigned d = dig[r];
            if (d < 256u) tkeys[loff[d] + wcnt[warp][d] + rank[r]] = k[r];
        }
        __syncthreads();
        const unsigned long long tile_n = (n - tile * kTileKeys) < (unsigned long long)kTileKeys
                                              ? (n - tile * kTileKeys) : (unsigned long long)kTileKeys;
        for (unsigned i = threadIdx.x; i < tile_n; i += kSortThreads) {
            const uint64_t key = tkeys[i];
            const unsigned d = (unsigned)(key >> shift) & 0xFFu;
            const unsigned long long dst =
                dbase[d] + (unsigned long long)tile_off[(unsigned long long)d * max_tiles + tile] + (i - loff[d]);
            out[dst] = key;
        }
        __syncthreads();
    }
}

// ------------------------------------------- unique / compaction ---------

// Per tile: number of positions i with keys[i] != keys[i-1] (i = 0 counts).
__global__ void __launch_bounds__(kSortThreads)
unique_count_kernel(const uint64_t *__restrict__ keys, const unsigned long long *n_ptr, unsigned long long cap,
                    unsigned *__restrict__ tile_cnt) {
    __shared__ unsigned long long sm[33];
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        unsigned long long c = 0;
        const unsigned long long base = tile * kTileKeys + (unsigned long long)threadIdx.x * kKeysPerThread;
        uint64_t prev = (base > 0 && base < n) ? keys[base - 1] : ~keys[0];
#pragma unroll
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + i;
            if (idx < n) {
                const uint64_t k = keys[idx];
                c += (idx == 0 || k != prev);
                prev = k;
            }
        }
        unsigned long long tot;
        block_excl_scan<unsigned long long>(c, sm, &tot);
        if (threadIdx.x == 0) tile_cnt[tile] = (unsigned)tot;
    }
}

// Single block: exclusive scan of the tile counts; total -> *total_out.
__global__ void __launch_bounds__(1024)
tile_scan_kernel(const unsigned long long *n_ptr, unsigned long long cap, unsigned long long *__restrict__ tile_io,
                 const unsigned *__restrict__ tile_cnt, unsigned long long *total_out) {
    __shared__ unsigned long long sm[33];
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    unsigned long long run = 0, tot;
    for (unsigned long long c0 = 0; c0 < ntiles; c0 += blockDim.x) {
        const unsigned long long i = c0 + threadIdx.x;
        unsigned long long x = i < ntiles ? tile_cnt[i] : 0;
        unsigned long long ex = block_excl_scan<unsigned long long>(x, sm, &tot);
        if (i < ntiles) tile_io[i] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) *total_out = run;
}

// Close a new layer: record its length and the next layer's 16-aligned offset.
__global__ void close_layer_kernel(int t, const unsigned long long *total, unsigned long long *layer_off,
                                   unsigned long long *layer_len, unsigned long long arena_cap, DevCtl *ctl) {
    const unsigned long long n = *total;
    const unsigned long long end = layer_off[t] + n;
    const unsigned long long next = (end + kSplitStride - 1) & ~(unsigned long long)(kSplitStride - 1);
    if (next > arena_cap || (ctl->err & kErrArenaOverflow)) {
        // does not fit: flag it and leave the layer empty, so every later
        // kernel of this pass stays inside the arena; the host re-runs the
        // pass with a larger arena
        atomicOr(&ctl->err, kErrArenaOverflow);
        layer_len[t] = 0;
        layer_off[t + 1] = layer_off[t];
        return;
    }
    layer_len[t] = n;
    layer_off[t + 1] = next;
}

// Write the unique keys of a sorted run as layer t of the arena, with the
// layer's splitters (every 16th key).
__global__ void __launch_bounds__(kSortThreads)
unique_write_kernel(const uint64_t *__restrict__ keys, const unsigned long long *n_ptr, unsigned long long cap,
                    const unsigned long long *__restrict__ tile_off, uint64_t *__restrict__ arena,
                    uint64_t *__restrict__ split, const unsigned long long *__restrict__ layer_off, int t,
                    unsigned long long arena_cap) {
    __shared__ unsigned long long sm[33];
    const unsigned long long n = clamp_n(*n_ptr, cap);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    const unsigned long long off = layer_off[t];
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const unsigned long long base = tile * kTileKeys + (unsigned long long)threadIdx.x * kKeysPerThread;
        uint64_t k[kKeysPerThread];
        unsigned head = 0, c = 0;
        uint64_t prev = (base > 0 && base < n) ? keys[base - 1] : 0;
#pragma unroll
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + i;
            k[i] = idx < n ? keys[idx] : 0;
            const bool h = idx < n && (idx == 0 || k[i] != prev);
            prev = k[i];
            head |= (unsigned)h << i;
            c += h;
        }
        unsigned long long tot;
        unsigned long long pos = tile_off[tile] + block_excl_scan<unsigned long long>(c, sm, &tot);
#pragma unroll
        for (int i = 0; i < kKeysPerThread; ++i) {
            if (head >> i & 1u) {
                const unsigned long long g = off + pos;
                if (g < arena_cap) {
                    arena[g] = k[i];
                    if ((pos & (kSplitStride - 1)) == 0) split[g / kSplitStride] = k[i];
                }
                ++pos;
            }
        }
    }
}

// ------------------------------------------------------ backward ---------

template <typename T> __device__ __forceinline__ T cast_rate(double x);
template <> __device__ __forceinline__ uint32_t cast_rate<uint32_t>(double x) { return (uint32_t)__double2uint_rz(x); }
template <> __device__ __forceinline__ uint64_t cast_rate<uint64_t>(double x) { return (uint64_t)__double2ull_rz(x); }
template <> __device__ __forceinline__ float cast_rate<float>(double x) { return __double2float_rn(x); }
template <> __device__ __forceinline__ double cast_rate<double>(double x) { return x; }

// Backward solve of layer t (recalculate_layer, native_core/src/BookSolver.cpp:
// 413-470). Per board: success with do_check -> max; else for every empty
// nibble ascending, best2 = max of layer t+1 rates over the kept moves of the
// spawn-2 board, acc = fma(best2, 1-p4, acc); best4 likewise from layer t+2,
// acc = fma(best4, p4, acc); rate = T(acc / #empty). The two fma() are the
// reference's `+=` statements as its -Ofast x86-64-v3 build contracts them.
template <typename T>
__global__ void __launch_bounds__(256)
solve_kernel(const uint64_t *__restrict__ arena, T *__restrict__ rates, const uint64_t *__restrict__ split,
             const unsigned long long *__restrict__ layer_off, const unsigned long long *__restrict__ layer_len,
             int t, DevSpec spec, int do_check, const uint32_t *__restrict__ tab, double p4, T zero, T maxv,
             DevCtl *ctl) {
    const unsigned long long n0 = layer_len[t];
    const unsigned long long o0 = layer_off[t], o1 = layer_off[t + 1], o2 = layer_off[t + 2];
    const unsigned long long n1 = layer_len[t + 1], n2 = layer_len[t + 2];
    const uint64_t *k1 = arena + o1, *k2 = arena + o2;
    const T *r1 = rates + o1, *r2 = rates + o2;
    const uint64_t *s1 = split + o1 / kSplitStride, *s2 = split + o2 / kSplitStride;
    const double w2 = 1.0 - p4;
    unsigned long long looks = 0;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n0;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t b = arena[o0 + i];
        if (do_check && is_success(b, spec)) {
            rates[o0 + i] = maxv;
            continue;
        }
        MoveCtx mc;
        move_ctx_init(tab, b, mc);
        uint64_t empt = empty_nibbles(b);
        double acc = 0.0;
        int nempty = 0;
        while (empt) {
            const int k = (__ffsll((long long)empt) - 1) >> 2;
            empt &= empt - 1;
            ++nempty;
#pragma unroll
            for (int v = 1; v <= 2; ++v) {
                uint64_t mv[4], s;
                spawn_moves(tab, mc, k, (uint64_t)v, s, mv);
                T best = zero;
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    if (mv[d] != s && is_pattern(mv[d], spec)) {
                        const uint64_t key = canonical(mv[d], spec.symm);
                        const T got = v == 1 ? layer_lookup<T>(k1, r1, n1, s1, key, zero)
                                             : layer_lookup<T>(k2, r2, n2, s2, key, zero);
                        ++looks;
                        if (best < got) best = got;
                    }
                }
                acc = fma((double)best, v == 1 ? w2 : p4, acc);
            }
        }
        rates[o0 + i] = nempty > 0 ? cast_rate<T>(acc / (double)nempty) : zero;
    }
    // warp-aggregated statistics
    for (int o = 16; o > 0; o >>= 1) looks += __shfl_xor_sync(0xFFFFFFFFu, looks, o);
    if ((threadIdx.x & 31) == 0 && looks) atomicAdd(&ctl->lookups, looks);
}

// Layers steps-2 and steps-1: success -> max, else zero
// (final_situation_process, native_core/src/BookSolver.cpp:237-261).
template <typename T>
__global__ void final_layer_kernel(const uint64_t *__restrict__ arena, T *__restrict__ rates,
                                   const unsigned long long *__restrict__ layer_off,
                                   const unsigned long long *__restrict__ layer_len, int t, DevSpec spec, T zero,
                                   T maxv) {
    const unsigned long long n = layer_len[t], o = layer_off[t];
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        rates[o + i] = is_success(arena[o + i], spec) ? maxv : zero;
}

// Book packing: live entries (rate > zero) of layer t as packed records
// {u64 board; T rate} (compact_live_entries + write_layer_file,
// native_core/src/BookSolver.cpp:380-394,206-231; SuccessEntry,
// native_core/include/FormationRuntime.h:191-199).
template <typename T>
__global__ void __launch_bounds__(kSortThreads)
book_count_kernel(const T *__restrict__ rates, const unsigned long long *__restrict__ layer_off,
                  const unsigned long long *__restrict__ layer_len, int t, T zero, unsigned *__restrict__ tile_cnt) {
    __shared__ unsigned long long sm[33];
    const unsigned long long n = layer_len[t], o = layer_off[t];
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        unsigned long long c = 0;
        const unsigned long long base = tile * kTileKeys + threadIdx.x;
#pragma unroll 4
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + (unsigned long long)i * kSortThreads;
            if (idx < n) c += rates[o + idx] > zero;
        }
        unsigned long long tot;
        block_excl_scan<unsigned long long>(c, sm, &tot);
        if (threadIdx.x == 0) tile_cnt[tile] = (unsigned)tot;
    }
}

template <typename T>
__global__ void __launch_bounds__(kSortThreads)
book_write_kernel(const uint64_t *__restrict__ arena, const T *__restrict__ rates,
                  const unsigned long long *__restrict__ layer_off, const unsigned long long *__restrict__ layer_len,
                  int t, T zero, const unsigned long long *__restrict__ tile_off, unsigned char *__restrict__ book,
                  unsigned long long book_off_bytes, unsigned long long book_cap_bytes, DevCtl *ctl) {
    __shared__ unsigned long long sm[33];
    constexpr int rec = 8 + (int)sizeof(T);
    const unsigned long long n = layer_len[t], o = layer_off[t];
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // contiguous run of 16 entries per thread keeps the output in order
        const unsigned long long base = tile * kTileKeys + (unsigned long long)threadIdx.x * kKeysPerThread;
        unsigned live = 0, c = 0;
#pragma unroll
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + i;
            const bool l = idx < n && rates[o + idx] > zero;
            live |= (unsigned)l << i;
            c += l;
        }
        unsigned long long tot;
        unsigned long long pos = tile_off[tile] + block_excl_scan<unsigned long long>(c, sm, &tot);
        for (int i = 0; i < kKeysPerThread; ++i) {
            if (live >> i & 1u) {
                const unsigned long long byte = book_off_bytes + pos * rec;
                if (byte + rec <= book_cap_bytes) {
                    const uint64_t key = arena[o + base + i];
                    const T r = rates[o + base + i];
                    if constexpr (rec == 16) {
                        *reinterpret_cast<uint64_t *>(book + byte) = key;
                        *reinterpret_cast<T *>(book + byte + 8) = r;
                    } else {
                        // 12-byte records are only 4-byte aligned
                        uint32_t *w = reinterpret_cast<uint32_t *>(book + byte);
                        w[0] = (uint32_t)key;
                        w[1] = (uint32_t)(key >> 32);
                        w[2] = *reinterpret_cast<const uint32_t *>(&r);
                    }
                } else {
                    atomicOr(&ctl->err, kErrBookOverflow);
                }
                ++pos;
            }
        }
    }
}

}  // namespace egtb
