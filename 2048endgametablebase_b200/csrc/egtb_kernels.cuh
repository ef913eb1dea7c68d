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
constexpr unsigned kErrDedupOverflow = 16u;
constexpr unsigned kErrIndexOverflow = 32u;

constexpr int kTileKeys = 4096;     // keys per sort / compaction tile
constexpr int kSortThreads = 256;   // 8 warps x 16 keys x 32 lanes
constexpr int kKeysPerThread = kTileKeys / kSortThreads;

// Control block in device memory.
struct DevCtl {
    unsigned long long stage_count[3];  // keys in the three layer staging buffers (layer L in buffer L % 3)
    unsigned long long blocks_done;     // last-block detection of the expand kernel
    unsigned long long cand_count[2];   // keys handed to a sort (sort API, per-layer fallback sorts)
    unsigned long long n_sort;          // keys handed to the sort
    unsigned long long n_unique;        // result of the last unique / compaction
    unsigned long long candidates;      // statistics: keys that reached a sort
    unsigned long long lookups;         // statistics: exact searches in the backward pass
    unsigned long long expand_next;     // next 32-parent chunk of the running expand launch
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

constexpr int kExpandThreads = 1024;                       // one block per SM
constexpr int kRowSmemBytes = 65536 * (int)sizeof(uint16_t);  // dynamic shared memory: the row table
constexpr int kStage = 64;  // per-warp staging slots per stream

// Children of one spawn of the lane's parent (value v in empty nibble k; k < 0:
// none): the four moves that moved the board and match the pattern,
// canonicalised, minus the ones the direct-mapped repeat filter has already
// seen (filter_bits 0: no filter). The four filter slots are read before any
// is written, so their loads are in flight together. Returns the kept moves
// as a 4-bit mask; *probes counts the children that reached the filter.
template <bool kVariantModes, typename Rows>
__device__ __forceinline__ unsigned spawn_children(const Rows &rows, const MoveCtx &mc, int k, uint64_t v,
                                                   const DevSpec &spec, uint64_t *filter, int filter_bits,
                                                   uint64_t key[4], unsigned long long &probes) {
    uint64_t mv[4], s = 0;
    if (k >= 0) spawn_moves(rows, mc, k, v, s, mv);
    unsigned keep = 0;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        key[d] = 0;
        if (k >= 0 && mv[d] != s && is_pattern(mv[d], spec)) {
            key[d] = canonical<kVariantModes>(mv[d], spec.symm);
            keep |= 1u << d;
        }
    }
    probes += __popc(keep);
    if (filter_bits && keep) {
        uint64_t slot[4], seen[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            slot[d] = filter_slot(key[d], filter_bits);
            seen[d] = (keep >> d & 1u) ? filter[slot[d]] : ~key[d];
        }
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            if (!(keep >> d & 1u)) continue;
            if (seen[d] == key[d]) keep &= ~(1u << d);
            else filter[slot[d]] = key[d];
        }
    }
    return keep;
}

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

// ------------------------------------------------- exact dedup sets ------
//
// Every layer under construction has a hash set of its keys (open addressing,
// u64 slots, linear probing). Keys of one layer share one tile sum, so a slot
// whose key has another tile sum - a key of an older layer, or 0 - is free:
// the two sets (by layer parity) are never cleared. A key placed at slot p
// only ever passed slots holding keys of its own layer, which stay until the
// layer is done, so a later probe for it always reaches p.

// Tile-value sums of every byte of a board (two nibbles; 0xF counts 32768).
__device__ __forceinline__ void init_byte_sums(unsigned *bsum) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        const unsigned lo = i & 15, hi = i >> 4;
        bsum[i] = (lo ? 1u << lo : 0u) + (hi ? 1u << hi : 0u);
    }
}

__device__ __forceinline__ long long board_tile_sum(uint64_t b, const unsigned *bsum) {
    long long s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += bsum[(b >> (8 * i)) & 0xFFu];
    return s;
}

// Longest probe chain a set insert walks. The host keeps every set at most
// half full, where chains stay far shorter; a longer chain means the set
// overflowed: the insert flags it (the host regrows the set and re-runs the
// pass) instead of walking an ever fuller table.
constexpr int kMaxProbe = 128;

// 1 when key is new in the set of the layer whose tile sum is want_sum.
__device__ __forceinline__ int dedup_insert(uint64_t *tab, unsigned long long mask, uint64_t key, long long want_sum,
                                           const unsigned *bsum, unsigned *err) {
    unsigned long long h = mix64(key) & mask;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        unsigned long long cur = __ldcg((const unsigned long long *)tab + h);
        for (;;) {
            if (cur == key) return 0;
            if (board_tile_sum(cur, bsum) != want_sum) {
                const unsigned long long prev =
                    atomicCAS((unsigned long long *)tab + h, cur, (unsigned long long)key);
                if (prev == cur) return 1;
                cur = prev;
                continue;
            }
            break;
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, kErrDedupOverflow);
    return 0;
}

// 1 when key is new in a set whose free slots hold 0 (a set cleared before
// its layer's first insert): one atomic per probed slot.
__device__ __forceinline__ int dedup_insert_zero(uint64_t *tab, unsigned long long mask, uint64_t key, unsigned *err) {
    unsigned long long h = mix64(key) & mask;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        const unsigned long long prev = atomicCAS((unsigned long long *)tab + h, 0ull, (unsigned long long)key);
        if (prev == 0ull) return 1;
        if (prev == key) return 0;
        h = (h + 1) & mask;
    }
    atomicOr(err, kErrDedupOverflow);
    return 0;
}

// Continue a zero-slot insert of key after its first probe found another key at h.
__device__ __forceinline__ int dedup_insert_zero_from(uint64_t *tab, unsigned long long mask, uint64_t key,
                                                      unsigned long long h, unsigned *err) {
    for (int probe = 1; probe < kMaxProbe; ++probe) {
        h = (h + 1) & mask;
        const unsigned long long prev = atomicCAS((unsigned long long *)tab + h, 0ull, (unsigned long long)key);
        if (prev == 0ull) return 1;
        if (prev == key) return 0;
    }
    atomicOr(err, kErrDedupOverflow);
    return 0;
}

// Flush a warp's staged keys (children that passed the repeat filter): the
// warp enters them in the layer's set 32 at a time, every lane busy, and
// appends the ones that are new to the layer's staging buffer. Flags
// kErrDedupOverflow when the layer passes half its set's capacity. kZero:
// the set's free slots hold 0 (else: a slot of another tile sum is free);
// then two keys per lane go at once, their first probes in flight together.
template <bool kZero>
__device__ __forceinline__ void stage_flush_dedup(uint64_t *stage, int &count, uint64_t *__restrict__ out,
                                                  unsigned long long *cnt, unsigned long long cap, uint64_t *set,
                                                  unsigned long long set_mask, long long want, const unsigned *bsum,
                                                  unsigned *err) {
    const int lane = threadIdx.x & 31;
    const unsigned long long half = (set_mask + 1) / 2;
    if constexpr (kZero) {
        const unsigned below = (1u << lane) - 1u;
        for (int b = 0; b < count; b += 64) {
            const int i0 = b + lane, i1 = b + 32 + lane;
            const bool v0 = i0 < count, v1 = i1 < count;
            const uint64_t k0 = v0 ? stage[i0] : 0, k1 = v1 ? stage[i1] : 0;
            const unsigned long long h0 = mix64(k0) & set_mask, h1 = mix64(k1) & set_mask;
            const unsigned long long p0 = v0 ? atomicCAS((unsigned long long *)set + h0, 0ull, (unsigned long long)k0) : 1ull;
            const unsigned long long p1 = v1 ? atomicCAS((unsigned long long *)set + h1, 0ull, (unsigned long long)k1) : 1ull;
            bool f0 = v0 && p0 == 0ull, f1 = v1 && p1 == 0ull;
            if (v0 && p0 != 0ull && p0 != k0) f0 = dedup_insert_zero_from(set, set_mask, k0, h0, err) != 0;
            if (v1 && p1 != 0ull && p1 != k1) f1 = dedup_insert_zero_from(set, set_mask, k1, h1, err) != 0;
            const unsigned m0 = __ballot_sync(0xFFFFFFFFu, f0), m1 = __ballot_sync(0xFFFFFFFFu, f1);
            const unsigned n = __popc(m0) + __popc(m1);
            if (n) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(cnt, (unsigned long long)n);
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base + n > cap) {
                    if (lane == 0) atomicOr(err, kErrCandOverflow);
                } else {
                    if (f0) out[base + __popc(m0 & below)] = k0;
                    if (f1) out[base + __popc(m0) + __popc(m1 & below)] = k1;
                }
                if (lane == 0 && base + n > half) atomicOr(err, kErrDedupOverflow);
            }
        }
    } else {
        for (int b = 0; b < count; b += 32) {
            const int i = b + lane;
            const uint64_t key = i < count ? stage[i] : 0;
            const bool fresh = i < count && dedup_insert(set, set_mask, key, want, bsum, err) != 0;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, fresh);
            if (m) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(cnt, (unsigned long long)__popc(m));
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                const unsigned long long pos = base + __popc(m & ((1u << lane) - 1u));
                if (base + __popc(m) > cap) {
                    if (lane == 0) atomicOr(err, kErrCandOverflow);
                } else if (fresh) {
                    out[pos] = key;
                }
                if (lane == 0 && base + __popc(m) > half) atomicOr(err, kErrDedupOverflow);
            }
        }
    }
    __syncwarp();
    count = 0;
}

// One forward step (gen_boards_*, native_core/src/BookGenerator.cpp:472-760,
// with sort + unique + merge, :1059-1078, done by the sets): expand layer t.
// Every parent, unless do_check and it is a success; every empty nibble k
// ascending; spawn 2 (v=1) and 4 (v=2); the four moves; a child is kept when
// it moved and matches the pattern, is canonicalised, and is appended to
// layer t+v's staging buffer iff it is new in layer t+v's set. The same
// kernel copies layer t into the arena at layer_off[t] and closes it (length,
// next 16-aligned offset, capacity check); its last block empties layer t's
// staging buffer for layer t+3. Sets rotate over three buffers (layer L in
// set L % 3): this step zeroes layer t's set, which layer t+3 fills next.
template <bool kVariantModes>
__global__ void __launch_bounds__(kExpandThreads, 1)
expand_dedup_kernel(uint64_t *__restrict__ stage_par, uint64_t *__restrict__ stage1, uint64_t *__restrict__ stage2,
                    int si_par, int si1, int si2, uint64_t *__restrict__ arena,
                    unsigned long long *__restrict__ layer_off, unsigned long long *__restrict__ layer_len,
                    unsigned long long arena_cap, int t, DevSpec spec, int do_check, const uint32_t *__restrict__ tab,
                    uint64_t *__restrict__ set1, uint64_t *__restrict__ set2, unsigned long long set_mask,
                    unsigned long long stage_cap, uint64_t *filter, int filter_bits, uint64_t *__restrict__ clear_set,
                    DevCtl *ctl, unsigned *progress, unsigned progress_value) {
    __shared__ uint64_t stage[kExpandThreads / 32][2][kStage];
    __shared__ int last_block;
    extern __shared__ uint16_t srows[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the row table does not depend on the step before: it is staged while
    // that step's last blocks finish (programmatic dependent launch)
    pdl_trigger();
    stage_rows(tab, srows);
    pdl_wait();
    const SharedRows rows{srows};
    {
        uint4 *z = reinterpret_cast<uint4 *>(clear_set);
        const unsigned long long nz = (set_mask + 1) / 2;
        for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nz;
             i += (unsigned long long)gridDim.x * blockDim.x)
            z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    // once this pass has overflowed a buffer it will be re-run: skip the work
    const unsigned long long n = (ctl->err & (kErrCandOverflow | kErrDedupOverflow)) ? 0 : ctl->stage_count[si_par];
    const unsigned long long off = layer_off[t];
    // arena == nullptr: layers stream out of the device (the host sorts and
    // ships layer t after this step); only the layer's length is recorded
    const bool fits = arena && !(ctl->err & kErrArenaOverflow) && off + n <= arena_cap;
    if (!arena && blockIdx.x == 0 && threadIdx.x == 0) {
        layer_len[t] = n;
        layer_off[t + 1] = 0;
    } else if (blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned long long next = (off + n + kSplitStride - 1) & ~(unsigned long long)(kSplitStride - 1);
        if (!fits || next > arena_cap) {
            atomicOr(&ctl->err, kErrArenaOverflow);
            layer_len[t] = 0;
            layer_off[t + 1] = off;
        } else {
            layer_len[t] = n;
            layer_off[t + 1] = next;
        }
    }
    __syncthreads();
    int cnt1 = 0, cnt2 = 0;  // keys staged in this warp for layers t+1 and t+2
    unsigned long long probes = 0;
    // warps claim 32-parent chunks as they go, so a warp whose parents have
    // few empty cells takes more of them (the last block resets the counter)
    for (;;) {
        unsigned long long chunk = 0;
        if (lane == 0) chunk = atomicAdd(&ctl->expand_next, 1ull);
        const unsigned long long base = __shfl_sync(0xFFFFFFFFu, chunk, 0) * 32;
        if (base >= n) break;
        const unsigned long long p = base + lane;
        bool active = p < n;
        uint64_t b = active ? stage_par[p] : 0;
        if (active && fits) arena[off + p] = b;
        if (active && do_check && is_success(b, spec)) active = false;
        uint64_t empt = active ? empty_nibbles(b) : 0;
        MoveCtx mc;
        move_ctx_init(rows, b, mc);
        unsigned any = __ballot_sync(0xFFFFFFFFu, empt != 0);
        while (any) {
            // next empty nibble of this lane (lanes advance independently; the
            // loop runs while any lane still has one)
            int k = -1;
            if (empt) {
                k = (__ffsll((long long)empt) - 1) >> 2;
                empt &= empt - 1;
            }
#pragma unroll 1
            for (int v = 1; v <= 2; ++v) {
                uint64_t *const set = v == 1 ? set1 : set2;
                uint64_t *const sbuf = stage[warp][v - 1];
                int c = v == 1 ? cnt1 : cnt2;
                // a direct-mapped filter drops most repeats with one load; a
                // key it holds has already been staged for its set
                uint64_t keys[4];
                const unsigned kept =
                    spawn_children<kVariantModes>(rows, mc, k, (uint64_t)v, spec, filter, filter_bits, keys, probes);
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    const bool keep = kept >> d & 1u;
                    const uint64_t key = keys[d];
                    const unsigned m = __ballot_sync(0xFFFFFFFFu, keep);
                    if (m) {
                        const int pos = c + __popc(m & ((1u << lane) - 1u));
                        if (keep) sbuf[pos] = key;
                        c += __popc(m);
                        __syncwarp();
                        if (c > kStage - 32)
                            stage_flush_dedup<true>(sbuf, c, v == 1 ? stage1 : stage2,
                                                    &ctl->stage_count[v == 1 ? si1 : si2], stage_cap, set, set_mask,
                                                    0, nullptr, &ctl->err);
                    }
                }
                if (v == 1) cnt1 = c; else cnt2 = c;
            }
            any = __ballot_sync(0xFFFFFFFFu, empt != 0);
        }
    }
    stage_flush_dedup<true>(stage[warp][0], cnt1, stage1, &ctl->stage_count[si1], stage_cap, set1, set_mask, 0,
                            nullptr, &ctl->err);
    stage_flush_dedup<true>(stage[warp][1], cnt2, stage2, &ctl->stage_count[si2], stage_cap, set2, set_mask, 0,
                            nullptr, &ctl->err);
    for (int o = 16; o > 0; o >>= 1) probes += __shfl_xor_sync(0xFFFFFFFFu, probes, o);
    if (lane == 0 && probes) atomicAdd(&ctl->candidates, probes);
    // the last block to finish empties layer t's staging buffer
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last_block = atomicAdd(&ctl->blocks_done, 1ull) == (unsigned long long)gridDim.x - 1;
    __syncthreads();
    if (last_block && threadIdx.x == 0) {
        ctl->stage_count[si_par] = 0;
        ctl->blocks_done = 0;
        ctl->expand_next = 0;
        if (progress) *(volatile unsigned *)progress = progress_value;
    }
}

// Copy a finished layer from its staging buffer into the arena and close it
// (the last two layers, which no expand step reads).
static __global__ void __launch_bounds__(256)
flush_layer_kernel(const uint64_t *__restrict__ stage_l, int si, uint64_t *__restrict__ arena,
                   unsigned long long *__restrict__ layer_off, unsigned long long *__restrict__ layer_len,
                   unsigned long long arena_cap, int L, DevCtl *ctl) {
    const unsigned long long n = ctl->stage_count[si];
    const unsigned long long off = layer_off[L];
    const bool fits = !(ctl->err & kErrArenaOverflow) && off + n <= arena_cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned long long next = (off + n + kSplitStride - 1) & ~(unsigned long long)(kSplitStride - 1);
        if (!fits || next > arena_cap) {
            atomicOr(&ctl->err, kErrArenaOverflow);
            layer_len[L] = 0;
            layer_off[L + 1] = off;
        } else {
            layer_len[L] = n;
            layer_off[L + 1] = next;
        }
    }
    if (!fits) return;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        arena[off + i] = stage_l[i];
}

// Insert keys already known to be in layer L (a resumed partial layer).
static __global__ void __launch_bounds__(256)
dedup_seed_kernel(const uint64_t *__restrict__ keys, unsigned long long n, uint64_t *set, unsigned long long mask,
                  DevCtl *ctl) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        dedup_insert_zero(set, mask, keys[i], &ctl->err);
}

// ------------------------------------------------------ free nibbles ----
//
// After the forward pass each layer holds its unique keys in arrival order;
// the layers are sorted by their free nibbles (the others are 0xF in every
// key of the pattern), each in its own arena region (seg_* kernels,
// egtb_sort.cuh), in the plain and the batched build alike.

struct FreeNibbles {
    int count;
    int idx[16];       // free nibble positions, least significant first
    uint64_t pinned;   // every other nibble is 0xF
};

// Single block: exclusive scan of the tile counts; total -> *total_out.
static __global__ void __launch_bounds__(1024)
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

// ------------------------------------------------------ backward ---------

template <typename T> __device__ __forceinline__ T cast_rate(double x);
template <> __device__ __forceinline__ uint32_t cast_rate<uint32_t>(double x) { return (uint32_t)__double2uint_rz(x); }
template <> __device__ __forceinline__ uint64_t cast_rate<uint64_t>(double x) { return (uint64_t)__double2ull_rz(x); }
template <> __device__ __forceinline__ float cast_rate<float>(double x) { return __double2float_rn(x); }
template <> __device__ __forceinline__ double cast_rate<double>(double x) { return x; }

// ------------------------------------------------- layer rate index ------
//
// The backward pass looks up every child position in the rates of layers
// t+1 and t+2. Each of those layers gets an open-addressing hash index of its
// live entries (rate > zero; a missing key reads as zero, exactly like a
// zero-rate entry): 16-byte slots {key, rate bits}, key 0 = empty (no board
// is 0), capacity a power of two of at least twice the layer, linear probing.
// A lookup costs ~1.3 dependent 16-byte loads instead of the ~18 of a binary
// search, and the eight lookups of one empty cell are issued together.


template <typename T> __device__ __forceinline__ unsigned long long rate_bits(T r) {
    if constexpr (sizeof(T) == 4) return (unsigned long long)__float_as_uint(*reinterpret_cast<const float *>(&r));
    else return (unsigned long long)__double_as_longlong(*reinterpret_cast<const double *>(&r));
}
template <typename T> __device__ __forceinline__ T rate_from_bits(unsigned long long b) {
    T r;
    if constexpr (sizeof(T) == 4) {
        const unsigned u = (unsigned)b;
        memcpy(&r, &u, 4);
    } else {
        memcpy(&r, &b, 8);
    }
    return r;
}

template <typename T>
__global__ void __launch_bounds__(256)
index_insert_kernel(const uint64_t *__restrict__ arena, const T *__restrict__ rates,
                    const unsigned long long *__restrict__ layer_off, const unsigned long long *__restrict__ layer_len,
                    int t, T zero, ulonglong2 *__restrict__ slots, unsigned long long mask, DevCtl *ctl) {
    const unsigned long long n = layer_len[t], o = layer_off[t];
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const T r = rates[o + i];
        if (!(r > zero)) continue;
        const uint64_t key = arena[o + i];
        unsigned long long h = mix64(key) & mask;
        bool placed = false;
        for (int probe = 0; probe < kMaxProbe * 32; ++probe) {
            const unsigned long long prev = atomicCAS(&slots[h].x, 0ull, (unsigned long long)key);
            if (prev == 0ull || prev == key) {
                slots[h].y = rate_bits<T>(r);
                placed = true;
                break;
            }
            h = (h + 1) & mask;
        }
        if (!placed) atomicOr(&ctl->err, kErrIndexOverflow);
    }
}

// {key, rate} into an index whose free slots hold key 0.
template <typename T>
__device__ __forceinline__ void index_insert_zero(ulonglong2 *slots, unsigned long long mask, uint64_t key, T r,
                                                  unsigned *err) {
    unsigned long long h = mix64(key) & mask;
    for (int probe = 0; probe < kMaxProbe * 32; ++probe) {
        const unsigned long long prev = atomicCAS(&slots[h].x, 0ull, (unsigned long long)key);
        if (prev == 0ull || prev == key) {
            slots[h].y = rate_bits<T>(r);
            return;
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, kErrIndexOverflow);
}

// Backward solve of layer t (recalculate_layer, native_core/src/BookSolver.cpp:
// 413-470). Per board: success with do_check -> max; else for every empty
// nibble ascending, best2 = max of layer t+1 rates over the kept moves of the
// spawn-2 board, acc = fma(best2, 1-p4, acc); best4 likewise from layer t+2,
// acc = fma(best4, p4, acc); rate = T(acc / #empty). The two fma() are the
// reference's `+=` statements as its -Ofast x86-64-v3 build contracts them.
// With idx0, layer t's live entries also enter its rate index (mask m0) for
// the solves of layers t-1 and t-2; with clear_idx, this launch zeroes
// clear_slots slots of another (unused) index for the next launch's inserts.
template <typename T, bool kVariantModes>
__global__ void __launch_bounds__(256, 4)
solve_kernel(const uint64_t *__restrict__ arena, T *__restrict__ rates,
             const unsigned long long *__restrict__ layer_off, const unsigned long long *__restrict__ layer_len,
             int t, DevSpec spec, int do_check, const uint32_t *__restrict__ tab, double p4, T zero, T maxv,
             const ulonglong2 *__restrict__ idx1, unsigned long long m1, const ulonglong2 *__restrict__ idx2,
             unsigned long long m2, DevCtl *ctl, ulonglong2 *__restrict__ idx0 = nullptr, unsigned long long m0 = 0,
             ulonglong2 *__restrict__ clear_idx = nullptr, unsigned long long clear_slots = 0,
             unsigned *progress = nullptr, unsigned progress_value = 0) {
    const GlobalRows rows{tab};
    pdl_trigger();
    pdl_wait();  // launched early (programmatic dependent launch): the launch before must be done
    const unsigned long long n0 = layer_len[t], o0 = layer_off[t];
    const double w2 = 1.0 - p4;
    unsigned long long looks = 0;
    if (progress && blockIdx.x == 0 && threadIdx.x == 0) *(volatile unsigned *)progress = progress_value;
    if (clear_idx) {
        uint4 *z = reinterpret_cast<uint4 *>(clear_idx);
        for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < clear_slots;
             i += (unsigned long long)gridDim.x * blockDim.x)
            z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n0;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t b = arena[o0 + i];
        if (do_check && is_success(b, spec)) {
            rates[o0 + i] = maxv;
            if (idx0 && maxv > zero) index_insert_zero<T>(idx0, m0, b, maxv, &ctl->err);
            continue;
        }
        MoveCtx mc;
        move_ctx_init(rows, b, mc);
        uint64_t empt = empty_nibbles(b);
        double acc = 0.0;
        int nempty = 0;
        while (empt) {
            const int k = (__ffsll((long long)empt) - 1) >> 2;
            empt &= empt - 1;
            ++nempty;
            // the eight children of this cell: j = 0..3 spawn 2, j = 4..7 spawn 4
            uint64_t key[8];
            unsigned pend = 0;
#pragma unroll
            for (int v = 1; v <= 2; ++v) {
                uint64_t mv[4], s;
                spawn_moves(rows, mc, k, (uint64_t)v, s, mv);
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    const int j = (v - 1) * 4 + d;
                    key[j] = canonical<kVariantModes>(mv[d], spec.symm);
                    if (mv[d] != s && is_pattern(mv[d], spec)) pend |= 1u << j;
                }
            }
            looks += __popc(pend);
            unsigned long long h[8];
            T got[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                got[j] = zero;
                h[j] = mix64(key[j]) & (j < 4 ? m1 : m2);
            }
            // ends: an index holds at most half as many keys as it has slots
            // (capacity >= 2 x the layer, cleared before its inserts), so every
            // probe chain meets an empty slot (a counter here measured 3-5 %
            // slower)
            while (pend) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (pend >> j & 1u) {
                        const ulonglong2 sl = __ldg((j < 4 ? idx1 : idx2) + h[j]);
                        if (sl.x == key[j]) {
                            got[j] = rate_from_bits<T>(sl.y);
                            pend &= ~(1u << j);
                        } else if (sl.x == 0ull) {
                            pend &= ~(1u << j);
                        } else {
                            h[j] = (h[j] + 1) & (j < 4 ? m1 : m2);
                        }
                    }
                }
            }
            T best2 = zero, best4 = zero;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (best2 < got[j]) best2 = got[j];
                if (best4 < got[j + 4]) best4 = got[j + 4];
            }
            acc = fma((double)best2, w2, acc);
            acc = fma((double)best4, p4, acc);
        }
        const T r = nempty > 0 ? cast_rate<T>(acc / (double)nempty) : zero;
        rates[o0 + i] = r;
        if (idx0 && r > zero) index_insert_zero<T>(idx0, m0, b, r, &ctl->err);
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

// ---------------------------------------------- all-layer book packing ----
//
// After the backward pass every layer is packed at once: the tiles of all
// layers form one sequence (layer L owns tiles first_tile[L] ..
// first_tile[L+1]-1), one count kernel, one scan, one write kernel.

__device__ __forceinline__ int layer_of_tile(const unsigned long long *first_tile, int n_layers,
                                             unsigned long long g) {
    int lo = 0, hi = n_layers;  // largest L with first_tile[L] <= g
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first_tile[mid] <= g) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

template <typename T>
__global__ void __launch_bounds__(kSortThreads)
book_count_all_kernel(const T *__restrict__ rates, const unsigned long long *__restrict__ layer_off,
                      const unsigned long long *__restrict__ layer_len, const unsigned long long *__restrict__ first_tile,
                      int n_layers, unsigned long long n_tiles, T zero, unsigned *__restrict__ tile_cnt,
                      unsigned long long *__restrict__ layer_max) {
    __shared__ unsigned long long sm[33];
    __shared__ unsigned long long smax;
    for (unsigned long long g = blockIdx.x; g < n_tiles; g += gridDim.x) {
        const int L = layer_of_tile(first_tile, n_layers, g);
        const unsigned long long n = layer_len[L], o = layer_off[L];
        const unsigned long long base = (g - first_tile[L]) * kTileKeys + threadIdx.x;
        if (threadIdx.x == 0) smax = 0;
        unsigned long long c = 0, mx = 0;
#pragma unroll 4
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + (unsigned long long)i * kSortThreads;
            if (idx < n) {
                const T r = rates[o + idx];
                if (r > zero) {
                    ++c;
                    const unsigned long long ob = ordered_bits((double)r);
                    mx = ob > mx ? ob : mx;
                }
            }
        }
        unsigned long long tot;
        block_excl_scan<unsigned long long>(c, sm, &tot);
        if (mx) atomicMax(&smax, mx);
        __syncthreads();
        if (threadIdx.x == 0) {
            tile_cnt[g] = (unsigned)tot;
            if (smax) atomicMax(layer_max + L, smax);
        }
        __syncthreads();
    }
}

// Single block: exclusive scan of `count` tile counts.
static __global__ void __launch_bounds__(1024)
scan_tiles_kernel(const unsigned *__restrict__ cnt, unsigned long long count, unsigned long long *__restrict__ off,
                  unsigned long long *total_out) {
    __shared__ unsigned long long sm[33];
    unsigned long long run = 0, tot;
    for (unsigned long long c0 = 0; c0 < count; c0 += blockDim.x) {
        const unsigned long long i = c0 + threadIdx.x;
        const unsigned long long x = i < count ? cnt[i] : 0;
        const unsigned long long ex = block_excl_scan<unsigned long long>(x, sm, &tot);
        if (i < count) off[i] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) *total_out = run;
}

static __global__ void book_lens_kernel(const unsigned long long *__restrict__ first_tile, int n_layers,
                                 unsigned long long n_tiles, const unsigned long long *__restrict__ tile_off,
                                 const unsigned long long *__restrict__ total, unsigned long long *__restrict__ book_len) {
    for (int L = blockIdx.x * blockDim.x + threadIdx.x; L < n_layers; L += gridDim.x * blockDim.x) {
        const unsigned long long a = first_tile[L] < n_tiles ? tile_off[first_tile[L]] : *total;
        const unsigned long long b = first_tile[L + 1] < n_tiles ? tile_off[first_tile[L + 1]] : *total;
        book_len[L] = b - a;
    }
}

template <typename T>
__global__ void __launch_bounds__(kSortThreads)
book_write_all_kernel(const uint64_t *__restrict__ arena, const T *__restrict__ rates,
                      const unsigned long long *__restrict__ layer_off, const unsigned long long *__restrict__ layer_len,
                      const unsigned long long *__restrict__ first_tile, int n_layers, unsigned long long n_tiles, T zero,
                      const unsigned long long *__restrict__ tile_off, unsigned char *__restrict__ book,
                      unsigned long long book_cap_bytes, DevCtl *ctl) {
    // tile entry w * kTileKeys/8 + r * 32 + lane for warp w, round r: every
    // load is coalesced, and a warp's live entries of one round go to
    // consecutive records
    constexpr int kWarps = kSortThreads / 32, kRounds = kTileKeys / kSortThreads;
    __shared__ unsigned wbase[kWarps + 1];
    constexpr int rec = 8 + (int)sizeof(T);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (unsigned long long g = blockIdx.x; g < n_tiles; g += gridDim.x) {
        const int L = layer_of_tile(first_tile, n_layers, g);
        const unsigned long long n = layer_len[L], o = layer_off[L];
        const unsigned long long base =
            (g - first_tile[L]) * kTileKeys + (unsigned long long)warp * (kTileKeys / kWarps) + lane;
        unsigned live = 0, wcount = 0;
#pragma unroll
        for (int r = 0; r < kRounds; ++r) {
            const unsigned long long idx = base + (unsigned long long)r * 32;
            const bool l = idx < n && rates[o + idx] > zero;
            live |= (unsigned)l << r;
            wcount += __popc(__ballot_sync(0xFFFFFFFFu, l));
        }
        if (lane == 0) wbase[warp] = wcount;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned run = 0;
            for (int w = 0; w < kWarps; ++w) {
                const unsigned c = wbase[w];
                wbase[w] = run;
                run += c;
            }
        }
        __syncthreads();
        unsigned long long pos = tile_off[g] - tile_off[first_tile[L]] + wbase[warp];
        const unsigned long long book0 = o * rec;
#pragma unroll 4
        for (int r = 0; r < kRounds; ++r) {
            const unsigned m = __ballot_sync(0xFFFFFFFFu, live >> r & 1u);
            if (live >> r & 1u) {
                const unsigned long long idx = base + (unsigned long long)r * 32;
                const unsigned long long byte = book0 + (pos + __popc(m & below)) * rec;
                if (byte + rec <= book_cap_bytes) {
                    const uint64_t key = arena[o + idx];
                    const T rt = rates[o + idx];
                    if constexpr (rec == 16) {
                        *reinterpret_cast<uint64_t *>(book + byte) = key;
                        *reinterpret_cast<T *>(book + byte + 8) = rt;
                    } else {
                        uint32_t *w = reinterpret_cast<uint32_t *>(book + byte);
                        w[0] = (uint32_t)key;
                        w[1] = (uint32_t)(key >> 32);
                        w[2] = *reinterpret_cast<const uint32_t *>(&rt);
                    }
                } else {
                    atomicOr(&ctl->err, kErrBookOverflow);
                }
            }
            pos += __popc(m);
        }
        __syncthreads();  // wbase is rewritten by the next tile
    }
}

// ------------------------------------------------ optimal-branch pass ----
//
// keep_only_optimal_branches_impl (native_core/src/BookSolver.cpp:688-735):
// for layer i >= 21, entry e of book i stays only when some position of book
// i-2 plus a 4 (or of book i-1 plus a 2) has e as its best move (first
// strictly largest rate over the moves left, right, up, down). Books i-2 and
// i-1 are the already-thinned ones.

// {key, position} index of a sorted book layer (key 0 = empty slot).
static __global__ void __launch_bounds__(256)
pos_index_kernel(const uint64_t *__restrict__ keys, unsigned long long n, ulonglong2 *__restrict__ slots,
                 unsigned long long mask) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t key = keys[i];
        unsigned long long h = mix64(key) & mask;
        for (unsigned long long probe = 0; probe <= mask; ++probe) {  // at most half full
            const unsigned long long prev = atomicCAS(&slots[h].x, 0ull, (unsigned long long)key);
            if (prev == 0ull || prev == key) {
                slots[h].y = i;
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

// find_optimal_branches (BookSolver.cpp:611-645): mark the best move's entry
// of book i for every position b | v << 4k of the parent book (empty k
// ascending). As the reference, a position with no move above zero marks
// entry 0.
template <typename T>
__global__ void __launch_bounds__(256)
optimal_mark_kernel(const uint64_t *__restrict__ par, unsigned long long n_par, uint64_t v, DevSpec spec,
                    const uint32_t *__restrict__ tab, const ulonglong2 *__restrict__ slots, unsigned long long mask,
                    const T *__restrict__ rates2, unsigned long long n2, T zero, uint8_t *__restrict__ marks) {
    for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; r < n_par;
         r += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t b = par[r];
        for (int k = 0; k < 16; ++k) {
            if ((b >> (4 * k)) & 0xFull) continue;
            const uint64_t spawned = b | (v << (4 * k));
            uint64_t mv[4];
            move_all_dir(tab, spawned, mv);
            T best = zero;
            unsigned long long best_index = 0;
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                if (mv[d] == spawned || !is_pattern(mv[d], spec)) continue;
                const uint64_t key = canonical(mv[d], spec.symm);
                unsigned long long h = mix64(key) & mask;
                for (unsigned long long probe = 0; probe <= mask; ++probe) {
                    const ulonglong2 sl = __ldg(slots + h);
                    if (sl.x == key) {
                        const T rate = rates2[sl.y];
                        if (rate > best) {
                            best = rate;
                            best_index = sl.y;
                        }
                        break;
                    }
                    if (sl.x == 0ull) break;
                    h = (h + 1) & mask;
                }
            }
            if (best_index < n2) marks[best_index] = 1;
        }
    }
}

// Order-preserving compaction of the marked entries: per 4096-entry tile
// counts, then (after a scan) the write of the kept keys and rates (SoA) and
// of their packed records.
static __global__ void __launch_bounds__(kSortThreads)
mark_count_kernel(const uint8_t *__restrict__ marks, unsigned long long n, unsigned *__restrict__ tile_cnt) {
    __shared__ unsigned long long sm[33];
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        unsigned long long c = 0;
        const unsigned long long base = tile * kTileKeys + threadIdx.x;
        for (int i = 0; i < kKeysPerThread; ++i) {
            const unsigned long long idx = base + (unsigned long long)i * kSortThreads;
            if (idx < n) c += marks[idx] != 0;
        }
        unsigned long long tot;
        block_excl_scan<unsigned long long>(c, sm, &tot);
        if (threadIdx.x == 0) tile_cnt[tile] = (unsigned)tot;
    }
}

template <typename T>
__global__ void __launch_bounds__(kSortThreads)
mark_write_kernel(const uint64_t *__restrict__ keys, const T *__restrict__ rates, const uint8_t *__restrict__ marks,
                  unsigned long long n, const unsigned long long *__restrict__ tile_off, uint64_t *__restrict__ keys_out,
                  T *__restrict__ rates_out, unsigned char *__restrict__ recs) {
    __shared__ unsigned long long sm[33];
    constexpr int rec = 8 + (int)sizeof(T);
    const unsigned long long ntiles = (n + kTileKeys - 1) / kTileKeys;
    for (unsigned long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const unsigned long long base = tile * kTileKeys + (unsigned long long)threadIdx.x * kKeysPerThread;
        unsigned keep = 0, c = 0;
        for (int i = 0; i < kKeysPerThread; ++i) {
            const bool k = base + i < n && marks[base + i] != 0;
            keep |= (unsigned)k << i;
            c += k;
        }
        unsigned long long tot;
        unsigned long long pos = tile_off[tile] + block_excl_scan<unsigned long long>(c, sm, &tot);
        for (int i = 0; i < kKeysPerThread; ++i) {
            if (!(keep >> i & 1u)) continue;
            const uint64_t key = keys[base + i];
            const T r = rates[base + i];
            keys_out[pos] = key;
            rates_out[pos] = r;
            if constexpr (rec == 16) {
                *reinterpret_cast<uint64_t *>(recs + pos * rec) = key;
                *reinterpret_cast<T *>(recs + pos * rec + 8) = r;
            } else {
                uint32_t *w = reinterpret_cast<uint32_t *>(recs + pos * rec);
                w[0] = (uint32_t)key;
                w[1] = (uint32_t)(key >> 32);
                w[2] = *reinterpret_cast<const uint32_t *>(&r);
            }
            ++pos;
        }
    }
}

}  // namespace egtb
