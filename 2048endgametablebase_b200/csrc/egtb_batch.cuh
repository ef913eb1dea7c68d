// Kernels of the batched build: many tables of uneven size advance together,
// one launch per global layer step for all of them.
//
// Every table owns slices of pooled buffers (arena region, staging buffers,
// dedup sets, repeat filter, rate-index planes) described by a BatchTable in
// device memory; its layers are global layers lbase .. lbase+steps of shared
// layer_off / layer_len arrays, so the all-layer kernels of the single-table
// build (book packing) run unchanged over the concatenation of all tables.
//
// Work of one launch = the concatenation of every active table's layer t.
// Each block computes the per-table prefix of that work in shared memory from
// counts that stay fixed during the launch, and maps a work index to its
// table by binary search; warps take contiguous runs of work items, so a warp
// changes table rarely and flushes its staged keys only then.
#pragma once

#include <cstdint>

#include "egtb_sort.cuh"

namespace egtb {

constexpr int kMaxBatchTables = 1024;
constexpr unsigned kErrBatchForward = kErrCandOverflow | kErrDedupOverflow | kErrArenaOverflow;

// Parameters of one table (constant during a build).
struct BatchTable {
    DevSpec spec;
    FreeNibbles fn;
    long long s0;                  // tile sum of layer 0
    double p4;                     // spawn rate of a 4
    int steps, docheck, lbase;     // layers 0..steps-1 are global layers lbase..lbase+steps-1
    int filter_bits;               // 0: no repeat filter
    unsigned long long abase, acap;  // arena region [abase, abase + acap)
    uint64_t *stage[3];            // staging buffers: layer L's new keys in stage[L % 3]
    unsigned long long stage_cap;
    uint64_t *set[2];              // exact dedup sets by layer parity
    unsigned long long set_mask;
    uint64_t *filter;
    ulonglong2 *index[4];          // rate index planes: layer L in index[L % 4], zeroed by step L+1
    unsigned long long index_mask;
};

// Mutable per-table state.
struct BatchCtl {
    unsigned long long stage_count[3];
    unsigned long long candidates;
    unsigned err;
    unsigned pad;
};

// Batch-wide counters.
struct BatchSync {
    unsigned long long blocks_done;
    unsigned long long next_item;  // next work item of the running expand launch (reset by its last block)
    unsigned long long lookups;
    unsigned err;
    unsigned pad;
};

// pre[i] = sum over j < i of cnt(j); pre[n] = total. Every thread of the
// block must call it; ends with a barrier.
template <typename F>
__device__ __forceinline__ void seg_prefix(int n, unsigned long long *pre, unsigned long long *scan_sm, F cnt) {
    unsigned long long run = 0;
    for (int c0 = 0; c0 < n; c0 += blockDim.x) {
        const int i = c0 + threadIdx.x;
        const unsigned long long x = i < n ? cnt(i) : 0ull;
        unsigned long long tot;
        const unsigned long long ex = block_excl_scan<unsigned long long>(x, scan_sm, &tot);
        if (i < n) pre[i] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) pre[n] = run;
    __syncthreads();
}

// The segment holding work index g < pre[n]: the largest i < n with pre[i] <= g.
__device__ __forceinline__ int seg_find(const unsigned long long *pre, int n, unsigned long long g) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= g) lo = mid; else hi = mid;
    }
    return lo;
}

// -------------------------------------------------------- forward step ----
//
// Global step t: for every table with t < steps, layer t (in its staging
// buffer t % 3) is copied into the table's arena region and closed; tables
// with t <= steps-3 also expand it exactly like expand_dedup_kernel (parents
// of layer t, success check when t+1 > docheck, children into the sets and
// staging buffers of layers t+1 and t+2). The last block empties every
// table's staging buffer t % 3.
constexpr int kBatchThreads = 256;

static __global__ void __launch_bounds__(kBatchThreads, 3)
batch_expand_kernel(const BatchTable *__restrict__ T, BatchCtl *C, int n_tables, int t, uint64_t *__restrict__ arena,
                    unsigned long long *__restrict__ layer_off, unsigned long long *__restrict__ layer_len,
                    const uint32_t *__restrict__ tab, unsigned chunk, BatchSync *sync, unsigned *progress,
                    unsigned progress_value) {
    __shared__ uint64_t stage[kBatchThreads / 32][2][kStage];
    __shared__ unsigned bsum[256];
    __shared__ unsigned long long pre[kMaxBatchTables + 1];
    __shared__ unsigned long long scan_sm[33];
    __shared__ int last_block;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sp = t % 3;
    init_byte_sums(bsum);
    // parents per table: the staging count of layer t is final before this
    // launch (clamped: an overflowed count is never read past capacity)
    auto parents = [&](int i) -> unsigned long long {
        if (t >= T[i].steps) return 0ull;
        return clamp_n(C[i].stage_count[sp], T[i].stage_cap);
    };
    seg_prefix(n_tables, pre, scan_sm, [&](int i) { return (parents(i) + chunk - 1) / chunk; });
    if (blockIdx.x == 0) {
        // close layer t of every table
        for (int i = threadIdx.x; i < n_tables; i += blockDim.x) {
            if (t >= T[i].steps) continue;
            const unsigned long long n = parents(i);
            const int g = T[i].lbase + t;
            const unsigned long long off = layer_off[g], end = T[i].abase + T[i].acap;
            const unsigned long long next = (off + n + kSplitStride - 1) & ~(unsigned long long)(kSplitStride - 1);
            if ((C[i].err & kErrArenaOverflow) || next > end) {
                atomicOr(&C[i].err, kErrArenaOverflow);
                layer_len[g] = 0;
                layer_off[g + 1] = off;
            } else {
                layer_len[g] = n;
                layer_off[g + 1] = next;
            }
        }
    }
    const unsigned long long total = pre[n_tables];
    int cur = -1;
    int cnt1 = 0, cnt2 = 0;
    unsigned long long probes = 0;
    // flush the warp's staged keys of table cur
    auto flush_table = [&]() {
        const BatchTable &tb = T[cur];
        stage_flush_dedup<false>(stage[warp][0], cnt1, tb.stage[(t + 1) % 3], &C[cur].stage_count[(t + 1) % 3], tb.stage_cap,
                          tb.set[(t + 1) & 1], tb.set_mask, tb.s0 + 2ll * (t + 1), bsum, &C[cur].err);
        stage_flush_dedup<false>(stage[warp][1], cnt2, tb.stage[(t + 2) % 3], &C[cur].stage_count[(t + 2) % 3], tb.stage_cap,
                          tb.set[(t + 2) & 1], tb.set_mask, tb.s0 + 2ll * (t + 2), bsum, &C[cur].err);
        unsigned long long p = probes;
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xFFFFFFFFu, p, o);
        if (lane == 0 && p) atomicAdd(&C[cur].candidates, p);
        probes = 0;
    };
    // warps claim work items (a chunk of one table's parents) as they go, in
    // increasing order, so consecutive claims mostly stay in one table
    for (;;) {
        unsigned long long claim = 0;
        if (lane == 0) claim = atomicAdd(&sync->next_item, 1ull);
        const unsigned long long it = __shfl_sync(0xFFFFFFFFu, claim, 0);
        if (it >= total) break;
        const int i = (cur >= 0 && it >= pre[cur] && it < pre[cur + 1]) ? cur : seg_find(pre, n_tables, it);
        if (i != cur) {
            if (cur >= 0 && T[cur].steps - 3 >= t) flush_table();
            cur = i;
        }
        const BatchTable &tb = T[i];
        const unsigned long long n = clamp_n(C[i].stage_count[sp], tb.stage_cap);
        const unsigned long long off = layer_off[tb.lbase + t];
        const unsigned err = *(volatile unsigned *)&C[i].err;
        const bool fits = !(err & kErrArenaOverflow) && off + n <= tb.abase + tb.acap;
        const bool expand = t <= tb.steps - 3 && !(err & (kErrCandOverflow | kErrDedupOverflow));
        const bool do_check = t + 1 > tb.docheck;
        const uint64_t *src = tb.stage[sp];
        const unsigned long long p0 = (it - pre[i]) * chunk;
        const unsigned long long p1 = p0 + chunk < n ? p0 + chunk : n;
        for (unsigned long long base = p0; base < p1; base += 32) {
            const unsigned long long p = base + lane;
            bool active = p < p1;
            const uint64_t b = active ? src[p] : 0;
            if (active && fits) arena[off + p] = b;
            if (!expand) continue;
            if (active && do_check && is_success(b, tb.spec)) active = false;
            uint64_t empt = active ? empty_nibbles(b) : 0;
            MoveCtx mc;
            move_ctx_init(tab, b, mc);
            unsigned any = __ballot_sync(0xFFFFFFFFu, empt != 0);
            while (any) {
                int k = -1;
                if (empt) {
                    k = (__ffsll((long long)empt) - 1) >> 2;
                    empt &= empt - 1;
                }
#pragma unroll 1
                for (int v = 1; v <= 2; ++v) {
                    uint64_t *const sbuf = stage[warp][v - 1];
                    int c = v == 1 ? cnt1 : cnt2;
                    uint64_t keys[4];
                    const unsigned kept = spawn_children<false>(tab, mc, k, (uint64_t)v, tb.spec, tb.filter, tb.filter_bits,
                                                         keys, probes);
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
                            if (c > kStage - 32) {
                                const int L = t + v;
                                stage_flush_dedup<false>(sbuf, c, tb.stage[L % 3], &C[i].stage_count[L % 3], tb.stage_cap,
                                                  tb.set[L & 1], tb.set_mask, tb.s0 + 2ll * L, bsum, &C[i].err);
                            }
                        }
                    }
                    if (v == 1) cnt1 = c; else cnt2 = c;
                }
                any = __ballot_sync(0xFFFFFFFFu, empt != 0);
            }
        }
    }
    if (cur >= 0 && T[cur].steps - 3 >= t) flush_table();
    // the last block to finish empties every table's staging buffer of layer t
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last_block = atomicAdd(&sync->blocks_done, 1ull) == (unsigned long long)gridDim.x - 1;
    __syncthreads();
    if (last_block) {
        __threadfence();
        for (int i = threadIdx.x; i < n_tables; i += blockDim.x)
            if (t < T[i].steps) C[i].stage_count[sp] = 0;
        if (threadIdx.x == 0) {
            sync->blocks_done = 0;
            sync->next_item = 0;
            if (progress) *(volatile unsigned *)progress = progress_value;
        }
    }
}

// Zero `words` 16-byte words at p with every thread of the grid.
__device__ __forceinline__ void grid_zero16(void *p, unsigned long long words) {
    uint4 *z = reinterpret_cast<uint4 *>(p);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < words;
         i += (unsigned long long)gridDim.x * blockDim.x)
        z[i] = make_uint4(0u, 0u, 0u, 0u);
}

// ------------------------------------------------------------ backward ----
//
// Four rate-index planes per table (layer L in plane L % 4), all zeroed before
// the backward pass; the solve of step t inserts layer t into plane t % 4 and
// zeroes plane (t-1) % 4, whose last layer (t+3) was read by steps t+1 and
// t+2, for the inserts of step t-1. A probe stops at a zero key.

// Layers steps-2 and steps-1 of every table: success -> max, else zero
// (final_situation_process, native_core/src/BookSolver.cpp:237-261); live
// entries of layers >= 1 enter their index plane.
template <typename T>
__global__ void __launch_bounds__(256)
batch_final_kernel(const BatchTable *__restrict__ TB, BatchCtl *C, int n_tables, const uint64_t *__restrict__ arena,
                   T *__restrict__ rates, const unsigned long long *__restrict__ layer_off,
                   const unsigned long long *__restrict__ layer_len, T zero, T maxv) {
    __shared__ unsigned long long pre[2 * kMaxBatchTables + 1];
    __shared__ unsigned long long scan_sm[33];
    const int nseg = 2 * n_tables;
    seg_prefix(nseg, pre, scan_sm, [&](int s) -> unsigned long long {
        const BatchTable &tb = TB[s >> 1];
        const int L = tb.steps - 2 + (s & 1);
        return L >= 0 ? layer_len[tb.lbase + L] : 0ull;
    });
    const unsigned long long total = pre[nseg];
    for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (unsigned long long)gridDim.x * blockDim.x) {
        const int s = seg_find(pre, nseg, g);
        const int i = s >> 1;
        const BatchTable &tb = TB[i];
        const int L = tb.steps - 2 + (s & 1);
        const unsigned long long o = layer_off[tb.lbase + L] + (g - pre[s]);
        const uint64_t b = arena[o];
        const T r = is_success(b, tb.spec) ? maxv : zero;
        rates[o] = r;
        if (L >= 1 && r > zero) index_insert_zero<T>(tb.index[L % 4], tb.index_mask, b, r, &C[i].err);
    }
}

// Backward step t of every table with t <= steps-3 (recalculate_layer,
// native_core/src/BookSolver.cpp:413-470; same arithmetic as solve_kernel),
// then layer t's live entries enter index plane t % 4 for steps t-1 and t-2.
template <typename T>
__global__ void __launch_bounds__(256, 3)
batch_solve_kernel(const BatchTable *__restrict__ TB, BatchCtl *C, int n_tables, int t,
                   const uint64_t *__restrict__ arena, T *__restrict__ rates,
                   const unsigned long long *__restrict__ layer_off, const unsigned long long *__restrict__ layer_len,
                   const uint32_t *__restrict__ tab, T zero, T maxv, BatchSync *sync, unsigned *progress,
                   unsigned progress_value) {
    __shared__ unsigned long long pre[kMaxBatchTables + 1];
    __shared__ unsigned long long scan_sm[33];
    seg_prefix(n_tables, pre, scan_sm, [&](int i) -> unsigned long long {
        return t <= TB[i].steps - 3 ? layer_len[TB[i].lbase + t] : 0ull;
    });
    if (t >= 2)
        for (int i = 0; i < n_tables; ++i)
            if (t <= TB[i].steps - 3) grid_zero16(TB[i].index[(t - 1) % 4], TB[i].index_mask + 1);
    if (progress && blockIdx.x == 0 && threadIdx.x == 0) *(volatile unsigned *)progress = progress_value;
    const unsigned long long total = pre[n_tables];
    unsigned long long looks = 0;
    for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (unsigned long long)gridDim.x * blockDim.x) {
        const int i = seg_find(pre, n_tables, g);
        const BatchTable &tb = TB[i];
        const unsigned long long o = layer_off[tb.lbase + t] + (g - pre[i]);
        const uint64_t b = arena[o];
        T r;
        if (t > tb.docheck && is_success(b, tb.spec)) {
            r = maxv;
        } else {
            const double p4 = tb.p4, w2 = 1.0 - p4;
            const ulonglong2 *idx1 = tb.index[(t + 1) % 4], *idx2 = tb.index[(t + 2) % 4];
            const unsigned long long m = tb.index_mask;
            MoveCtx mc;
            move_ctx_init(tab, b, mc);
            uint64_t empt = empty_nibbles(b);
            double acc = 0.0;
            int nempty = 0;
            while (empt) {
                const int k = (__ffsll((long long)empt) - 1) >> 2;
                empt &= empt - 1;
                ++nempty;
                uint64_t key[8];
                unsigned pend = 0;
#pragma unroll
                for (int v = 1; v <= 2; ++v) {
                    uint64_t mv[4], s;
                    spawn_moves(tab, mc, k, (uint64_t)v, s, mv);
#pragma unroll
                    for (int d = 0; d < 4; ++d) {
                        const int j = (v - 1) * 4 + d;
                        key[j] = canonical<false>(mv[d], tb.spec.symm);  // batched tables: modes 0-3
                        if (mv[d] != s && is_pattern(mv[d], tb.spec)) pend |= 1u << j;
                    }
                }
                looks += __popc(pend);
                unsigned long long h[8];
                T got[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    got[j] = zero;
                    h[j] = mix64(key[j]) & m;
                }
                int guard = 0;
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
                                h[j] = (h[j] + 1) & m;
                            }
                        }
                    }
                    if (++guard > kMaxProbe * 32) {
                        atomicOr(&C[i].err, kErrIndexOverflow);
                        break;
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
            r = nempty > 0 ? cast_rate<T>(acc / (double)nempty) : zero;
        }
        rates[o] = r;
        if (t > 0 && r > zero) index_insert_zero<T>(tb.index[t % 4], tb.index_mask, b, r, &C[i].err);
    }
    for (int o = 16; o > 0; o >>= 1) looks += __shfl_xor_sync(0xFFFFFFFFu, looks, o);
    if ((threadIdx.x & 31) == 0 && looks) atomicAdd(&sync->lookups, looks);
}

}  // namespace egtb
