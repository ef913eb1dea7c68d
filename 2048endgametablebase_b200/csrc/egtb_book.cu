// Book lookup of libegtb_gpu: books of a table held in device memory as
// sorted keys + rates (+ one splitter per 16 keys) and a batched kernel that
// answers move_on_dic for many positions at once (the reader side of the
// reference, native_core/src/ReaderRuntime.cpp:739-840 and 1050-1133).
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "egtb_host.h"
#include "egtb_device.cuh"
#include "egtb_trie.h"

namespace egtb {

struct BookLayer {
    uint64_t *keys = nullptr;
    void *rates = nullptr;
    uint64_t *split = nullptr;
    ulonglong2 *index = nullptr;  // sorted layers: {key, rate bits} hash index
    unsigned long long index_mask = 0;
    unsigned long long n = 0;
    int state = 0;  // 0 not looked at, 1 loaded, 2 file missing
    int sorted = 1;
    // compressed layer (<name>_<t>.z): its trie levels and block table; the
    // decoded entries' low 32 bits in `low`, their rates in `rates`
    int compressed = 0;
    uint8_t *i_key = nullptr, *ii_key = nullptr;
    uint32_t *i_next = nullptr, *seg_index = nullptr, *low = nullptr;
    uint16_t *ii_next = nullptr;
    unsigned long long *block_end = nullptr;
    unsigned long long n_i = 0, n_ii = 0, n_seg = 0;
    struct TrieDesc *d_trie = nullptr;  // the device copy of the above (TrieDesc)
};

// A compressed layer as the lookup kernel reads it (one per such layer, in
// device memory, pointed to by its LayerDesc).
struct TrieDesc {
    const uint8_t *i_key, *ii_key;
    const uint32_t *i_next, *seg_index, *low;
    const uint16_t *ii_next;
    const unsigned long long *block_end;
    unsigned long long n_i, n_ii, n_seg;
};

// Layer descriptor read by the lookup kernel.
struct LayerDesc {
    const uint64_t *keys;
    const void *rates;
    const uint64_t *split;
    const ulonglong2 *index;
    unsigned long long index_mask;
    unsigned long long n;
    int exists;
    int sorted;
    const TrieDesc *trie;  // compressed layer (keys / split / index unused), else null
};

// ------------------------------------------------------ layer hash index ---
//
// A sorted book layer (unique keys) also gets an open-addressing index of
// 16-byte slots {key, rate bits}, capacity a power of two of at least twice
// its entries, key 0 = empty (no board is 0): a search is ~1.3 dependent
// 16-byte loads instead of a ~20-step binary search, and it finds exactly what
// the binary search finds (the key's rate, or nothing).

template <typename T> __device__ __forceinline__ unsigned long long book_rate_bits(T r) {
    unsigned long long b = 0;
    memcpy(&b, &r, sizeof(T));
    return b;
}

template <typename T> __device__ __forceinline__ T book_rate_from_bits(unsigned long long b) {
    T r;
    memcpy(&r, &b, sizeof(T));
    return r;
}

template <typename T>
__global__ void __launch_bounds__(256)
book_index_kernel(const uint64_t *__restrict__ keys, const T *__restrict__ rates, unsigned long long n,
                  ulonglong2 *__restrict__ slots, unsigned long long mask) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t key = keys[i];
        unsigned long long h = mix64(key) & mask;
        for (unsigned long long probe = 0; probe <= mask; ++probe) {  // at most half full: ends long before
            const unsigned long long prev = atomicCAS(&slots[h].x, 0ull, (unsigned long long)key);
            if (prev == 0ull || prev == key) {
                slots[h].y = book_rate_bits<T>(rates[i]);
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

// The four move lookups of one position at once: every first slot load is
// issued before any is compared, so a thread has up to four misses in flight
// instead of one dependent chain after another.
template <typename T>
__device__ __forceinline__ void index_lookup4(const ulonglong2 *__restrict__ slots, unsigned long long mask,
                                              const uint64_t key[4], unsigned pend, T zero, T r[4]) {
    unsigned long long h[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        r[d] = zero;
        h[d] = mix64(key[d]) & mask;
    }
    for (unsigned long long probe = 0; pend && probe <= mask; ++probe) {
        ulonglong2 sl[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) sl[d] = (pend >> d & 1u) ? __ldg(slots + h[d]) : make_ulonglong2(0ull, 0ull);
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            if (!(pend >> d & 1u)) continue;
            if (sl[d].x == key[d]) {
                r[d] = book_rate_from_bits<T>(sl[d].y);
                pend &= ~(1u << d);
            } else if (sl[d].x == 0ull) {
                pend &= ~(1u << d);
            } else {
                h[d] = (h[d] + 1) & mask;
            }
        }
    }
}

}  // namespace egtb

struct egtb_book {
    std::string dir, pattern_full;
    int dtype = 0;
    int device = 0;
    long long nums_adjust = 0;
    bool variant = false;  // variant boards: wall-merge moves, the board as given only
    egtb::DevSpec spec;
    std::vector<egtb::BookLayer> layers;
    egtb::LayerDesc *d_desc = nullptr;
    int d_desc_cap = 0;
    bool desc_dirty = true;
    bool any_compressed = false;  // some loaded layer is a compressed (.z) one
    cudaStream_t stream = nullptr;
    std::mutex mu;
    // scratch for host-buffer lookups
    uint64_t *d_pos = nullptr;
    double *d_val = nullptr;
    uint8_t *d_valid = nullptr;
    int8_t *d_op = nullptr;
    size_t scratch_cap = 0;
};

namespace egtb {

static std::string layer_path(const egtb_book &b, long long nums) {
    return b.dir + "/" + b.pattern_full + "_" + std::to_string(nums) + ".book";
}

template <typename T>
__global__ void split_records_kernel(const unsigned char *__restrict__ recs, unsigned long long n,
                                     uint64_t *__restrict__ keys, T *__restrict__ rates, uint64_t *__restrict__ split,
                                     int *__restrict__ unsorted) {
    constexpr int rec = 8 + (int)sizeof(T);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t *w = reinterpret_cast<const uint32_t *>(recs + i * rec);
        const uint64_t k = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
        keys[i] = k;
        T r;
        memcpy(&r, recs + i * rec + 8, sizeof(T));
        rates[i] = r;
        if ((i % kSplitStride) == 0) split[i / kSplitStride] = k;
        if (i > 0) {
            const uint32_t *q = reinterpret_cast<const uint32_t *>(recs + (i - 1) * rec);
            const uint64_t kp = (uint64_t)q[0] | ((uint64_t)q[1] << 32);
            if (kp >= k) *unsorted = 1;
        }
    }
}

template <typename V>
static V *upload(const std::vector<V> &h, cudaStream_t s) {
    V *d = nullptr;
    EGTB_CUDA(cudaMalloc(&d, std::max<size_t>(h.size(), 1) * sizeof(V)));
    if (!h.empty()) EGTB_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, s));
    return d;
}

// Load a compressed layer: every xz block decoded on the host (threads), the
// trie levels, block table and decoded entries uploaded as they are; the
// lookup kernel searches them the way the reference's reader does.
static bool load_compressed_layer(egtb_book &b, BookLayer &L, long long nums) {
    const std::string zdir = b.dir + "/" + b.pattern_full + "_" + std::to_string(nums) + ".z";
    struct stat st;
    if (::stat(zdir.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) return false;
    TrieLayer z;
    const size_t es = dtype_size(b.dtype);
    const int threads = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (!read_compressed_book(zdir, b.pattern_full + "_" + std::to_string(nums) + ".", es, z, threads)) return false;
    cudaStream_t s = b.stream;
    L.i_key = upload(z.i_key, s);
    L.i_next = upload(z.i_next, s);
    L.ii_key = upload(z.ii_key, s);
    L.ii_next = upload(z.ii_next, s);
    L.seg_index = upload(z.seg_index, s);
    std::vector<unsigned long long> be(z.block_end.begin(), z.block_end.end());
    L.block_end = upload(be, s);
    L.low = upload(z.low, s);
    L.rates = upload(z.rates, s);
    L.n_i = z.i_key.size();
    L.n_ii = z.ii_key.size();
    L.n_seg = z.seg_index.size();
    const TrieDesc td{L.i_key, L.ii_key, L.i_next, L.seg_index, L.low, L.ii_next, L.block_end, L.n_i, L.n_ii, L.n_seg};
    EGTB_CUDA(cudaMalloc(&L.d_trie, sizeof(TrieDesc)));
    EGTB_CUDA(cudaMemcpyAsync(L.d_trie, &td, sizeof td, cudaMemcpyHostToDevice, s));
    L.n = z.low.size();
    L.compressed = 1;
    L.sorted = 1;
    b.any_compressed = true;
    EGTB_CUDA(cudaStreamSynchronize(s));
    return true;
}

// Load layer `nums` from its .book file, else from its compressed .z
// directory (state 2 when neither is there).
static void load_layer(egtb_book &b, long long nums) {
    if (nums < 0) return;
    if ((long long)b.layers.size() <= nums) b.layers.resize(nums + 1);
    BookLayer &L = b.layers[nums];
    const std::string path = layer_path(b, nums);
    if (L.state == 1) return;
    if (!file_exists(path)) {
        L.state = load_compressed_layer(b, L, nums) ? 1 : 2;
        b.desc_dirty = true;
        return;
    }
    const size_t rec = record_size(b.dtype);
    std::vector<unsigned char> host = read_file(path);
    const unsigned long long n = host.size() / rec;
    L.n = n;
    const size_t es = dtype_size(b.dtype);
    EGTB_CUDA(cudaMalloc(&L.keys, std::max<size_t>(n, 1) * 8));
    EGTB_CUDA(cudaMalloc(&L.rates, std::max<size_t>(n, 1) * es));
    EGTB_CUDA(cudaMalloc(&L.split, (n / kSplitStride + 1) * 8));
    if (n) {
        unsigned char *d = nullptr;
        int *d_flag = nullptr;
        EGTB_CUDA(cudaMalloc(&d, n * rec));
        EGTB_CUDA(cudaMalloc(&d_flag, sizeof(int)));
        EGTB_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), b.stream));
        EGTB_CUDA(cudaMemcpyAsync(d, host.data(), n * rec, cudaMemcpyHostToDevice, b.stream));
        const int grid = 592;
        if (es == 4) {
            if (b.dtype == EGTB_DTYPE_UINT32)
                split_records_kernel<uint32_t><<<grid, 256, 0, b.stream>>>(d, n, L.keys, (uint32_t *)L.rates, L.split, d_flag);
            else
                split_records_kernel<float><<<grid, 256, 0, b.stream>>>(d, n, L.keys, (float *)L.rates, L.split, d_flag);
        } else {
            if (b.dtype == EGTB_DTYPE_UINT64)
                split_records_kernel<uint64_t><<<grid, 256, 0, b.stream>>>(d, n, L.keys, (uint64_t *)L.rates, L.split, d_flag);
            else
                split_records_kernel<double><<<grid, 256, 0, b.stream>>>(d, n, L.keys, (double *)L.rates, L.split, d_flag);
        }
        int unsorted = 0;
        EGTB_CUDA(cudaMemcpyAsync(&unsorted, d_flag, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
        EGTB_CUDA(cudaStreamSynchronize(b.stream));
        EGTB_CUDA(cudaGetLastError());
        cudaFree(d);
        cudaFree(d_flag);
        L.sorted = unsorted ? 0 : 1;
        if (L.sorted) {
            unsigned long long slots = 64;
            while (slots < 2 * n) slots <<= 1;
            EGTB_CUDA(cudaMalloc(&L.index, slots * sizeof(ulonglong2)));
            EGTB_CUDA(cudaMemsetAsync(L.index, 0, slots * sizeof(ulonglong2), b.stream));
            L.index_mask = slots - 1;
            switch (b.dtype) {
                case EGTB_DTYPE_UINT32:
                    book_index_kernel<uint32_t><<<grid, 256, 0, b.stream>>>(L.keys, (const uint32_t *)L.rates, n, L.index,
                                                                          L.index_mask);
                    break;
                case EGTB_DTYPE_UINT64:
                    book_index_kernel<uint64_t><<<grid, 256, 0, b.stream>>>(L.keys, (const uint64_t *)L.rates, n, L.index,
                                                                          L.index_mask);
                    break;
                case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32:
                    book_index_kernel<float><<<grid, 256, 0, b.stream>>>(L.keys, (const float *)L.rates, n, L.index,
                                                                       L.index_mask);
                    break;
                default:
                    book_index_kernel<double><<<grid, 256, 0, b.stream>>>(L.keys, (const double *)L.rates, n, L.index,
                                                                        L.index_mask);
                    break;
            }
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaStreamSynchronize(b.stream));
        }
    }
    L.state = 1;
    b.desc_dirty = true;
}

static void upload_desc(egtb_book &b) {
    if (!b.desc_dirty) return;
    const int n = (int)b.layers.size();
    if (n > b.d_desc_cap) {
        if (b.d_desc) cudaFree(b.d_desc);
        b.d_desc_cap = std::max(n, 64);
        EGTB_CUDA(cudaMalloc(&b.d_desc, sizeof(LayerDesc) * b.d_desc_cap));
    }
    std::vector<LayerDesc> h(std::max(n, 1));
    for (int i = 0; i < n; ++i) {
        const BookLayer &L = b.layers[i];
        h[i] = {L.keys, L.rates, L.split, L.index, L.index_mask, L.n, L.state == 1 ? 1 : 0, L.sorted,
                L.compressed ? L.d_trie : nullptr};
    }
    if (n) EGTB_CUDA(cudaMemcpyAsync(b.d_desc, h.data(), sizeof(LayerDesc) * n, cudaMemcpyHostToDevice, b.stream));
    EGTB_CUDA(cudaStreamSynchronize(b.stream));
    b.desc_dirty = false;
}

__device__ __forceinline__ long long tile_sum(uint64_t b) {
    long long s = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int v = (int)((b >> (4 * k)) & 0xF);
        s += v ? (1ll << v) : 0ll;
    }
    return s;
}

// find_success_entry_in_file's probe sequence (ReaderRuntime.cpp:279-316),
// used for layers whose file is not in ascending order (a table's layer 0
// holds the seeds as given).
template <typename T>
__device__ __forceinline__ bool probe_unsorted(const uint64_t *keys, const T *rates, unsigned long long n, uint64_t key,
                                               T &out) {
    if (n == 0) return false;
    unsigned long long left = 0, right = n - 1;
    while (left <= right) {
        const unsigned long long mid = (left + right) / 2;
        const uint64_t k = keys[mid];
        if (k == key) {
            out = rates[mid];
            return true;
        }
        if (k < key) {
            left = mid + 1;
        } else {
            if (mid == 0) break;
            right = mid - 1;
        }
    }
    return false;
}

// Search of a compressed layer, step for step as trie_search_with_context
// (ReaderRuntime.cpp:318-477) runs it over the files: three binary searches
// down the byte-7/6/5 levels of i, one over the byte-4 groups in ii, the
// block whose s entry is the first at or after the group, then a lower-bound
// search of the low 32 bits inside the range the group's neighbours give.
// The reference's range rules are kept as they are, including its reading of
// a relative `next` of 0 and its first-entry check, so every answer (hit,
// miss, or the entry those rules land on) is the reference's. *out = the
// rate found, or zero.
template <typename T>
__device__ __forceinline__ void trie_find(const TrieDesc &L, const T *__restrict__ rates, uint64_t board, T zero, T &out) {
    out = zero;
    if (L.n_i < 2 || L.n_seg < 2) return;
    unsigned long long low = 2, high = (unsigned long long)L.i_next[1] - 1ull;
    for (int level = 0; level < 3; ++level) {
        const uint8_t want = (uint8_t)(board >> (56 - 8 * level));
        if (high >= L.n_i) high = L.n_i - 1;  // stays inside i (a well-formed file never needs it)
        bool found = false;
        unsigned long long mid = low;
        while (low <= high) {
            mid = (low + high) / 2;
            const uint8_t k = L.i_key[mid];
            if (k == want) {
                found = true;
                break;
            }
            if (k < want) {
                low = mid + 1;
            } else {
                if (mid == 0) break;
                high = mid - 1;
            }
        }
        if (!found) return;
        low = (unsigned long long)L.i_next[mid - 1] + 1ull;
        high = L.i_next[mid];
    }
    // ii entries low-1 .. high: the groups under the byte-5 entry and the one before
    const unsigned long long first = low - 1, count = high - low + 2;
    if (count <= 1 || first + count > L.n_ii) return;
    const uint8_t want4 = (uint8_t)(board >> 32);
    unsigned long long lo = 1, hi = count - 1, pos = 0;
    bool found = false;
    while (lo <= hi) {
        const unsigned long long mid = (lo + hi) / 2;
        const uint8_t k = L.ii_key[first + mid];
        if (k == want4) {
            pos = mid - 1;
            found = true;
            break;
        }
        if (k < want4) {
            lo = mid + 1;
        } else {
            if (mid == 0) break;
            hi = mid - 1;
        }
    }
    if (!found) return;
    // the block: the first s entry at or after ii index pos + low
    const unsigned long long target = pos + low;
    long long blk = -1;
    {
        unsigned long long a = 0, c = L.n_seg - 1;
        while (a <= c) {
            const unsigned long long mid = (a + c) / 2;
            if ((unsigned long long)L.seg_index[mid] < target) {
                a = mid + 1;
            } else {
                blk = (long long)mid;
                if (mid == 0) break;
                c = mid - 1;
            }
        }
    }
    unsigned long long base = 0, size = 0;
    if (blk >= 1) {
        base = L.block_end[blk - 1];
        size = L.block_end[blk] - base;
    }
    const uint32_t t32 = (uint32_t)board;
    unsigned long long sub_low = L.ii_next[first + pos], sub_high = (unsigned long long)L.ii_next[first + pos + 1] + 1;
    if (sub_high == 1) {
        if (size != 0 && t32 == L.low[base]) {
            out = rates[base];
            return;
        }
        sub_high = size;
    }
    if (sub_low != 0) ++sub_low;
    if (sub_high > size) sub_high = size;  // stays inside the block (a well-formed file never needs it)
    while (sub_low < sub_high) {
        const unsigned long long mid = (sub_low + sub_high) / 2;
        if (L.low[base + mid] < t32) sub_low = mid + 1;
        else sub_high = mid;
    }
    if (sub_low < size && L.low[base + sub_low] == t32) out = rates[base + sub_low];
}

// normalize_raw_value + maybe_round_value (ReaderRuntime.cpp:208-214,271-277):
// integer kinds divide by their scale; names containing "32" are rounded to
// 9 decimals above 1e-7. The reference's -Ofast build turns the division by
// 10^9 into a multiplication by its reciprocal, reproduced here.
template <typename T>
__device__ __forceinline__ double present(T raw, double scale, int round9) {
    double v = (double)raw;
    if (scale > 1.0) v = v / scale;
    if (round9 && fabs(v) > 1e-7) v = round(v * 1e9) * 1e-9;
    return v;
}

// Operation index -> symmetry applied to the board (apply_operation,
// ReaderRuntime.cpp:127-147, as cell maps).
__device__ __constant__ int kOpSym[8] = {0, 6, 5, 7, 1, 4, 2, 3};

// adjust_direction (ReaderRuntime.cpp:149-169) for the move index m of the
// transformed board (0 left, 1 right, 2 up, 3 down); returns the slot in the
// order up, right, down, left.
__device__ __forceinline__ int adjusted_slot(int op, int m) {
    // name of move m: left=3, right=1, up=0, down=2 in {up,right,down,left}
    int idx = (m == 0) ? 3 : (m == 1) ? 1 : (m == 2) ? 0 : 2;
    if (op >= 4) {
        if (idx == 3) idx = 1;
        else if (idx == 1) idx = 3;
    }
    return (idx + (op & 3)) & 3;
}

// move_on_dic of one position (evaluate_classic_result_candidates,
// native_core/src/ReaderRuntime.cpp:739-840): four values in direction order
// up, right, down, left, the mask of directions with a value, and the op used.
// kTrie: the build that also searches compressed layers (taken only for books
// that have some; the plain build keeps the registers of the hash search).
template <typename T, typename OutT, bool kVariantModes, bool kTrie>
__device__ __forceinline__ void lookup_position(const LayerDesc *__restrict__ desc, int n_desc, uint64_t board,
                                                long long nums_adjust, const DevSpec &spec,
                                                const uint32_t *__restrict__ tab, int op_mode, double scale,
                                                int round9, T zero, OutT out[4], uint8_t &mask, int &used) {
#pragma unroll
    for (int d = 0; d < 4; ++d) out[d] = 0;
    mask = 0;
    used = -1;
    const long long nums = (tile_sum(board) + nums_adjust) / 2;  // C division, ReaderRuntime.cpp:749
    if (nums < 0) {
        used = -2;
        return;
    }
    if (nums >= n_desc || !desc[nums].exists) {
        used = -3;
        return;
    }
    const LayerDesc L = desc[nums];
    const T *rates = (const T *)L.rates;
    // [last_op, 0..7] (operation_sequence, ReaderRuntime.cpp:171-182), or one op
    const int single = op_mode >= 8 ? op_mode - 8 : -1;
    const int count = single >= 0 ? 1 : 9;
    for (int j = 0; j < count && used < 0; ++j) {
        const int op = single >= 0 ? single : (j == 0 ? op_mode : j - 1);
        const uint64_t tb = apply_sym(board, kOpSym[op]);
        if (!is_pattern(tb, spec)) continue;
        uint64_t mv[4], key[4];
        move_all_dir(tab, tb, mv);
        unsigned live = 0;  // moves that moved and stay in the pattern
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            key[d] = 0;
            if (mv[d] == tb || !is_pattern(mv[d], spec)) continue;
            key[d] = canonical<kVariantModes>(mv[d], spec.symm);
            live |= 1u << d;
        }
        T r[4];
        if (kTrie && L.trie) {
            const TrieDesc Z = *L.trie;
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                r[d] = zero;
                if (live >> d & 1u) trie_find<T>(Z, rates, key[d], zero, r[d]);
            }
        } else if (L.sorted && L.index) {
            index_lookup4<T>(L.index, L.index_mask, key, live, zero, r);
        } else {
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                r[d] = zero;
                if (!(live >> d & 1u)) continue;
                if (L.sorted) {
                    r[d] = layer_lookup<T>(L.keys, rates, L.n, L.split, key[d], zero);
                } else {
                    T got;
                    if (probe_unsorted<T>(L.keys, rates, L.n, key[d], got)) r[d] = got;
                }
            }
        }
        uint8_t m = 0;
        OutT vals[4] = {0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            if (!(live >> d & 1u)) continue;
            const int slot = adjusted_slot(op, d);
            vals[slot] = (OutT)present<T>(r[d], scale, round9);
            m |= (uint8_t)(1u << slot);
        }
        if (m) {
            used = op;
            mask = m;
#pragma unroll
            for (int d = 0; d < 4; ++d) out[d] = vals[d];
        }
    }
}

template <typename T, typename OutT, bool kVariantModes, bool kTrie>
__global__ void __launch_bounds__(256)
lookup_kernel(const LayerDesc *__restrict__ desc, int n_desc, const uint64_t *__restrict__ pos, size_t n,
              long long nums_adjust, DevSpec spec, const uint32_t *__restrict__ tab, int op_mode, double scale,
              int round9, T zero, OutT *__restrict__ values4, uint8_t *__restrict__ valid, int8_t *__restrict__ op_used) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        OutT out[4];
        uint8_t mask;
        int used;
        lookup_position<T, OutT, kVariantModes, kTrie>(desc, n_desc, pos[i], nums_adjust, spec, tab, op_mode, scale, round9, zero, out,
                                 mask, used);
#pragma unroll
        for (int d = 0; d < 4; ++d) values4[4 * i + d] = out[d];
        valid[i] = mask;
        if (op_used) op_used[i] = (int8_t)used;
    }
}

// The same over a list of requests whose positions and answers live in
// caller memory the device can address (registered host memory): request r
// covers work items prefix[r] .. prefix[r+1]-1.
template <typename T, bool kVariantModes, bool kTrie>
__global__ void __launch_bounds__(256)
lookup_requests_kernel(const LayerDesc *__restrict__ desc, int n_desc, const ServeReq *__restrict__ reqs, int n_req,
                       long long nums_adjust, DevSpec spec, const uint32_t *__restrict__ tab, int op_mode,
                       double scale, int round9, T zero) {
    const unsigned long long total = reqs[n_req].at;
    for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (unsigned long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_req;  // largest r with reqs[r].at <= g
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (reqs[mid].at <= g) lo = mid; else hi = mid;
        }
        const ServeReq q = reqs[lo];
        const unsigned long long i = g - q.at;
        float out[4];
        uint8_t mask;
        int used;
        lookup_position<T, float, kVariantModes, kTrie>(desc, n_desc, q.pos[i], nums_adjust, spec, tab, op_mode, scale, round9, zero, out,
                                  mask, used);
        reinterpret_cast<float4 *>(q.out)[i] = make_float4(out[0], out[1], out[2], out[3]);
        if (q.valid) q.valid[i] = mask;
    }
}

static bool round9_for(int dtype) {
    // names containing "32": uint32, float32, 1-float32
    return dtype == EGTB_DTYPE_UINT32 || dtype == EGTB_DTYPE_FLOAT32 || dtype == EGTB_DTYPE_1_FLOAT32;
}

static double scale_for(int dtype) {
    // dtype_info_for_name max_scale (ReaderRuntime.cpp:186-206); only > 1 divides
    if (dtype == EGTB_DTYPE_UINT32) return 4e9;
    if (dtype == EGTB_DTYPE_UINT64) return 1.6e18;
    return dtype_is_one_minus(dtype) ? 0.0 : 1.0;
}

template <typename OutT>
static void launch_lookup(egtb_book &b, const uint64_t *d_pos, size_t n, int op_mode, OutT *d_vals, uint8_t *d_valid,
                          int8_t *d_op, cudaStream_t s) {
    const uint32_t *tab = device_row_table(b.variant);
    // a variant reader tries the board as given only (operation_sequence,
    // ReaderRuntime.cpp:171-182): single operation 0
    if (b.variant) op_mode = 8;
    const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    if (n == 0) return;
    const double scale = scale_for(b.dtype);
    const int r9 = round9_for(b.dtype) ? 1 : 0;
    const int nd = (int)b.layers.size();
    // the kernel build with the variant symmetry modes only for tables that use
    // them, the one with the compressed-layer search only for books that have such layers
    auto run = [&](auto variant_modes, auto trie) {
        constexpr bool W = decltype(variant_modes)::value;
        constexpr bool Z = decltype(trie)::value;
        switch (b.dtype) {
            case EGTB_DTYPE_UINT32:
                lookup_kernel<uint32_t, OutT, W, Z><<<grid, 256, 0, s>>>(b.d_desc, nd, d_pos, n, b.nums_adjust, b.spec, tab, op_mode,
                                                                   scale, r9, 0u, d_vals, d_valid, d_op);
                break;
            case EGTB_DTYPE_UINT64:
                lookup_kernel<uint64_t, OutT, W, Z><<<grid, 256, 0, s>>>(b.d_desc, nd, d_pos, n, b.nums_adjust, b.spec, tab, op_mode,
                                                                   scale, r9, 0ull, d_vals, d_valid, d_op);
                break;
            case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32:
                lookup_kernel<float, OutT, W, Z><<<grid, 256, 0, s>>>(b.d_desc, nd, d_pos, n, b.nums_adjust, b.spec, tab, op_mode,
                                                                scale, r9, (float)dtype_zero(b.dtype), d_vals, d_valid, d_op);
                break;
            default:
                lookup_kernel<double, OutT, W, Z><<<grid, 256, 0, s>>>(b.d_desc, nd, d_pos, n, b.nums_adjust, b.spec, tab, op_mode,
                                                                 scale, r9, dtype_zero(b.dtype), d_vals, d_valid, d_op);
                break;
        }
    };
    const bool trie = b.any_compressed;
    if (b.spec.symm >= 4) {
        if (trie) run(std::true_type{}, std::true_type{});
        else run(std::true_type{}, std::false_type{});
    } else {
        if (trie) run(std::false_type{}, std::true_type{});
        else run(std::false_type{}, std::false_type{});
    }
    EGTB_CUDA(cudaGetLastError());
}

static long long host_tile_sum(uint64_t b) {
    long long s = 0;
    for (int k = 0; k < 16; ++k) {
        const int v = (int)((b >> (4 * k)) & 0xF);
        s += v ? (1ll << v) : 0ll;
    }
    return s;
}

// ----------------------------------------------- single-file value cache --

struct FileBook {
    std::string path;
    uint64_t size = 0;
    int dtype = 0;
    BookLayer layer;
};

static std::mutex g_fb_mu;
static std::vector<std::unique_ptr<FileBook>> g_fb;  // small LRU by path

template <typename T>
__global__ void find_one_kernel(const uint64_t *keys, const T *rates, unsigned long long n, int sorted, uint64_t key,
                                double scale, T zero, double *out) {
    // find_success_entry_in_file (ReaderRuntime.cpp:279-316): a hit gives the
    // normalised value, a miss the dtype's zero value as it is
    bool hit = false;
    T r = zero;
    if (sorted) {
        unsigned long long lo = 0, len = n;
        while (len > 0) {
            const unsigned long long half = len >> 1;
            if (keys[lo + half] < key) {
                lo += half + 1;
                len -= half + 1;
            } else {
                len = half;
            }
        }
        hit = lo < n && keys[lo] == key;
        if (hit) r = rates[lo];
    } else {
        hit = probe_unsorted<T>(keys, rates, n, key, r);
    }
    double v = (double)r;
    if (hit && scale > 1.0) v = v / scale;
    *out = hit ? v : (double)zero;
}

}  // namespace egtb

using namespace egtb;

extern "C" int egtb_book_open(const char *dir, const char *pattern_full, int32_t dtype, const egtb_pattern_spec *spec,
                              int64_t nums_adjust, int32_t device, egtb_book **out) {
    return guarded([&] {
        if (!dir || !pattern_full || !spec || !out) throw Error(EGTB_ERR_ARG, "NULL argument");
        dtype_size(dtype);
        int n = 0;
        EGTB_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw Error(EGTB_ERR_ARG, "device not present");
        EGTB_CUDA(cudaSetDevice(device));
        auto b = std::make_unique<egtb_book>();
        b->dir = dir;
        while (b->dir.size() > 1 && b->dir.back() == '/') b->dir.pop_back();
        b->pattern_full = pattern_full;
        b->dtype = dtype;
        b->device = device;
        b->nums_adjust = nums_adjust;
        b->spec = make_dev_spec(*spec, 0);
        EGTB_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        *out = b.release();
    });
}

extern "C" int egtb_book_set_variant(egtb_book *b, int32_t is_variant) {
    return guarded([&] {
        if (!b) throw Error(EGTB_ERR_ARG, "NULL book");
        std::lock_guard<std::mutex> lk(b->mu);
        b->variant = is_variant != 0;
    });
}

extern "C" int egtb_book_close(egtb_book *b) {
    return guarded([&] {
        if (!b) return;
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->stream);
        for (auto &L : b->layers) {
            for (void *p : {(void *)L.keys, L.rates, (void *)L.split, (void *)L.index, (void *)L.i_key, (void *)L.ii_key,
                            (void *)L.i_next, (void *)L.seg_index, (void *)L.low, (void *)L.ii_next, (void *)L.d_trie,
                            (void *)L.block_end})
                if (p) cudaFree(p);
        }
        if (b->d_desc) cudaFree(b->d_desc);
        if (b->d_pos) cudaFree(b->d_pos);
        if (b->d_val) cudaFree(b->d_val);
        if (b->d_valid) cudaFree(b->d_valid);
        if (b->d_op) cudaFree(b->d_op);
        cudaStreamDestroy(b->stream);
        delete b;
    });
}

extern "C" int egtb_book_load_all(egtb_book *b, int32_t *layers_loaded) {
    return guarded([&] {
        if (!b) throw Error(EGTB_ERR_ARG, "NULL book");
        std::lock_guard<std::mutex> lk(b->mu);
        EGTB_CUDA(cudaSetDevice(b->device));
        // scan layer files until a long run of missing indices
        int loaded = 0, misses = 0;
        for (long long nums = 0; misses < 64; ++nums) {
            load_layer(*b, nums);
            if (b->layers[nums].state == 1) {
                ++loaded;
                misses = 0;
            } else {
                ++misses;
            }
        }
        upload_desc(*b);
        if (layers_loaded) *layers_loaded = loaded;
    });
}

extern "C" int egtb_book_lookup(egtb_book *b, const uint64_t *positions, size_t n, int32_t last_op, double *values4,
                                uint8_t *valid_mask, int8_t *op_used) {
    return guarded([&] {
        if (!b) throw Error(EGTB_ERR_ARG, "NULL book");
        if (n && (!positions || !values4 || !valid_mask)) throw Error(EGTB_ERR_ARG, "NULL buffer");
        if (last_op < 0 || last_op > 15) throw Error(EGTB_ERR_ARG, "last_op out of range");
        std::lock_guard<std::mutex> lk(b->mu);
        EGTB_CUDA(cudaSetDevice(b->device));
        // make sure every layer these positions read is loaded (or known missing);
        // a missing file is looked for again on every call, as the reference does
        std::vector<char> seen;
        for (size_t i = 0; i < n; ++i) {
            const long long nums = (host_tile_sum(positions[i]) + b->nums_adjust) / 2;
            if (nums < 0) continue;
            if ((long long)seen.size() <= nums) seen.resize(nums + 1, 0);
            if (seen[nums]) continue;
            seen[nums] = 1;
            if ((long long)b->layers.size() > nums && b->layers[nums].state == 2) {
                b->layers[nums].state = 0;
                b->desc_dirty = true;
            }
            load_layer(*b, nums);
        }
        upload_desc(*b);
        if (n == 0) return;
        if (n > b->scratch_cap) {
            if (b->d_pos) cudaFree(b->d_pos);
            if (b->d_val) cudaFree(b->d_val);
            if (b->d_valid) cudaFree(b->d_valid);
            if (b->d_op) cudaFree(b->d_op);
            b->scratch_cap = std::max<size_t>(n, 4096);
            EGTB_CUDA(cudaMalloc(&b->d_pos, b->scratch_cap * 8));
            EGTB_CUDA(cudaMalloc(&b->d_val, b->scratch_cap * 32));
            EGTB_CUDA(cudaMalloc(&b->d_valid, b->scratch_cap));
            EGTB_CUDA(cudaMalloc(&b->d_op, b->scratch_cap));
        }
        EGTB_CUDA(cudaMemcpyAsync(b->d_pos, positions, n * 8, cudaMemcpyHostToDevice, b->stream));
        launch_lookup<double>(*b, b->d_pos, n, last_op, b->d_val, b->d_valid, b->d_op, b->stream);
        EGTB_CUDA(cudaMemcpyAsync(values4, b->d_val, n * 32, cudaMemcpyDeviceToHost, b->stream));
        EGTB_CUDA(cudaMemcpyAsync(valid_mask, b->d_valid, n, cudaMemcpyDeviceToHost, b->stream));
        if (op_used) EGTB_CUDA(cudaMemcpyAsync(op_used, b->d_op, n, cudaMemcpyDeviceToHost, b->stream));
        EGTB_CUDA(cudaStreamSynchronize(b->stream));
    });
}

extern "C" int egtb_book_lookup_device(egtb_book *b, const uint64_t *d_positions, size_t n, int32_t last_op,
                                       float *d_values4, uint8_t *d_valid_mask, void *stream) {
    return guarded([&] {
        if (!b) throw Error(EGTB_ERR_ARG, "NULL book");
        if (last_op < 0 || last_op > 15) throw Error(EGTB_ERR_ARG, "last_op out of range");
        if (b->desc_dirty) {
            std::lock_guard<std::mutex> lk(b->mu);
            upload_desc(*b);
        }
        if (!b->d_desc && n) throw Error(EGTB_ERR_ARG, "no layers loaded (egtb_book_load_all)");
        launch_lookup<float>(*b, d_positions, n, last_op, d_values4, d_valid_mask, nullptr, (cudaStream_t)stream);
    });
}

namespace egtb {
int book_device(const egtb_book *b) { return b->device; }

// Enqueue move_on_dic (last_op 0) for n_req requests of this book listed at
// d_reqs (n_req + 1 entries) covering `total` positions.
void book_lookup_requests(egtb_book *b, const ServeReq *d_reqs, int n_req, unsigned long long total,
                          cudaStream_t s) {
    if (b->desc_dirty) {
        std::lock_guard<std::mutex> lk(b->mu);
        upload_desc(*b);
    }
    if (!b->d_desc) throw Error(EGTB_ERR_ARG, "no layers loaded (egtb_book_load_all)");
    if (total == 0) return;
    const uint32_t *tab = device_row_table(b->variant);
    const int op_mode = b->variant ? 8 : 0;  // variant: the board as given only
    const int grid = (int)std::min<unsigned long long>((total + 255) / 256, 148 * 8);
    const double scale = scale_for(b->dtype);
    const int r9 = round9_for(b->dtype) ? 1 : 0;
    const int nd = (int)b->layers.size();
    auto run = [&](auto variant_modes, auto trie) {
        constexpr bool W = decltype(variant_modes)::value;
        constexpr bool Z = decltype(trie)::value;
        switch (b->dtype) {
            case EGTB_DTYPE_UINT32:
                lookup_requests_kernel<uint32_t, W, Z><<<grid, 256, 0, s>>>(b->d_desc, nd, d_reqs, n_req, b->nums_adjust, b->spec,
                                                                     tab, op_mode, scale, r9, 0u);
                break;
            case EGTB_DTYPE_UINT64:
                lookup_requests_kernel<uint64_t, W, Z><<<grid, 256, 0, s>>>(b->d_desc, nd, d_reqs, n_req, b->nums_adjust, b->spec,
                                                                     tab, op_mode, scale, r9, 0ull);
                break;
            case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32:
                lookup_requests_kernel<float, W, Z><<<grid, 256, 0, s>>>(b->d_desc, nd, d_reqs, n_req, b->nums_adjust, b->spec,
                                                                  tab, op_mode, scale, r9, (float)dtype_zero(b->dtype));
                break;
            default:
                lookup_requests_kernel<double, W, Z><<<grid, 256, 0, s>>>(b->d_desc, nd, d_reqs, n_req, b->nums_adjust, b->spec,
                                                                   tab, op_mode, scale, r9, dtype_zero(b->dtype));
                break;
        }
    };
    const bool trie = b->any_compressed;
    if (b->spec.symm >= 4) {
        if (trie) run(std::true_type{}, std::true_type{});
        else run(std::true_type{}, std::false_type{});
    } else {
        if (trie) run(std::false_type{}, std::true_type{});
        else run(std::false_type{}, std::false_type{});
    }
    EGTB_CUDA(cudaGetLastError());
}
}  // namespace egtb

extern "C" int egtb_find_classic_value(const char *pathname, const char *filename, uint64_t key, int32_t dtype,
                                       int32_t device, double *value, int32_t *found) {
    return guarded([&] {
        if (!pathname || !filename || !value || !found) throw Error(EGTB_ERR_ARG, "NULL argument");
        dtype_size(dtype);
        std::string path = std::string(pathname);
        if (!path.empty() && path.back() != '/') path += "/";
        path += filename;
        *value = 0.0;
        *found = 0;
        if (!file_exists(path)) return;  // the file could not be opened: not found
        int n = 0;
        EGTB_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw Error(EGTB_ERR_ARG, "device not present");
        EGTB_CUDA(cudaSetDevice(device));
        std::lock_guard<std::mutex> lk(g_fb_mu);
        FileBook *fb = nullptr;
        const uint64_t sz = file_size(path);
        for (auto &e : g_fb)
            if (e->path == path && e->size == sz && e->dtype == dtype) fb = e.get();
        if (!fb) {
            if (g_fb.size() >= 8) {
                auto &old = g_fb.front();
                cudaFree(old->layer.keys);
                cudaFree(old->layer.rates);
                cudaFree(old->layer.split);
                g_fb.erase(g_fb.begin());
            }
            auto e = std::make_unique<FileBook>();
            e->path = path;
            e->size = sz;
            e->dtype = dtype;
            cudaStream_t st = nullptr;
            EGTB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> st_guard(st, [](cudaStream_t q) { cudaStreamDestroy(q); });
            const size_t rec = record_size(dtype);
            std::vector<unsigned char> host = read_file(path);
            BookLayer &L = e->layer;
            L.n = host.size() / rec;
            const size_t es = dtype_size(dtype);
            EGTB_CUDA(cudaMalloc(&L.keys, std::max<size_t>(L.n, 1) * 8));
            EGTB_CUDA(cudaMalloc(&L.rates, std::max<size_t>(L.n, 1) * es));
            EGTB_CUDA(cudaMalloc(&L.split, (L.n / kSplitStride + 1) * 8));
            if (L.n) {
                unsigned char *d = nullptr;
                int *flag = nullptr;
                EGTB_CUDA(cudaMalloc(&d, L.n * rec));
                EGTB_CUDA(cudaMalloc(&flag, sizeof(int)));
                EGTB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
                EGTB_CUDA(cudaMemcpyAsync(d, host.data(), L.n * rec, cudaMemcpyHostToDevice, st));
                if (dtype == EGTB_DTYPE_UINT32)
                    split_records_kernel<uint32_t><<<592, 256, 0, st>>>(d, L.n, L.keys, (uint32_t *)L.rates, L.split, flag);
                else if (dtype == EGTB_DTYPE_UINT64)
                    split_records_kernel<uint64_t><<<592, 256, 0, st>>>(d, L.n, L.keys, (uint64_t *)L.rates, L.split, flag);
                else if (es == 4)
                    split_records_kernel<float><<<592, 256, 0, st>>>(d, L.n, L.keys, (float *)L.rates, L.split, flag);
                else
                    split_records_kernel<double><<<592, 256, 0, st>>>(d, L.n, L.keys, (double *)L.rates, L.split, flag);
                int unsorted = 0;
                EGTB_CUDA(cudaMemcpyAsync(&unsorted, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
                EGTB_CUDA(cudaStreamSynchronize(st));
                cudaFree(d);
                cudaFree(flag);
                L.sorted = unsorted ? 0 : 1;
            }
            L.state = 1;
            g_fb.push_back(std::move(e));
            fb = g_fb.back().get();
        }
        double *d_out = nullptr;
        EGTB_CUDA(cudaMalloc(&d_out, sizeof(double)));
        const BookLayer &L = fb->layer;
        const double scale = scale_for(dtype);
        switch (dtype) {
            case EGTB_DTYPE_UINT32:
                find_one_kernel<uint32_t><<<1, 1>>>(L.keys, (const uint32_t *)L.rates, L.n, L.sorted, key, scale, 0u, d_out);
                break;
            case EGTB_DTYPE_UINT64:
                find_one_kernel<uint64_t><<<1, 1>>>(L.keys, (const uint64_t *)L.rates, L.n, L.sorted, key, scale, 0ull, d_out);
                break;
            case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32:
                find_one_kernel<float><<<1, 1>>>(L.keys, (const float *)L.rates, L.n, L.sorted, key, scale,
                                                 (float)dtype_zero(dtype), d_out);
                break;
            default:
                find_one_kernel<double><<<1, 1>>>(L.keys, (const double *)L.rates, L.n, L.sorted, key, scale,
                                                  dtype_zero(dtype), d_out);
                break;
        }
        EGTB_CUDA(cudaGetLastError());
        EGTB_CUDA(cudaMemcpy(value, d_out, sizeof(double), cudaMemcpyDeviceToHost));
        cudaFree(d_out);
        *found = 1;
    });
}
