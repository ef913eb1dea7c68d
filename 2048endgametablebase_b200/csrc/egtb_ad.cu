// Masked-board primitives of the reference's advanced algorithm (namespace
// FormationAD): the masked mover, the board masker, the tile statistics and
// the validity test of a masked board. In a masked board every tile of 64 and
// up is held as a 0xF ("32k") nibble; 0xF never merges, and a merge that
// makes a tile of 64 or more yields 0xF and raises mask_new_tile.
//
//   row rule and mover      native_core/src/BoardMoverAD.cpp:27-89,171-178
//   mask_board              native_core/src/BoardMaskerAD.cpp:112-121
//   tile statistics         native_core/src/BoardMaskerAD.cpp:24-50 (per-row
//                           info), :123-144, :169-190, :219-257
//   tiles combinations      native_core/src/BoardMaskerAD.cpp:259-289,524-531
//   validate                native_core/src/BoardMaskerAD.cpp:409-443
//   permutations, unmask    native_core/src/BoardMaskerAD.cpp:291-358,445-512
//
// One thread per board; the row moves come from a 65536-entry table built on
// the host from the rule, the per-row statistics are computed in registers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "egtb_host.h"

namespace egtb {
namespace {

constexpr int kAdCombos = 2560;  // tiles-combination entries: a + 256 b, b < 10
constexpr int kAdComboVals = 16;

// One row moved toward column 0 (reverse = false) or column 3 under the
// masked rule: slide the tiles, merge each adjacent equal pair once, first
// pair first; 0xF slides but never merges; a merged tile of 64 or more
// (nibble 6 and up) is written as 0xF and sets *made_32k.
uint32_t ad_row_after_move(uint32_t row, bool reverse, bool *made_32k) {
    int cell[4];
    for (int i = 0; i < 4; ++i) cell[i] = (row >> (12 - 4 * i)) & 0xF;  // column 0 first
    if (reverse) {
        std::swap(cell[0], cell[3]);
        std::swap(cell[1], cell[2]);
    }
    int out[4] = {0, 0, 0, 0};
    int m = 0, pending = 0;
    for (int i = 0; i < 4; ++i) {
        if (!cell[i]) continue;
        if (pending && pending == cell[i] && pending != 0xF) {
            int v = pending + 1;
            if (v >= 6) {
                v = 0xF;
                *made_32k = true;
            }
            out[m++] = v;
            pending = 0;
        } else {
            if (pending) out[m++] = pending;
            pending = cell[i];
        }
    }
    if (pending) out[m++] = pending;
    if (reverse) {
        std::swap(out[0], out[3]);
        std::swap(out[1], out[2]);
    }
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) r |= (uint32_t)out[i] << (12 - 4 * i);
    return r;
}

struct AdTables {
    std::vector<uint32_t> moves;  // left xor | right xor << 16
    std::vector<uint8_t> flags;   // the left merge made a 32k tile
    std::vector<uint8_t> lens;    // tiles combinations: entry length
    std::vector<uint8_t> vals;    // ... and values (log2 of the large tiles, ascending)
};

// The large tiles a masked board's 32k cells may hold: `count` tiles of 64
// and up summing to `sum`, taken largest first with the reference's early
// exits; empty when none fits.
std::vector<uint8_t> large_tiles_for(uint64_t sum, int count) {
    std::vector<uint8_t> out;
    for (int lg = 13; lg >= 6; --lg) {
        const uint64_t tile = 1ull << lg;
        if (tile > sum) continue;
        if (tile == sum) {
            if (count == 1) {
                out.push_back((uint8_t)lg);
                return out;
            }
            continue;
        }
        if (2 * tile == sum && count == 2) {
            out.push_back((uint8_t)lg);
            out.push_back((uint8_t)lg);
            return out;
        }
        if (tile != 64 && sum == 192 && count == 3) {
            out.push_back(6);
            out.push_back(6);
            out.push_back(6);
            return out;
        }
        sum -= tile;
        --count;
        out.push_back((uint8_t)lg);
    }
    return {};
}

// The rows of permutation slot (m, n): every way to put the values 0..n-1
// into n distinct cells of m (row[j] = the cell that gets value j), in the
// reference's order: by the cells' contents read from cell 0 to cell m-1, a
// cell left out reading as 15 (resort_permutations, BoardMaskerAD.cpp:291-332).
std::vector<uint8_t> permutation_rows(int m, int n) {
    std::vector<std::pair<uint64_t, std::vector<uint8_t>>> rows;
    std::vector<uint8_t> row((size_t)n);
    std::vector<bool> used((size_t)m, false);
    auto fill = [&](auto &&self, int j) -> void {
        if (j == n) {
            uint64_t key = 0;
            for (int c = 0; c < m; ++c) {
                uint64_t nib = 15;
                for (int v = 0; v < n; ++v)
                    if (row[(size_t)v] == c) nib = (uint64_t)v;
                key = (key << 4) | nib;
            }
            rows.emplace_back(key, row);
            return;
        }
        for (int c = 0; c < m; ++c) {
            if (used[(size_t)c]) continue;
            used[(size_t)c] = true;
            row[(size_t)j] = (uint8_t)c;
            self(self, j + 1);
            used[(size_t)c] = false;
        }
    };
    fill(fill, 0);
    std::sort(rows.begin(), rows.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    std::vector<uint8_t> flat;
    flat.reserve(rows.size() * (size_t)n);
    for (const auto &r : rows) flat.insert(flat.end(), r.second.begin(), r.second.end());
    return flat;
}

const AdTables &host_ad_tables() {
    static const AdTables t = [] {
        AdTables a;
        a.moves.resize(65536);
        a.flags.resize(65536);
        for (uint32_t r = 0; r < 65536; ++r) {
            bool made = false, ignored = false;
            const uint32_t l = ad_row_after_move(r, false, &made) ^ r;
            const uint32_t rr = ad_row_after_move(r, true, &ignored) ^ r;
            a.moves[r] = l | (rr << 16);
            a.flags[r] = made ? 1 : 0;
        }
        a.lens.assign(kAdCombos, 0);
        a.vals.assign((size_t)kAdCombos * kAdComboVals, 0);
        for (int s = 1; s < 256; ++s)
            for (int c = 1; c < 10; ++c) {
                std::vector<uint8_t> v = large_tiles_for((uint64_t)s << 6, c);
                std::reverse(v.begin(), v.end());
                const int e = s + 256 * c;
                a.lens[e] = (uint8_t)v.size();
                std::copy(v.begin(), v.end(), a.vals.begin() + (size_t)e * kAdComboVals);
            }
        return a;
    }();
    return t;
}

struct AdDeviceTables {
    uint32_t *moves = nullptr;
    uint8_t *flags = nullptr, *lens = nullptr, *vals = nullptr;
};

// The tables in device memory, uploaded once per device (kept until exit).
AdDeviceTables device_ad_tables(int device) {
    static std::mutex mu;
    static std::vector<AdDeviceTables> per_device;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)per_device.size() <= device) per_device.resize(device + 1);
    AdDeviceTables &d = per_device[device];
    if (!d.moves) {
        const AdTables &h = host_ad_tables();
        AdDeviceTables n;
        EGTB_CUDA(cudaMalloc(&n.moves, h.moves.size() * sizeof(uint32_t)));
        EGTB_CUDA(cudaMalloc(&n.flags, h.flags.size()));
        EGTB_CUDA(cudaMalloc(&n.lens, h.lens.size()));
        EGTB_CUDA(cudaMalloc(&n.vals, h.vals.size()));
        EGTB_CUDA(cudaMemcpy(n.moves, h.moves.data(), h.moves.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        EGTB_CUDA(cudaMemcpy(n.flags, h.flags.data(), h.flags.size(), cudaMemcpyHostToDevice));
        EGTB_CUDA(cudaMemcpy(n.lens, h.lens.data(), h.lens.size(), cudaMemcpyHostToDevice));
        EGTB_CUDA(cudaMemcpy(n.vals, h.vals.data(), h.vals.size(), cudaMemcpyHostToDevice));
        // a copy from pageable memory may still be landing when cudaMemcpy
        // returns, and the kernels run on another stream: wait once for it
        EGTB_CUDA(cudaDeviceSynchronize());
        d = n;
    }
    return d;
}

// ------------------------------------------------------------ device ----

struct AdParamDev {
    uint64_t fixed;
    uint32_t small_limit, target, num_free, num_fixed;
};

__device__ __forceinline__ uint64_t ad_moved_rows(const uint32_t *tab, uint64_t b, int half) {
    uint64_t x = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) x |= (uint64_t)((__ldg(tab + ((b >> (16 * k)) & 0xFFFFu)) >> (16 * half)) & 0xFFFFu)
                                    << (16 * k);
    return b ^ x;
}

__device__ __forceinline__ uint8_t ad_any_flag(const uint8_t *flags, uint64_t b) {
    uint8_t f = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) f |= __ldg(flags + ((b >> (16 * k)) & 0xFFFFu));
    return f;
}

__global__ void ad_moves_kernel(const uint32_t *tab, const uint8_t *flags, const uint64_t *in, size_t n,
                                uint64_t *out4, uint8_t *f4) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t b = in[i], t = transpose(b);
        const uint8_t fh = ad_any_flag(flags, b), fv = ad_any_flag(flags, t);
        out4[4 * i + 0] = ad_moved_rows(tab, b, 0);
        out4[4 * i + 1] = ad_moved_rows(tab, b, 1);
        out4[4 * i + 2] = transpose(ad_moved_rows(tab, t, 0));
        out4[4 * i + 3] = transpose(ad_moved_rows(tab, t, 1));
        f4[4 * i + 0] = fh;
        f4[4 * i + 1] = fh;
        f4[4 * i + 2] = fv;
        f4[4 * i + 3] = fv;
    }
}

__global__ void ad_mask_kernel(const uint64_t *in, size_t n, long long threshold, uint64_t *out) {
    const uint64_t th = (uint64_t)threshold;  // compared as the reference compares: unsigned 64-bit
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t b = in[i], m = b;
        for (int k = 0; k < 16; ++k)
            if (((b >> (4 * k)) & 0xFull) >= th) m |= 0xFull << (4 * k);
        out[i] = m;
    }
}

// Statistics of one 16-bit row, nibbles from the highest: a 32k cell is 0xF
// (masked_only) or any tile of 64 and up; the other tiles add to a 16-bit sum
// (it wraps as the reference's uint16_t field does); a 0xF cell met before
// any non-0xF 32k cell of the row counts toward pos_rank.
struct AdRowInfo {
    uint32_t sum16, count, pos, merged_count, merged_xor, rank;
};

__device__ __forceinline__ AdRowInfo ad_row_info(uint32_t row, bool masked_only) {
    AdRowInfo r{0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 3; i >= 0; --i) {
        const uint32_t v = (row >> (4 * i)) & 0xFu;
        const bool large = masked_only ? v == 0xFu : v > 5u;
        if (large) {
            r.pos |= 0xFu << (4 * i);
            ++r.count;
            if (v == 0xFu) {
                if (r.merged_count == 0) ++r.rank;
            } else {
                ++r.merged_count;
                r.merged_xor ^= v;
            }
        } else if (v > 0u) {
            r.sum16 += 1u << v;
        }
    }
    r.sum16 &= 0xFFFFu;
    return r;
}

__device__ __forceinline__ egtb_ad_tile_count ad_stats(uint64_t board, const AdParamDev &p, int kind) {
    board &= ~p.fixed;
    AdRowInfo r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = ad_row_info((uint32_t)((board >> (16 * k)) & 0xFFFFu), kind == 1);
    egtb_ad_tile_count s = {};
    s.total_sum = r[0].sum16 + r[1].sum16 + r[2].sum16 + r[3].sum16;
    s.count_32k = (int32_t)(r[0].count + r[1].count + r[2].count + r[3].count);
    s.pos_bitmap = (uint64_t)r[0].pos | ((uint64_t)r[1].pos << 16) | ((uint64_t)r[2].pos << 32) |
                   ((uint64_t)r[3].pos << 48);
    if (kind == 4) {
        s.merged_tile_found = r[0].merged_count + r[1].merged_count + r[2].merged_count + r[3].merged_count;
        s.merged_tile = r[0].merged_xor ^ r[1].merged_xor ^ r[2].merged_xor ^ r[3].merged_xor;
        // 0xF cells from the top row down to the row of the first merged tile
        const uint32_t s3 = r[3].rank, s2 = s3 + r[2].rank, s1 = s2 + r[1].rank, s0 = s1 + r[0].rank;
        s.pos_rank = r[3].merged_count ? s3 : r[2].merged_count ? s2 : r[1].merged_count ? s1 : s0;
        s.is_success = (s.merged_tile == (p.target & 0xFFu) && s.merged_tile_found == 1) ? 1u : 0u;
    }
    return s;
}

__global__ void ad_stats_kernel(const uint64_t *in, size_t n, AdParamDev p, int kind, egtb_ad_tile_count *out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = ad_stats(in[i], p, kind);
}

__global__ void ad_validate_kernel(const uint64_t *in, const uint32_t *orig, size_t n, AdParamDev p,
                                   const uint8_t *lens, const uint8_t *vals, uint8_t *out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const egtb_ad_tile_count s = ad_stats(in[i], p, 2);
        const int8_t count = (int8_t)s.count_32k, free32k = (int8_t)(uint8_t)p.num_free;
        uint8_t ok;
        if (s.total_sum >= p.small_limit + 64u) {
            ok = 0;
        } else if (count == free32k) {
            ok = 1;
        } else {
            const uint32_t large = orig[i] - s.total_sum - ((uint32_t)((p.num_free & 0xFFu) + (p.num_fixed & 0xFFu)) << 15);
            const uint32_t a = (uint8_t)(large >> 6), c = (uint8_t)(count - free32k);
            const int len = c < 10 ? lens[a + 256 * c] : 0;
            const uint8_t *v = vals + (size_t)(a + 256 * c) * kAdComboVals;
            if (len == 0 || v[len - 1] == (uint8_t)p.target) {
                ok = 0;
            } else if (count < 2) {
                ok = 1;
            } else if (len > 2 && v[0] == v[2]) {
                ok = s.total_sum >= p.small_limit - 64u ? 0 : 1;
            } else if (len > 1 && v[0] == v[1]) {
                ok = s.total_sum >= p.small_limit ? 0 : 1;
            } else {
                ok = 1;
            }
        }
        out[i] = ok;
    }
}

// Permutation slot (m, n) = index (m << 4) + n: its rows in one buffer.
struct AdPermSlot {
    unsigned long long off;
    unsigned rows, cols;
};

// What unmask_board does with one board: 0 = nothing, 1 = the board itself,
// 2 = one board per permutation row of slot `slot` (values from combination
// entry `combo`); pos[] = the 0xF cells (fixed ones excluded), highest first.
__device__ __forceinline__ int ad_unmask_plan(uint64_t board, uint32_t orig, const AdParamDev &p, const uint8_t *lens,
                                              int &slot, int &combo, int &npos, uint8_t pos[16]) {
    const uint64_t masked = board & ~p.fixed;
    uint32_t total = 0;
    npos = 0;
#pragma unroll
    for (int k = 3; k >= 0; --k) total += ad_row_info((uint32_t)((masked >> (16 * k)) & 0xFFFFu), true).sum16;
    for (int sh = 60; sh >= 0; sh -= 4)
        if (((masked >> sh) & 0xFull) == 0xFull) pos[npos++] = (uint8_t)sh;
    const int8_t count = (int8_t)npos, free32k = (int8_t)(uint8_t)p.num_free;
    if (count == 0 || count == free32k) return 1;
    const uint32_t large = orig - total - ((uint32_t)((p.num_free & 0xFFu) + (p.num_fixed & 0xFFu)) << 15);
    const uint32_t a = (uint8_t)(large >> 6), c = (uint8_t)(count - free32k);
    if (c >= 10) return 0;  // past the reference's table (its read is out of bounds)
    combo = (int)(a + 256 * c);
    if (lens[combo] == 0) return 0;
    // init_masker builds slots (n + num_free_32k, n) for 1 <= n < target - 4
    if ((int)c < 1 || (int)c >= (int)(p.target & 0xFFu) - 4 || npos > 15) return 0;
    slot = (npos << 4) + (int)c;
    return 2;
}

__global__ void ad_unmask_count_kernel(const uint64_t *in, const uint32_t *orig, size_t n, AdParamDev p,
                                       const uint8_t *lens, const uint8_t *vals, const AdPermSlot *slots,
                                       const uint8_t *rows, uint32_t *counts) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int slot = 0, combo = 0, npos = 0;
        uint8_t pos[16];
        const int plan = ad_unmask_plan(in[i], orig[i], p, lens, slot, combo, npos, pos);
        uint32_t cnt = plan == 1 ? 1u : 0u;
        if (plan == 2) {
            const AdPermSlot s = slots[slot];
            const uint8_t *v = vals + (size_t)combo * kAdComboVals;
            if (lens[combo] > 1 && v[0] == v[1]) {
                // equal first two tiles: only rows with row[1] < row[0]
                for (unsigned r = 0; r < s.rows; ++r) {
                    const uint8_t *row = rows + s.off + (size_t)r * s.cols;
                    cnt += row[1] < row[0];
                }
            } else {
                cnt = s.rows;
            }
        }
        counts[i] = cnt;
    }
}

__global__ void ad_unmask_write_kernel(const uint64_t *in, const uint32_t *orig, size_t n, AdParamDev p,
                                       const uint8_t *lens, const uint8_t *vals, const AdPermSlot *slots,
                                       const uint8_t *rows, const unsigned long long *offs, uint64_t *out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t board = in[i];
        int slot = 0, combo = 0, npos = 0;
        uint8_t pos[16];
        const int plan = ad_unmask_plan(board, orig[i], p, lens, slot, combo, npos, pos);
        unsigned long long o = offs[i];
        if (plan == 1) out[o] = board;
        if (plan != 2) continue;
        const AdPermSlot s = slots[slot];
        const int len = lens[combo];
        const uint8_t *v = vals + (size_t)combo * kAdComboVals;
        const bool ordered = len > 1 && v[0] == v[1];
        for (unsigned r = 0; r < s.rows; ++r) {
            const uint8_t *row = rows + s.off + (size_t)r * s.cols;
            if (ordered && !(row[1] < row[0])) continue;
            uint64_t clear = 0, set = 0;
            for (int j = 0; j < len; ++j) {
                const int sh = pos[row[j]];
                clear |= 0xFull << sh;
                set |= (uint64_t)v[j] << sh;
            }
            out[o++] = (board & ~clear) | set;
        }
    }
}

// -------------------------------------------------------------- host ----

AdParamDev ad_param(const egtb_ad_param *p) {
    if (!p) throw Error(EGTB_ERR_ARG, "NULL parameter block");
    return AdParamDev{p->pos_fixed_32k_mask, p->small_tile_sum_limit, p->target, p->num_free_32k, p->num_fixed_32k};
}

// The stream the primitives of one device run on, created once per device:
// non-blocking, so a call waits on no other work of the device (a build or a
// serving loop on the library's own streams) and nothing waits on it.
cudaStream_t ad_stream(int device) {
    static std::mutex mu;
    static std::vector<cudaStream_t> per_device;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)per_device.size() <= device) per_device.resize(device + 1, nullptr);
    if (!per_device[device]) EGTB_CUDA(cudaStreamCreateWithFlags(&per_device[device], cudaStreamNonBlocking));
    return per_device[device];
}

// Device buffers of one call, allocated and freed in the order of the call's
// stream (no device-wide synchronisation), freed on every exit.
struct AdBuffers {
    cudaStream_t s;
    std::vector<void *> ptrs;
    explicit AdBuffers(cudaStream_t st) : s(st) {}
    void *get(size_t bytes) {
        void *p = nullptr;
        EGTB_CUDA(cudaMallocAsync(&p, std::max<size_t>(bytes, 16), s));
        ptrs.push_back(p);
        return p;
    }
    ~AdBuffers() {
        for (void *p : ptrs) cudaFreeAsync(p, s);
    }
};

// Run f(stream, grid) for one call on `device` (grid: four 256-thread blocks
// per SM for the grid-stride kernels); returns once the call's work and
// copies are done.
template <typename F>
void on_device(int device, F &&f) {
    int count = 0;
    EGTB_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw Error(EGTB_ERR_ARG, "device out of range");
    EGTB_CUDA(cudaSetDevice(device));
    int sms = 0;
    EGTB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const cudaStream_t s = ad_stream(device);
    f(s, 4 * std::max(1, sms));
    EGTB_CUDA(cudaGetLastError());
    EGTB_CUDA(cudaStreamSynchronize(s));
}

constexpr int kAdBlock = 256;

}  // namespace
}  // namespace egtb

using namespace egtb;

extern "C" int egtb_ad_move_all_dir(int device, const uint64_t *boards, size_t n, uint64_t *out4, uint8_t *flags4) {
    return guarded([&] {
        if (n == 0) return;
        if (!boards || !out4 || !flags4) throw Error(EGTB_ERR_ARG, "NULL buffer");
        on_device(device, [&](cudaStream_t s, int grid) {
            const AdDeviceTables t = device_ad_tables(device);
            AdBuffers buf(s);
            auto *din = (uint64_t *)buf.get(n * 8);
            auto *dout = (uint64_t *)buf.get(n * 32);
            auto *dfl = (uint8_t *)buf.get(n * 4);
            EGTB_CUDA(cudaMemcpyAsync(din, boards, n * 8, cudaMemcpyHostToDevice, s));
            ad_moves_kernel<<<grid, kAdBlock, 0, s>>>(t.moves, t.flags, din, n, dout, dfl);
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaMemcpyAsync(out4, dout, n * 32, cudaMemcpyDeviceToHost, s));
            EGTB_CUDA(cudaMemcpyAsync(flags4, dfl, n * 4, cudaMemcpyDeviceToHost, s));
        });
    });
}

extern "C" int egtb_ad_mask_board(int device, const uint64_t *boards, size_t n, int32_t threshold, uint64_t *out) {
    return guarded([&] {
        if (n == 0) return;
        if (!boards || !out) throw Error(EGTB_ERR_ARG, "NULL buffer");
        on_device(device, [&](cudaStream_t s, int grid) {
            AdBuffers buf(s);
            auto *din = (uint64_t *)buf.get(n * 8);
            auto *dout = (uint64_t *)buf.get(n * 8);
            EGTB_CUDA(cudaMemcpyAsync(din, boards, n * 8, cudaMemcpyHostToDevice, s));
            ad_mask_kernel<<<grid, kAdBlock, 0, s>>>(din, n, (long long)threshold, dout);
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaMemcpyAsync(out, dout, n * 8, cudaMemcpyDeviceToHost, s));
        });
    });
}

extern "C" int egtb_ad_tile_stats(int device, const uint64_t *boards, size_t n, const egtb_ad_param *param,
                                  int32_t kind, egtb_ad_tile_count *out) {
    return guarded([&] {
        if (kind != 1 && kind != 2 && kind != 4) throw Error(EGTB_ERR_ARG, "kind must be 1, 2 or 4");
        const AdParamDev p = ad_param(param);
        if (n == 0) return;
        if (!boards || !out) throw Error(EGTB_ERR_ARG, "NULL buffer");
        on_device(device, [&](cudaStream_t s, int grid) {
            AdBuffers buf(s);
            auto *din = (uint64_t *)buf.get(n * 8);
            auto *dout = (egtb_ad_tile_count *)buf.get(n * sizeof(egtb_ad_tile_count));
            EGTB_CUDA(cudaMemcpyAsync(din, boards, n * 8, cudaMemcpyHostToDevice, s));
            ad_stats_kernel<<<grid, kAdBlock, 0, s>>>(din, n, p, kind, dout);
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaMemcpyAsync(out, dout, n * sizeof(egtb_ad_tile_count), cudaMemcpyDeviceToHost, s));
        });
    });
}

extern "C" int egtb_ad_validate(int device, const uint64_t *boards, size_t n, const uint32_t *original_sums,
                                const egtb_ad_param *param, uint8_t *out) {
    return guarded([&] {
        const AdParamDev p = ad_param(param);
        if (n == 0) return;
        if (!boards || !original_sums || !out) throw Error(EGTB_ERR_ARG, "NULL buffer");
        on_device(device, [&](cudaStream_t s, int grid) {
            const AdDeviceTables t = device_ad_tables(device);
            AdBuffers buf(s);
            auto *din = (uint64_t *)buf.get(n * 8);
            auto *dsum = (uint32_t *)buf.get(n * 4);
            auto *dout = (uint8_t *)buf.get(n);
            EGTB_CUDA(cudaMemcpyAsync(din, boards, n * 8, cudaMemcpyHostToDevice, s));
            EGTB_CUDA(cudaMemcpyAsync(dsum, original_sums, n * 4, cudaMemcpyHostToDevice, s));
            ad_validate_kernel<<<grid, kAdBlock, 0, s>>>(din, dsum, n, p, t.lens, t.vals, dout);
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaMemcpyAsync(out, dout, n, cudaMemcpyDeviceToHost, s));
        });
    });
}

extern "C" int egtb_ad_row_tables(uint32_t *moves, uint8_t *flags) {
    return guarded([&] {
        if (!moves || !flags) throw Error(EGTB_ERR_ARG, "NULL buffer");
        const AdTables &t = host_ad_tables();
        std::memcpy(moves, t.moves.data(), t.moves.size() * sizeof(uint32_t));
        std::memcpy(flags, t.flags.data(), t.flags.size());
    });
}

extern "C" int egtb_ad_tiles_combinations(uint8_t *lens, uint8_t *vals16) {
    return guarded([&] {
        if (!lens || !vals16) throw Error(EGTB_ERR_ARG, "NULL buffer");
        const AdTables &t = host_ad_tables();
        std::memcpy(lens, t.lens.data(), t.lens.size());
        std::memcpy(vals16, t.vals.data(), t.vals.size());
    });
}

extern "C" int egtb_ad_unmask(int device, const uint64_t *boards, size_t n, const uint32_t *original_sums,
                              const egtb_ad_param *param, uint32_t *counts, uint64_t *out, size_t cap,
                              uint64_t *total) {
    return guarded([&] {
        const AdParamDev p = ad_param(param);
        if (!total) throw Error(EGTB_ERR_ARG, "NULL total");
        *total = 0;
        if (n == 0) return;
        if (!boards || !original_sums || !counts || (cap && !out)) throw Error(EGTB_ERR_ARG, "NULL buffer");
        // the permutation slots init_masker builds: (n + num_free_32k, n), 1 <= n < target - 4
        std::vector<AdPermSlot> slots(256, AdPermSlot{0, 0, 0});
        std::vector<uint8_t> rows;
        for (int k = 1; k < (int)(p.target & 0xFFu) - 4; ++k) {
            const int m = k + (int)(p.num_free & 0xFFu);
            if (m > 15) break;
            double perms = 1.0;
            for (int j = 0; j < k; ++j) perms *= (double)(m - j);
            if (perms * k > (double)(1u << 28))
                throw Error(EGTB_ERR_UNSUPPORTED, "permutation table above 256 MiB for this target and num_free_32k");
            const std::vector<uint8_t> r = permutation_rows(m, k);
            slots[(size_t)((m << 4) + k)] = AdPermSlot{(unsigned long long)rows.size(), (unsigned)(r.size() / k),
                                                        (unsigned)k};
            rows.insert(rows.end(), r.begin(), r.end());
        }
        on_device(device, [&](cudaStream_t s, int grid) {
            const AdDeviceTables t = device_ad_tables(device);
            AdBuffers buf(s);
            auto *din = (uint64_t *)buf.get(n * 8);
            auto *dsum = (uint32_t *)buf.get(n * 4);
            auto *dcnt = (uint32_t *)buf.get(n * 4);
            auto *dslots = (AdPermSlot *)buf.get(slots.size() * sizeof(AdPermSlot));
            auto *drows = (uint8_t *)buf.get(rows.size());
            EGTB_CUDA(cudaMemcpyAsync(din, boards, n * 8, cudaMemcpyHostToDevice, s));
            EGTB_CUDA(cudaMemcpyAsync(dsum, original_sums, n * 4, cudaMemcpyHostToDevice, s));
            EGTB_CUDA(cudaMemcpyAsync(dslots, slots.data(), slots.size() * sizeof(AdPermSlot), cudaMemcpyHostToDevice, s));
            if (!rows.empty()) EGTB_CUDA(cudaMemcpyAsync(drows, rows.data(), rows.size(), cudaMemcpyHostToDevice, s));
            ad_unmask_count_kernel<<<grid, kAdBlock, 0, s>>>(din, dsum, n, p, t.lens, t.vals, dslots, drows, dcnt);
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaMemcpyAsync(counts, dcnt, n * 4, cudaMemcpyDeviceToHost, s));
            EGTB_CUDA(cudaStreamSynchronize(s));  // the offsets below read the counts
            std::vector<unsigned long long> offs(n);
            unsigned long long sum = 0;
            for (size_t i = 0; i < n; ++i) {
                offs[i] = sum;
                sum += counts[i];
            }
            *total = sum;
            if (sum > cap) throw Error(EGTB_ERR_CAPACITY, "unmasked boards exceed the output capacity");
            if (sum == 0) return;
            auto *doffs = (unsigned long long *)buf.get(n * 8);
            auto *dout = (uint64_t *)buf.get(sum * 8);
            EGTB_CUDA(cudaMemcpyAsync(doffs, offs.data(), n * 8, cudaMemcpyHostToDevice, s));
            ad_unmask_write_kernel<<<grid, kAdBlock, 0, s>>>(din, dsum, n, p, t.lens, t.vals, dslots, drows, doffs, dout);
            EGTB_CUDA(cudaGetLastError());
            EGTB_CUDA(cudaMemcpyAsync(out, dout, sum * 8, cudaMemcpyDeviceToHost, s));
        });
    });
}
