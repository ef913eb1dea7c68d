// Device-side board primitives for the classic tablebase path (sm_100a).
//
// Board: 4x4 cells in a uint64, one log2 nibble per cell; nibble k is row
// 3-k/4, column 3-k%4, so row 0 is the high 16 bits and column 0 the high
// nibble of a row (native_core/include/BoardCodec.h:20-30). Nibble 0xF is the
// 32768 tile, which never merges (native_core/include/BoardMover.h:31).
#pragma once

#include <cstdint>

namespace egtb {

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while the kernel before it in the stream finishes.
// pdl_trigger lets the next such kernel launch (its blocks take SM resources
// only as this kernel's blocks leave them); pdl_wait blocks until the kernel
// before this one has completed and its memory operations are visible. Both
// are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Default number of polls of a bounded wait on another block (sort look-back).
constexpr unsigned kSpinLimit = 1u << 22;


constexpr int kMaxMasks = 32;

// Pattern parameters handed to every kernel by value.
struct DevSpec {
    uint64_t masks[kMaxMasks];
    int n_masks;
    int symm;              // 0 identity, 1 full, 2 diagonal, 3 horizontal
    uint64_t succ_hi;      // bit 4k+3 set for every success nibble k
    uint64_t target_rep;   // target log2 replicated in every nibble
    int has_success;       // 0: no success shifts -> everything is a success
    int target;
};

// ---------------------------------------------------------------- moves ---

// Row-move XOR deltas: low 16 bits move toward column 0, high 16 bits toward
// column 3. Built on the host by egtb::host_row_tables().
struct RowTables {
    const uint32_t *delta;  // 65536 entries
};

__device__ __forceinline__ uint32_t row_delta(const uint32_t *__restrict__ tab, uint32_t row) {
    return __ldg(tab + row);
}

// 4x4 nibble-matrix transpose: swap the off-diagonal 2x2 blocks (24-bit
// shift), then the off-diagonal cells inside each block (12-bit shift).
__device__ __forceinline__ uint64_t transpose(uint64_t b) {
    uint64_t x =(b & 0xFF00FF0000FF00FFull) | ((b & 0x00FF00FF00000000ull) >> 24) |
                 ((b & 0x00000000FF00FF00ull) << 24);
    return (x & 0xF0F00F0FF0F00F0Full) | ((x & 0x0F0F00000F0F0000ull) >> 12) |
           ((x & 0x0000F0F00000F0F0ull) << 12);
}

// Mirror columns: reverse the four nibbles of every 16-bit row.
__device__ __forceinline__ uint64_t mirror_cols(uint64_t b) {
    b = ((b & 0xFF00FF00FF00FF00ull) >> 8) | ((b & 0x00FF00FF00FF00FFull) << 8);
    return ((b & 0xF0F0F0F0F0F0F0F0ull) >> 4) | ((b & 0x0F0F0F0F0F0F0F0Full) << 4);
}

// Mirror rows: reverse the four 16-bit rows.
__device__ __forceinline__ uint64_t mirror_rows(uint64_t b) {
    b = (b >> 32) | (b << 32);
    return ((b & 0xFFFF0000FFFF0000ull) >> 16) | ((b & 0x0000FFFF0000FFFFull) << 16);
}

__device__ __forceinline__ uint64_t umin(uint64_t a, uint64_t b) { return a < b ? a : b; }

// The eight symmetries, numbered like apply_sym_like
// (native_core/include/SymmetryUtils.h:9-29): 1 mirror columns, 2 mirror rows,
// 3 transpose, 4 anti-transpose, 5 half turn, 6 quarter turn
// counter-clockwise, 7 quarter turn clockwise.
__device__ __forceinline__ uint64_t apply_sym(uint64_t b, int idx) {
    switch (idx) {
        case 1: return mirror_cols(b);
        case 2: return mirror_rows(b);
        case 3: return transpose(b);
        case 4: return mirror_cols(mirror_rows(transpose(b)));
        case 5: return mirror_cols(mirror_rows(b));
        case 6: return mirror_rows(transpose(b));
        case 7: return mirror_cols(transpose(b));
        default: return b;
    }
}

// Swap rows 0 and 2 (row 0 is the high 16 bits), all four columns.
__device__ __forceinline__ uint64_t swap_rows02(uint64_t b) {
    return (b & 0x0000FFFF0000FFFFull) | ((b >> 32) & 0x00000000FFFF0000ull) | ((b << 32) & 0xFFFF000000000000ull);
}

// Swap columns 0 and 2 (column 0 is the high nibble of a row), all four rows.
__device__ __forceinline__ uint64_t swap_cols02(uint64_t b) {
    return (b & 0x0F0F0F0F0F0F0F0Full) | ((b >> 8) & 0x00F000F000F000F0ull) | ((b << 8) & 0xF000F000F000F000ull);
}

// Bit offset of cell (r, c): row r (0 = high 16 bits), column c (0 = high nibble).
__host__ __device__ constexpr int cell_shift(int r, int c) { return 60 - 16 * r - 4 * c; }

// A symmetry of the top-left 3x3 block, every other cell fixed: kind 0 the
// transpose (r,c)->(c,r), 1 the anti-transpose (2-c,2-r), 2 the half turn
// (2-r,2-c), 3 and 4 the quarter turns (c,2-r) and (2-c,r).
template <int kKind>
__device__ __forceinline__ uint64_t block33(uint64_t b) {
    uint64_t o = b & 0x000F000F000FFFFFull;  // column 3 of rows 0-2 and row 3
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int R = kKind == 0 ? c : kKind == 1 ? 2 - c : kKind == 2 ? 2 - r : kKind == 3 ? c : 2 - c;
            const int C = kKind == 0 ? r : kKind == 1 ? 2 - r : kKind == 2 ? 2 - c : kKind == 3 ? 2 - r : r;
            o |= ((b >> cell_shift(r, c)) & 0xFull) << cell_shift(R, C);
        }
    }
    return o;
}

// Minimum over the symmetry group (canonical_by_mode,
// native_core/include/SymmetryUtils.h:31-49; the min33/min24/min34 groups of
// the variant boards, native_core/include/Calculator.h:192-203): 4 min33, the
// eight symmetries of the 3x3 block (its row and column swaps over whole
// rows and columns); 5 min24, the mirrors and half turn of the whole board;
// 6 min34, the column mirror and the row-0/row-2 swap of the 3x4 block and
// their product.
// Modes 4-6 (variant boards only).
__device__ __forceinline__ uint64_t canonical_variant(uint64_t b, int symm) {
    if (symm == 4) {
        uint64_t m = umin(b, umin(swap_cols02(b), swap_rows02(b)));
        m = umin(m, umin(block33<0>(b), block33<1>(b)));
        m = umin(m, block33<2>(b));
        return umin(m, umin(block33<3>(b), block33<4>(b)));
    }
    const uint64_t c = mirror_cols(b);
    if (symm == 5) return umin(umin(b, c), umin(mirror_rows(b), mirror_rows(c)));
    return umin(umin(b, c), umin(swap_rows02(b), swap_rows02(c)));
}

// kVariantModes = false leaves modes 4-6 out of the code (the hot kernels
// are instantiated both ways and launched by the table's mode): the caller
// then guarantees symm < 4.
template <bool kVariantModes = true>
__device__ __forceinline__ uint64_t canonical(uint64_t b, int symm) {
    if (symm == 0) return b;
    if (symm == 2) return umin(b, transpose(b));
    if (symm == 3) return umin(b, mirror_cols(b));
    if constexpr (kVariantModes) {
        if (symm >= 4) return canonical_variant(b, symm);
    }
    // full group: b and its transpose, each with the four row/column mirrors
    uint64_t t = transpose(b);
    uint64_t m = umin(b, t);
    uint64_t br = mirror_rows(b), tr = mirror_rows(t);
    m = umin(m, umin(br, tr));
    m = umin(m, umin(mirror_cols(b), mirror_cols(t)));
    m = umin(m, umin(mirror_cols(br), mirror_cols(tr)));
    return m;
}

// is_pattern (native_core/include/Formation.h:11-17)
__device__ __forceinline__ bool is_pattern(uint64_t b, const DevSpec &s) {
    if (s.n_masks == 0) return true;
    for (int i = 0; i < s.n_masks; ++i)
        if ((b & s.masks[i]) == s.masks[i]) return true;
    return false;
}

// is_success_by_shifts (native_core/include/Formation.h:32-43) as a
// zero-nibble test of b ^ target over the success nibbles.
__device__ __forceinline__ bool is_success(uint64_t b, const DevSpec &s) {
    if (!s.has_success) return true;
    const uint64_t x = b ^ s.target_rep;
    const uint64_t m7 = 0x7777777777777777ull;
    const uint64_t zero_hi = ~(((x & m7) + m7) | x | m7);
    return (zero_hi & s.succ_hi) != 0;
}

// The four moves of a board in the order left, right, up, down
// (move_all_dir, native_core/include/CommonMover.h:136-139).
__device__ __forceinline__ void move_all_dir(const uint32_t *__restrict__ tab, uint64_t b, uint64_t out[4]) {
    uint64_t dl = 0, dr = 0, ul = 0, ur = 0;
    const uint64_t t = transpose(b);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        uint32_t d = row_delta(tab, (uint32_t)(b >> (16 * r)) & 0xFFFFu);
        dl |= (uint64_t)(d & 0xFFFFu) << (16 * r);
        dr |= (uint64_t)(d >> 16) << (16 * r);
        uint32_t e = row_delta(tab, (uint32_t)(t >> (16 * r)) & 0xFFFFu);
        ul |= (uint64_t)(e & 0xFFFFu) << (16 * r);
        ur |= (uint64_t)(e >> 16) << (16 * r);
    }
    out[0] = b ^ dl;
    out[1] = b ^ dr;
    out[2] = transpose(t ^ ul);
    out[3] = transpose(t ^ ur);
}

// Row-table accessors: rows(row) = left delta | right delta << 16.
// GlobalRows reads the 65536-entry u32 table in global memory; SharedRows
// reads a u16 table of left deltas staged in shared memory (128 KB) and gets
// the right delta of a row as the reversed left delta of the reversed row.
struct GlobalRows {
    const uint32_t *__restrict__ t;
    __device__ __forceinline__ uint32_t operator()(uint32_t row) const { return __ldg(t + row); }
};

__device__ __forceinline__ uint32_t reverse_row(uint32_t r) {
    return ((r & 0xFu) << 12) | ((r & 0xF0u) << 4) | ((r >> 4) & 0xF0u) | (r >> 12);
}

struct SharedRows {
    const uint16_t *t;
    __device__ __forceinline__ uint32_t operator()(uint32_t row) const {
        return (uint32_t)t[row] | (reverse_row(t[reverse_row(row)]) << 16);
    }
};

// Copy the left halves of the u32 table into shared memory (every thread of
// the block calls it; ends with a barrier).
__device__ __forceinline__ void stage_rows(const uint32_t *__restrict__ tab, uint16_t *srows) {
    const uint4 *src = reinterpret_cast<const uint4 *>(tab);
    uint2 *dst = reinterpret_cast<uint2 *>(srows);
    for (int i = threadIdx.x; i < 65536 / 4; i += blockDim.x) {
        const uint4 q = __ldg(src + i);
        dst[i] = make_uint2((q.x & 0xFFFFu) | (q.y << 16), (q.z & 0xFFFFu) | (q.w << 16));
    }
    __syncthreads();
}

// Per-parent move context: the parent's row deltas (for left/right) and the
// transposed board's row deltas (for up/down). A spawn touches one row and
// one column, so a child's four moves need only the deltas of the touched
// row and column to be looked up again.
struct MoveCtx {
    uint64_t b, t;       // board and transpose
    uint64_t dl, dr;     // left/right deltas of b, all rows
    uint64_t ul, ur;     // left/right deltas of t, all rows (= up/down of b)
};

template <typename Rows>
__device__ __forceinline__ void move_ctx_init(const Rows &rows, uint64_t b, MoveCtx &c) {
    c.b = b;
    c.t = transpose(b);
    c.dl = c.dr = c.ul = c.ur = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        uint32_t d = rows((uint32_t)(b >> (16 * r)) & 0xFFFFu);
        c.dl |= (uint64_t)(d & 0xFFFFu) << (16 * r);
        c.dr |= (uint64_t)(d >> 16) << (16 * r);
        uint32_t e = rows((uint32_t)(c.t >> (16 * r)) & 0xFFFFu);
        c.ul |= (uint64_t)(e & 0xFFFFu) << (16 * r);
        c.ur |= (uint64_t)(e >> 16) << (16 * r);
    }
}

__device__ __forceinline__ void move_ctx_init(const uint32_t *__restrict__ tab, uint64_t b, MoveCtx &c) {
    move_ctx_init(GlobalRows{tab}, b, c);
}

// Transposed nibble index of nibble k: (r, c) -> (c, r) keeps k/4 <-> k%4.
__device__ __forceinline__ int transposed_nibble(int k) { return ((k & 3) << 2) | (k >> 2); }

// Moves of s = parent | v << 4k (nibble k empty in the parent).
template <typename Rows>
__device__ __forceinline__ void spawn_moves(const Rows &rows, const MoveCtx &c, int k, uint64_t v, uint64_t &s,
                                            uint64_t out[4]) {
    s = c.b | (v << (4 * k));
    const int row = k >> 2;
    const uint64_t rmask = 0xFFFFull << (16 * row);
    const uint32_t d = rows((uint32_t)(s >> (16 * row)) & 0xFFFFu);
    out[0] = s ^ ((c.dl & ~rmask) | ((uint64_t)(d & 0xFFFFu) << (16 * row)));
    out[1] = s ^ ((c.dr & ~rmask) | ((uint64_t)(d >> 16) << (16 * row)));
    const int kt = transposed_nibble(k);
    const uint64_t ts = c.t | (v << (4 * kt));
    const int trow = kt >> 2;
    const uint64_t tmask = 0xFFFFull << (16 * trow);
    const uint32_t e = rows((uint32_t)(ts >> (16 * trow)) & 0xFFFFu);
    out[2] = transpose(ts ^ ((c.ul & ~tmask) | ((uint64_t)(e & 0xFFFFu) << (16 * trow))));
    out[3] = transpose(ts ^ ((c.ur & ~tmask) | ((uint64_t)(e >> 16) << (16 * trow))));
}

__device__ __forceinline__ void spawn_moves(const uint32_t *__restrict__ tab, const MoveCtx &c, int k, uint64_t v,
                                            uint64_t &s, uint64_t out[4]) {
    spawn_moves(GlobalRows{tab}, c, k, v, s, out);
}

// Bit set in nibble k's low bit for every empty nibble of b.
__device__ __forceinline__ uint64_t empty_nibbles(uint64_t b) {
    uint64_t x = b | (b >> 1);
    x |= x >> 2;
    return ~x & 0x1111111111111111ull;
}

// Multiplicative hash for the device-side repeat filter (any hash works: the
// filter only drops repeats, never a first occurrence).
__device__ __forceinline__ uint64_t filter_slot(uint64_t key, int bits) {
    return (key * 0x9E3779B97F4A7C15ull) >> (64 - bits);
}

// 64-bit mix (the finaliser of MurmurHash3) for the device hash sets.
__device__ __forceinline__ uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xFF51AFD7ED558CCDull;
    k ^= k >> 33;
    k *= 0xC4CEB9FE1A85EC53ull;
    k ^= k >> 33;
    return k;
}

constexpr int kSplitStride = 16;  // one splitter per 16 keys (one 128-byte line)

// Exact search of key in layer keys[0..n) with splitters split[j] =
// keys[16j]: branchless search over the splitters, then over one 16-key line.
template <typename T>
__device__ __forceinline__ T layer_lookup(const uint64_t *__restrict__ keys, const T *__restrict__ rates,
                                          unsigned long long n, const uint64_t *__restrict__ split, uint64_t key,
                                          T zero) {
    if (n == 0) return zero;
    const unsigned long long ns = (n + kSplitStride - 1) / kSplitStride;
    if (key < __ldg(split)) return zero;
    unsigned long long lo = 0, len = ns;
    while (len > 1) {
        const unsigned long long half = len >> 1;
        lo = (__ldg(split + lo + half) <= key) ? lo + half : lo;
        len -= half;
    }
    unsigned long long b = lo * kSplitStride;
    unsigned long long m = n - b < (unsigned long long)kSplitStride ? n - b : (unsigned long long)kSplitStride;
    // lower bound inside the line
    while (m > 1) {
        const unsigned long long half = m >> 1;
        b = (__ldg(keys + b + half) <= key) ? b + half : b;
        m -= half;
    }
    return __ldg(keys + b) == key ? rates[b] : zero;
}

}  // namespace egtb
