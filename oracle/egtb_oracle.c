/*
 * CPU oracle for the classic endgame-tablebase build/lookup path.
 *
 * TEST INFRASTRUCTURE ONLY — a plain-C restatement of the reference algorithm
 * (game-difficulty/2048EndgameTablebase, native_core/). Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as
 * the checker. Built with -ffp-contract=off so the one place the reference's
 * -Ofast build contracts to FMA (the backward accumulation, see or_solve_layer)
 * is written out explicitly with fma().
 *
 * Board layout (native_core/include/BoardCodec.h:20-30): 4x4 board packed in a
 * uint64, one log2 nibble per cell; nibble k holds row 3-k/4, column 3-k%4, so
 * row 0 is the high 16 bits and column 0 the high nibble of each row.
 */
#include "egtb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- rows --- */

static uint16_t g_left[2][65536], g_right[2][65536];  /* [0] classic, [1] variant */
static int g_tables_ready = 0;

/* One row moved toward column 0 (reverse=0) or column 3 (reverse=1).
 * walls=0 restates StandardMergePolicy::_internal_merge,
 * native_core/include/BoardMover.h:6-55: slide non-empty cells, merge each
 * adjacent equal pair once (first pair first), the 32768 tile (nibble 0xF)
 * never merges. walls=1 restates WallMergePolicy::_internal_merge,
 * native_core/include/VBoardMover.h:7-76: 0xF cells stay where they are and
 * split the row into stretches, each moved like a row of its own.
 * Works on log2 nibbles. */
static uint16_t row_move(uint16_t row, int reverse, int walls) {
    int line[4], out[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) line[i] = (row >> (4 * (3 - i))) & 0xF;
    if (reverse) {
        int t = line[0]; line[0] = line[3]; line[3] = t;
        t = line[1]; line[1] = line[2]; line[2] = t;
    }
    int lo = 0;
    while (lo < 4) {
        if (walls && line[lo] == 0xF) {
            out[lo] = 0xF;
            ++lo;
            continue;
        }
        int hi = lo, nz[4], n = 0, m = lo;
        while (hi < 4 && !(walls && line[hi] == 0xF)) {
            if (line[hi]) nz[n++] = line[hi];
            ++hi;
        }
        for (int i = 0; i < n; ++i) {
            if (i + 1 < n && nz[i] == nz[i + 1] && nz[i] != 0xF) {
                out[m++] = nz[i] + 1;
                ++i;
            } else {
                out[m++] = nz[i];
            }
        }
        lo = hi;
    }
    if (reverse) {
        int t = out[0]; out[0] = out[3]; out[3] = t;
        t = out[1]; out[1] = out[2]; out[2] = t;
    }
    uint16_t r = 0;
    for (int i = 0; i < 4; ++i) r |= (uint16_t)((out[i] & 0xF) << (4 * (3 - i)));
    return r;
}

/* XOR-delta row tables, native_core/include/CommonMover.h:87-94 */
static void init_tables(void) {
    if (g_tables_ready) return;
    for (int w = 0; w < 2; ++w)
        for (uint32_t r = 0; r < 65536; ++r) {
            g_left[w][r] = (uint16_t)(row_move((uint16_t)r, 0, w) ^ r);
            g_right[w][r] = (uint16_t)(row_move((uint16_t)r, 1, w) ^ r);
        }
    g_tables_ready = 1;
}

void or_row_tables(uint16_t *left_xor, uint16_t *right_xor) {
    init_tables();
    memcpy(left_xor, g_left[0], sizeof g_left[0]);
    memcpy(right_xor, g_right[0], sizeof g_right[0]);
}

void or_row_tables_variant(uint16_t *left_xor, uint16_t *right_xor) {
    init_tables();
    memcpy(left_xor, g_left[1], sizeof g_left[1]);
    memcpy(right_xor, g_right[1], sizeof g_right[1]);
}

/* ------------------------------------------------------------ symmetry --- */

static inline int nib(uint64_t b, int r, int c) { return (int)((b >> (4 * ((3 - r) * 4 + (3 - c)))) & 0xF); }
static inline uint64_t put(int v, int r, int c) { return (uint64_t)v << (4 * ((3 - r) * 4 + (3 - c))); }

/* The eight symmetries of the square as cell maps (r,c) -> (r',c'),
 * numbered as apply_sym_like, native_core/include/SymmetryUtils.h:9-29 /
 * native_core/include/Calculator.h:28-78:
 * 0 identity, 1 mirror columns, 2 mirror rows, 3 transpose, 4 anti-transpose,
 * 5 half turn, 6 quarter turn counter-clockwise, 7 quarter turn clockwise. */
uint64_t or_apply_sym(uint64_t b, int idx) {
    uint64_t o = 0;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            int v = nib(b, r, c), R = r, C = c;
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
            o |= put(v, R, C);
        }
    return o;
}

/* A cell map on the board: cell (r,c) goes to (R,C) = f(r,c); cells the map
 * does not move keep their value. */
static uint64_t cell_map(uint64_t b, int kind) {
    uint64_t o = 0;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            int R = r, C = c;
            const int in33 = r < 3 && c < 3;
            switch (kind) {
                case 0: if (c == 0) C = 2; else if (c == 2) C = 0; break;       /* columns 0 <-> 2 */
                case 1: if (r == 0) R = 2; else if (r == 2) R = 0; break;       /* rows 0 <-> 2 */
                case 2: if (in33) { R = c; C = r; } break;                      /* 3x3 transpose */
                case 3: if (in33) { R = 2 - c; C = 2 - r; } break;              /* 3x3 anti-transpose */
                case 4: if (in33) { R = 2 - r; C = 2 - c; } break;              /* 3x3 half turn */
                case 5: if (in33) { R = c; C = 2 - r; } break;                  /* 3x3 quarter turn */
                case 6: if (in33) { R = 2 - c; C = r; } break;                  /* 3x3 quarter turn */
                default: break;
            }
            o |= put(nib(b, r, c), R, C);
        }
    return o;
}

static inline uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

/* canonical_by_mode, native_core/include/SymmetryUtils.h:31-49 with
 * Calculator::canonical_{identity,full,diagonal,horizontal,min33,min24,min34}
 * (native_core/include/Calculator.h:80-97, 192-203): the minimum over the
 * group. min33: the eight symmetries of the top-left 3x3 block, its column
 * and row swaps taken over whole columns and rows; min24: the mirrors and
 * half turn of the board; min34: the column mirror, the swap of rows 0 and
 * 2, and both. */
uint64_t or_canonical(uint64_t b, int mode) {
    uint64_t m = b, t;
    switch (mode) {
        case OR_SYM_MIN33:
            for (int k = 0; k < 7; ++k) m = umin64(m, cell_map(b, k));
            return m;
        case OR_SYM_MIN24:
            m = umin64(m, or_apply_sym(b, 1));
            m = umin64(m, or_apply_sym(b, 2));
            return umin64(m, or_apply_sym(b, 5));
        case OR_SYM_MIN34:
            t = or_apply_sym(b, 1);
            m = umin64(m, t);
            m = umin64(m, cell_map(b, 1));
            return umin64(m, cell_map(t, 1));
        case OR_SYM_FULL:
            for (int i = 1; i < 8; ++i) {
                t = or_apply_sym(b, i);
                if (t < m) m = t;
            }
            return m;
        case OR_SYM_DIAGONAL:
            t = or_apply_sym(b, 3);
            return t < m ? t : m;
        case OR_SYM_HORIZONTAL:
            t = or_apply_sym(b, 1);
            return t < m ? t : m;
        default:
            return b;
    }
}

/* -------------------------------------------------------------- moves --- */

/* transpose, the reference's reverse_board (native_core/include/CommonMover.h:33-37) */
static inline uint64_t transpose(uint64_t b) { return or_apply_sym(b, 3); }

static inline uint64_t rows_apply(uint64_t b, const uint16_t *tab) {
    uint64_t o = b;
    for (int r = 0; r < 4; ++r) o ^= (uint64_t)tab[(b >> (16 * r)) & 0xFFFF] << (16 * r);
    return o;
}

/* move_all_dir: {left, right, up, down}, native_core/include/CommonMover.h:136-139,
 * with the classic (BoardMover) or the variant (VBoardMover) row rule */
static void move_all_dir_w(uint64_t b, uint64_t out[4], int variant) {
    init_tables();
    const int w = variant ? 1 : 0;
    uint64_t t = transpose(b);
    out[0] = rows_apply(b, g_left[w]);
    out[1] = rows_apply(b, g_right[w]);
    out[2] = transpose(rows_apply(t, g_left[w]));
    out[3] = transpose(rows_apply(t, g_right[w]));
}

void or_move_all_dir(uint64_t b, uint64_t out[4]) { move_all_dir_w(b, out, 0); }

void or_move_all_dir_batch(const uint64_t *b, size_t n, uint64_t *out4) {
    for (size_t i = 0; i < n; ++i) move_all_dir_w(b[i], out4 + 4 * i, 0);
}

void or_move_all_dir_variant_batch(const uint64_t *b, size_t n, uint64_t *out4) {
    for (size_t i = 0; i < n; ++i) move_all_dir_w(b[i], out4 + 4 * i, 1);
}

void or_canonical_batch(const uint64_t *b, size_t n, int mode, uint64_t *out) {
    for (size_t i = 0; i < n; ++i) out[i] = or_canonical(b[i], mode);
}

/* is_pattern, native_core/include/Formation.h:11-17 */
int or_is_pattern(uint64_t b, const or_spec *s) {
    if (s->n_masks == 0) return 1;
    for (int i = 0; i < s->n_masks; ++i)
        if ((b & s->masks[i]) == s->masks[i]) return 1;
    return 0;
}

/* is_success_by_shifts, native_core/include/Formation.h:32-43 */
int or_is_success(uint64_t b, int target, const or_spec *s) {
    if (s->n_shifts == 0) return 1;
    for (int i = 0; i < s->n_shifts; ++i)
        if (((b >> s->shifts[i]) & 0xF) == (uint64_t)target) return 1;
    return 0;
}

/* ------------------------------------------------------------- forward --- */

/* Children of one parent layer: for each parent (skipped when do_check and
 * it is a success), each empty nibble i ascending, spawn 2 then 4, the four
 * moves; a child is kept if it moved and matches the pattern, and is stored
 * canonicalised. Restates gen_boards_simple / gen_boards_internal_naive,
 * native_core/src/BookGenerator.cpp:717-760 and :472-589 (the lossy hash
 * prefilter of :112-127,150-181 only drops repeats and is omitted). */
size_t or_expand(const uint64_t *parents, size_t n, const or_spec *spec, int target, int do_check,
                 uint64_t *out1, uint64_t *out2, size_t cap, size_t *n2) {
    size_t c1 = 0, c2 = 0;
    uint64_t mv[4];
    for (size_t p = 0; p < n; ++p) {
        uint64_t b = parents[p];
        if (do_check && or_is_success(b, target, spec)) continue;
        for (int i = 0; i < 16; ++i) {
            if ((b >> (4 * i)) & 0xF) continue;
            for (uint64_t v = 1; v <= 2; ++v) {
                uint64_t s = b | (v << (4 * i));
                move_all_dir_w(s, mv, spec->is_variant);
                for (int d = 0; d < 4; ++d) {
                    if (mv[d] == s || !or_is_pattern(mv[d], spec)) continue;
                    uint64_t k = or_canonical(mv[d], spec->symm_mode);
                    if (v == 1) {
                        if (c1 < cap) out1[c1] = k;
                        ++c1;
                    } else {
                        if (c2 < cap) out2[c2] = k;
                        ++c2;
                    }
                }
            }
        }
    }
    *n2 = c2;
    return c1;
}

/* LSD radix sort, 16-bit digits, then in-place unique. Any correct sort gives
 * the reference's result: sort_array + parallel_unique
 * (native_core/src/BookGeneratorUtils.cpp:138-158) leave a strictly
 * ascending array. */
static size_t sort_unique(uint64_t *a, size_t n) {
    if (n < 2) return n;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    size_t *cnt = (size_t *)malloc(65536 * sizeof(size_t));
    uint64_t *src = a, *dst = tmp;
    for (int pass = 0; pass < 4; ++pass) {
        int sh = 16 * pass;
        memset(cnt, 0, 65536 * sizeof(size_t));
        for (size_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xFFFF]++;
        size_t s = 0;
        for (int d = 0; d < 65536; ++d) {
            size_t c = cnt[d];
            cnt[d] = s;
            s += c;
        }
        for (size_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
        uint64_t *t = src; src = dst; dst = t;
    }
    /* four passes: result is back in a */
    size_t m = 1;
    for (size_t i = 1; i < n; ++i)
        if (a[i] != a[m - 1]) a[m++] = a[i];
    free(tmp);
    free(cnt);
    return m;
}

struct or_build {
    int steps;
    uint64_t **keys;
    size_t *len;
    void **rates;
    int dtype;
    or_spec spec;
    uint64_t *masks;
    uint8_t *shifts;
    int target, docheck;
};

/* The layer loop of generate_process, native_core/src/BookGenerator.cpp:963-1121:
 * layer 0 = the seeds; for i = 1 .. steps-2 the parents are layer i-1, checked
 * for success iff i > docheck_step (:991); layer i = unique(partial_i U spawn-2
 * children) (:1059-1078); the spawn-4 children become partial_{i+1}. The last
 * layer (steps-1) is left partial, as the reference leaves it (:978). */
or_build *or_generate(const uint64_t *seeds, size_t n_seeds, const or_spec *spec,
                      int target, int steps, int docheck_step) {
    init_tables();
    or_build *b = (or_build *)calloc(1, sizeof(or_build));
    b->steps = steps;
    b->keys = (uint64_t **)calloc((size_t)steps, sizeof(uint64_t *));
    b->len = (size_t *)calloc((size_t)steps, sizeof(size_t));
    b->rates = (void **)calloc((size_t)steps, sizeof(void *));
    b->masks = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(spec->n_masks + 1));
    b->shifts = (uint8_t *)malloc((size_t)spec->n_shifts + 1);
    memcpy(b->masks, spec->masks, sizeof(uint64_t) * (size_t)spec->n_masks);
    memcpy(b->shifts, spec->shifts, (size_t)spec->n_shifts);
    b->spec = *spec;
    b->spec.masks = b->masks;
    b->spec.shifts = b->shifts;
    b->target = target;
    b->docheck = docheck_step;

    b->keys[0] = (uint64_t *)malloc(sizeof(uint64_t) * (n_seeds + 1));
    memcpy(b->keys[0], seeds, sizeof(uint64_t) * n_seeds);
    b->len[0] = n_seeds; /* written as-is, BookGenerator.cpp:417-419 */

    uint64_t *partial = NULL;
    size_t npartial = 0;
    for (int i = 1; i < steps - 1; ++i) {
        const uint64_t *par = b->keys[i - 1];
        size_t np = b->len[i - 1];
        int do_check = i > docheck_step;
        size_t cap = np * 64 + 16, n2 = 0;
        uint64_t *s1 = (uint64_t *)malloc(sizeof(uint64_t) * (cap + npartial));
        uint64_t *s2 = (uint64_t *)malloc(sizeof(uint64_t) * cap);
        size_t n1 = or_expand(par, np, &b->spec, target, do_check, s1, s2, cap, &n2);
        if (npartial) memcpy(s1 + n1, partial, sizeof(uint64_t) * npartial);
        free(partial);
        n1 = sort_unique(s1, n1 + npartial);
        n2 = sort_unique(s2, n2);
        b->keys[i] = s1;
        b->len[i] = n1;
        partial = s2;
        npartial = n2;
    }
    if (steps >= 2) {
        b->keys[steps - 1] = partial ? partial : (uint64_t *)malloc(8);
        b->len[steps - 1] = npartial;
    }
    return b;
}

int or_num_layers(const or_build *b) { return b->steps; }
size_t or_layer_len(const or_build *b, int t) { return b->len[t]; }
const uint64_t *or_layer_keys(const or_build *b, int t) { return b->keys[t]; }
const void *or_layer_rates(const or_build *b, int t) { return b->rates[t]; }

void or_free(or_build *b) {
    if (!b) return;
    for (int t = 0; t < b->steps; ++t) {
        free(b->keys[t]);
        free(b->rates[t]);
    }
    free(b->keys);
    free(b->len);
    free(b->rates);
    free(b->masks);
    free(b->shifts);
    free(b);
}

/* ------------------------------------------------------------ backward --- */

static size_t dtype_size(int dtype) {
    switch (dtype) {
        case OR_U64: case OR_F64: case OR_1F64: return 8;
        default: return 4;
    }
}

/* zero_value_for_dtype / max_scale_value_for_dtype,
 * native_core/include/FormationRuntime.h:257-312 (the "1-float" kinds store
 * success-1, so 'zero' is -1 and 'max' is 0). */
static double dtype_zero(int dtype) { return (dtype == OR_1F32 || dtype == OR_1F64) ? -1.0 : 0.0; }
static double dtype_max(int dtype) {
    switch (dtype) {
        case OR_U32: return 4000000000.0;
        case OR_U64: return 1600000000000000000.0;
        case OR_F32: case OR_F64: return 1.0;
        default: return 0.0;
    }
}

/* exact search: the value stored for key, or the dtype's zero on a miss
 * (search_arr, native_core/src/BookSolver.cpp:329-346) */
#define DEFINE_LOOKUP(T, NAME)                                                       \
    static T NAME(const uint64_t *k, const T *r, size_t n, uint64_t key, T zero) {  \
        size_t lo = 0, hi = n;                                                       \
        while (lo < hi) {                                                            \
            size_t mid = lo + (hi - lo) / 2;                                         \
            if (k[mid] < key) lo = mid + 1; else hi = mid;                           \
        }                                                                            \
        return (lo < n && k[lo] == key) ? r[lo] : zero;                              \
    }
DEFINE_LOOKUP(uint32_t, lookup_u32)
DEFINE_LOOKUP(uint64_t, lookup_u64)
DEFINE_LOOKUP(float, lookup_f32)
DEFINE_LOOKUP(double, lookup_f64)

/* recalculate_layer, native_core/src/BookSolver.cpp:413-470, per board:
 *   success and do_check -> max scale;
 *   else acc = 0.0 (double); for every empty nibble i ascending:
 *     best2 = max over kept moves of rate_{t+1}(canonical(move(b | 1<<4i))), T-typed, from zero
 *     acc   = fma(double(best2), 1 - p4, acc)
 *     best4 = likewise from layer t+2 with b | 2<<4i
 *     acc   = fma(double(best4), p4, acc)
 *   rate = T(acc / double(#empty)), or zero when there is no empty nibble.
 * The two fma() calls are the reference's `success_probability += ...`
 * statements as its -Ofast -march=x86-64-v3 build compiles them (FMA
 * contraction; native_core/CMakeLists.txt:80-87). */
#define DEFINE_SOLVE(T, NAME, LOOKUP, CAST)                                                     \
    static void NAME(const uint64_t *keys0, size_t n0, T *out, const uint64_t *k1, const T *r1,  \
                     size_t n1, const uint64_t *k2, const T *r2, size_t n2, const or_spec *spec,  \
                     int target, int do_check, int dtype, double p4) {                          \
        const T zero = (T)dtype_zero(dtype), maxv = (T)dtype_max(dtype);                         \
        const double w2 = 1.0 - p4;                                                              \
        _Pragma("omp parallel for schedule(dynamic, 1024)")                                      \
        for (size_t k = 0; k < n0; ++k) {                                                        \
            uint64_t b = keys0[k], mv[4];                                                        \
            if (do_check && or_is_success(b, target, spec)) {                                    \
                out[k] = maxv;                                                                   \
                continue;                                                                        \
            }                                                                                    \
            double acc = 0.0;                                                                    \
            int empty = 0;                                                                       \
            for (int i = 0; i < 16; ++i) {                                                       \
                if ((b >> (4 * i)) & 0xF) continue;                                              \
                ++empty;                                                                         \
                for (uint64_t v = 1; v <= 2; ++v) {                                              \
                    uint64_t s = b | (v << (4 * i));                                             \
                    T best = zero;                                                               \
                    move_all_dir_w(s, mv, spec->is_variant);                                     \
                    for (int d = 0; d < 4; ++d) {                                                \
                        if (mv[d] == s || !or_is_pattern(mv[d], spec)) continue;                 \
                        uint64_t key = or_canonical(mv[d], spec->symm_mode);                     \
                        T got = (v == 1) ? LOOKUP(k1, r1, n1, key, zero)                         \
                                         : LOOKUP(k2, r2, n2, key, zero);                        \
                        if (best < got) best = got;                                              \
                    }                                                                            \
                    acc = fma((double)best, v == 1 ? w2 : p4, acc);                              \
                }                                                                                \
            }                                                                                    \
            out[k] = empty > 0 ? CAST(acc / (double)empty) : zero;                               \
        }                                                                                        \
    }
#define CAST_U32(x) ((uint32_t)(x))
#define CAST_U64(x) ((uint64_t)(x))
#define CAST_F32(x) ((float)(x))
#define CAST_F64(x) ((double)(x))
DEFINE_SOLVE(uint32_t, solve_u32, lookup_u32, CAST_U32)
DEFINE_SOLVE(uint64_t, solve_u64, lookup_u64, CAST_U64)
DEFINE_SOLVE(float, solve_f32, lookup_f32, CAST_F32)
DEFINE_SOLVE(double, solve_f64, lookup_f64, CAST_F64)

void or_solve_layer(const uint64_t *keys0, size_t n0, void *rates0,
                    const uint64_t *k1, const void *r1, size_t n1,
                    const uint64_t *k2, const void *r2, size_t n2,
                    const or_spec *spec, int target, int do_check, int dtype, double p4) {
    init_tables();
    switch (dtype) {
        case OR_U32:
            solve_u32(keys0, n0, (uint32_t *)rates0, k1, (const uint32_t *)r1, n1, k2, (const uint32_t *)r2, n2,
                      spec, target, do_check, dtype, p4);
            break;
        case OR_U64:
            solve_u64(keys0, n0, (uint64_t *)rates0, k1, (const uint64_t *)r1, n1, k2, (const uint64_t *)r2, n2,
                      spec, target, do_check, dtype, p4);
            break;
        case OR_F32: case OR_1F32:
            solve_f32(keys0, n0, (float *)rates0, k1, (const float *)r1, n1, k2, (const float *)r2, n2,
                      spec, target, do_check, dtype, p4);
            break;
        default:
            solve_f64(keys0, n0, (double *)rates0, k1, (const double *)r1, n1, k2, (const double *)r2, n2,
                      spec, target, do_check, dtype, p4);
            break;
    }
}

/* final_situation_process for layers steps-2 and steps-1
 * (native_core/src/BookSolver.cpp:237-284): success -> max scale, else zero;
 * then recalculate_process_impl (:513-605) for layers steps-3 .. 0 with
 * do_check = i > docheck_step (:562). */
int or_solve(or_build *b, int dtype, double spawn_rate4) {
    init_tables();
    const size_t es = dtype_size(dtype);
    b->dtype = dtype;
    const double zero = dtype_zero(dtype), maxv = dtype_max(dtype);
    for (int t = b->steps - 2; t < b->steps; ++t) {
        if (t < 0) continue;
        free(b->rates[t]);
        b->rates[t] = malloc(es * (b->len[t] + 1));
        for (size_t k = 0; k < b->len[t]; ++k) {
            int s = or_is_success(b->keys[t][k], b->target, &b->spec);
            double v = s ? maxv : zero;
            switch (dtype) {
                case OR_U32: ((uint32_t *)b->rates[t])[k] = (uint32_t)v; break;
                case OR_U64: ((uint64_t *)b->rates[t])[k] = (uint64_t)v; break;
                case OR_F32: case OR_1F32: ((float *)b->rates[t])[k] = (float)v; break;
                default: ((double *)b->rates[t])[k] = v; break;
            }
        }
    }
    for (int t = b->steps - 3; t >= 0; --t) {
        free(b->rates[t]);
        b->rates[t] = malloc(es * (b->len[t] + 1));
        or_solve_layer(b->keys[t], b->len[t], b->rates[t], b->keys[t + 1], b->rates[t + 1], b->len[t + 1],
                       b->keys[t + 2], b->rates[t + 2], b->len[t + 2], &b->spec, b->target,
                       t > b->docheck, dtype, spawn_rate4);
    }
    return 0;
}

/* ================================================================ advanced ===
 * The advanced algorithm's masked-board primitives (namespace FormationAD),
 * restated on tile values: a masked board holds every tile of 64 and up as
 * the 0xF ("32k", value 32768) nibble. */

static uint32_t tile_value(int nibble) { return nibble ? 1u << nibble : 0u; }

static int tile_nibble(uint32_t v) {
    int n = 0;
    while (v > 1) {
        v >>= 1;
        ++n;
    }
    return n;
}

/* One line of four cells moved toward cell 0 (merge_line,
 * native_core/src/BoardMoverAD.cpp:49-89): 32768 never merges; a merged
 * value of 64 or more becomes 32768 and sets *made. */
static void ad_merge_line(int cells[4], int *made) {
    uint32_t nz[4], out[4] = {0, 0, 0, 0};
    int k = 0, m = 0;
    for (int i = 0; i < 4; ++i)
        if (cells[i]) nz[k++] = tile_value(cells[i]);
    for (int i = 0; i < k; ++i) {
        if (i + 1 < k && nz[i] == nz[i + 1] && nz[i] != 32768u) {
            uint32_t v = nz[i] * 2u;
            if (v >= 64u) {
                *made = 1;
                v = 32768u;
            }
            out[m++] = v;
            ++i;
        } else {
            out[m++] = nz[i];
        }
    }
    for (int i = 0; i < 4; ++i) cells[i] = tile_nibble(out[i]);
}

/* every row of b moved toward column 0 (reverse=0) or column 3 */
static uint64_t ad_rows(uint64_t b, int reverse, int *made) {
    uint64_t o = 0;
    for (int r = 0; r < 4; ++r) {
        int cells[4];
        for (int c = 0; c < 4; ++c) cells[reverse ? 3 - c : c] = nib(b, r, c);
        ad_merge_line(cells, made);
        for (int c = 0; c < 4; ++c) o |= put(cells[reverse ? 3 - c : c], r, c);
    }
    return o;
}

/* m_move_all_dir, native_core/src/BoardMoverAD.cpp:171-178: {left, right,
 * up, down}; left and right carry the left merge's flag, up and down the up
 * merge's */
void or_ad_move_all_dir_batch(const uint64_t *b, size_t n, uint64_t *out4, uint8_t *flags4) {
    for (size_t i = 0; i < n; ++i) {
        int fh = 0, fv = 0, ignored = 0;
        const uint64_t t = transpose(b[i]);
        out4[4 * i + 0] = ad_rows(b[i], 0, &fh);
        out4[4 * i + 1] = ad_rows(b[i], 1, &ignored);
        out4[4 * i + 2] = transpose(ad_rows(t, 0, &fv));
        out4[4 * i + 3] = transpose(ad_rows(t, 1, &ignored));
        flags4[4 * i + 0] = flags4[4 * i + 1] = (uint8_t)fh;
        flags4[4 * i + 2] = flags4[4 * i + 3] = (uint8_t)fv;
    }
}

/* mask_board, native_core/src/BoardMaskerAD.cpp:112-121 */
uint64_t or_ad_mask_board(uint64_t b, int threshold) {
    uint64_t m = b;
    for (int k = 0; k < 16; ++k)
        if (((b >> (4 * k)) & 0xFull) >= (uint64_t)(int64_t)threshold) m |= 0xFull << (4 * k);
    return m;
}

/* Tile statistics after the fixed 32k cells are cleared:
 * kind 1 tile_sum_and_32k_count (BoardMaskerAD.cpp:123-144, 32k = 0xF only),
 * kind 2 tile_sum_and_32k_count2 (:169-190, 32k = 64 and up),
 * kind 4 tile_sum_and_32k_count4 (:219-257). Per 16-bit row as the
 * reference's info tables hold it (:24-50): a uint16 tile sum, and pos_rank =
 * the 0xF cells met, from the row's high nibble down, before its first
 * non-0xF 32k tile. out8: total_sum, count_32k, pos_bitmap low, high,
 * pos_rank, merged_tile_found, merged_tile, is_success. */
void or_ad_tile_stats(uint64_t b, const or_ad_param *p, int kind, int64_t out8[8]) {
    b &= ~p->pos_fixed_32k_mask;
    uint32_t total = 0, count = 0, found = 0, merged = 0, rank[4], rowfound[4];
    uint64_t pos = 0;
    for (int k = 0; k < 4; ++k) {
        uint16_t sum16 = 0;
        rank[k] = rowfound[k] = 0;
        for (int i = 3; i >= 0; --i) {
            const int sh = 16 * k + 4 * i;
            const int v = (int)((b >> sh) & 0xF);
            const int large = kind == 1 ? v == 15 : v > 5;
            if (large) {
                pos |= 0xFull << sh;
                ++count;
                if (v == 15) {
                    if (rowfound[k] == 0) ++rank[k];
                } else {
                    ++rowfound[k];
                    merged ^= (uint32_t)v;
                }
            } else if (v > 0) {
                sum16 = (uint16_t)(sum16 + (1u << v));
            }
        }
        total += sum16;
        found += rowfound[k];
    }
    memset(out8, 0, 8 * sizeof(int64_t));
    out8[0] = total;
    out8[1] = count;
    out8[2] = (int64_t)(pos & 0xFFFFFFFFull);
    out8[3] = (int64_t)(pos >> 32);
    if (kind == 4) {
        /* the 0xF cells counted from the top row down to the first row with a merged tile */
        uint32_t r = 0;
        for (int k = 3; k >= 0; --k) {
            r += rank[k];
            if (rowfound[k]) break;
        }
        out8[4] = r;
        out8[5] = found;
        out8[6] = merged;
        out8[7] = (merged == (p->target & 0xFFu) && found == 1) ? 1 : 0;
    }
}

/* masked_tiles_combinations (BoardMaskerAD.cpp:259-289), stored ascending as
 * init_masker stores it (:524-531): count tiles of 64 .. 8192 summing to
 * sum, largest first, with the reference's early exits; returns the length
 * (0: none). */
static int ad_combination(uint32_t sum, int count, uint8_t out[16]) {
    uint8_t tiles[16];
    int len = 0;
    for (uint32_t tile = 8192; tile >= 64; tile >>= 1) {
        if (tile > sum) continue;
        if (tile == sum) {
            if (count == 1) {
                tiles[len++] = (uint8_t)tile_nibble(tile);
                goto done;
            }
            continue;
        }
        if (2 * tile == sum && count == 2) {
            tiles[len++] = (uint8_t)tile_nibble(tile);
            tiles[len++] = (uint8_t)tile_nibble(tile);
            goto done;
        }
        if (tile != 64 && sum == 192 && count == 3) {
            tiles[len++] = 6;
            tiles[len++] = 6;
            tiles[len++] = 6;
            goto done;
        }
        sum -= tile;
        --count;
        tiles[len++] = (uint8_t)tile_nibble(tile);
    }
    return 0;
done:
    for (int i = 0; i < len; ++i) out[i] = tiles[len - 1 - i];
    return len;
}

/* validate, native_core/src/BoardMaskerAD.cpp:409-443 (boards whose 32k count
 * is num_free_32k .. num_free_32k + 9, where the reference's table lookup
 * stays inside its table) */
int or_ad_validate(uint64_t b, uint32_t original_sum, const or_ad_param *p) {
    int64_t st[8];
    or_ad_tile_stats(b, p, 2, st);
    const uint32_t total = (uint32_t)st[0];
    const int8_t count = (int8_t)st[1], free32k = (int8_t)p->num_free_32k;
    if (total >= p->small_tile_sum_limit + 64u) return 0;
    if (count == free32k) return 1;
    const uint32_t large = original_sum - total - ((uint32_t)(p->num_free_32k + p->num_fixed_32k) << 15);
    const uint8_t a = (uint8_t)(large >> 6), c = (uint8_t)(count - free32k);
    uint8_t tc[16];
    const int len = (a == 0 || c >= 10) ? 0 : ad_combination((uint32_t)a << 6, c, tc);  /* table: a > 0, c < 10 */
    if (len == 0) return 0;
    if (tc[len - 1] == (uint8_t)p->target) return 0;
    if (count < 2) return 1;
    if (len > 2 && tc[0] == tc[2]) return total >= p->small_tile_sum_limit - 64u ? 0 : 1;
    if (len > 1 && tc[0] == tc[1]) return total >= p->small_tile_sum_limit ? 0 : 1;
    return 1;
}

/* unmask_board, native_core/src/BoardMaskerAD.cpp:445-512, over the slots
 * of init_masker (:514-533). The permutation rows of slot (m, n) come in
 * the order resort_permutations gives them (:291-332): by the cells'
 * contents read from cell 0 to cell m-1 (value j, or 15 for a cell left
 * out), produced here directly in that order by a depth-first walk that
 * tries a cell's values smallest first and "left out" last. */
typedef struct {
    uint64_t board;
    const uint8_t *pos; /* 0xF cells, highest first */
    const uint8_t *tc;
    int m, n, len, ordered;
    uint64_t *out;
    size_t cap, total;
} ad_walk;

static void ad_emit(ad_walk *w, const int cell_of[16]) {
    if (w->ordered && !(cell_of[1] < cell_of[0])) return;
    uint64_t clear = 0, set = 0;
    for (int j = 0; j < w->len; ++j) {
        clear += 0xFull << w->pos[cell_of[j]];
        set += (uint64_t)w->tc[j] << w->pos[cell_of[j]];
    }
    if (w->total < w->cap) w->out[w->total] = (w->board & ~clear) | set;
    ++w->total;
}

static void ad_walk_cells(ad_walk *w, int cell, int placed, int used_mask, int cell_of[16]) {
    if (cell == w->m) {
        if (placed == w->n) ad_emit(w, cell_of);
        return;
    }
    for (int j = 0; j < w->n; ++j) {
        if (used_mask >> j & 1) continue;
        cell_of[j] = cell;
        ad_walk_cells(w, cell + 1, placed + 1, used_mask | (1 << j), cell_of);
    }
    if (w->m - cell - 1 >= w->n - placed) ad_walk_cells(w, cell + 1, placed, used_mask, cell_of);
}

size_t or_ad_unmask(uint64_t b, uint32_t original_sum, const or_ad_param *p, uint64_t *out, size_t cap) {
    const uint64_t masked = b & ~p->pos_fixed_32k_mask;
    int64_t st[8];
    or_ad_tile_stats(b, p, 1, st);
    uint8_t pos[16];
    int npos = 0;
    for (int sh = 60; sh >= 0; sh -= 4)
        if (((masked >> sh) & 0xF) == 0xF) pos[npos++] = (uint8_t)sh;
    const int8_t count = (int8_t)npos, free32k = (int8_t)p->num_free_32k;
    if (count == 0 || count == free32k) {
        if (cap) out[0] = b;
        return 1;
    }
    const uint32_t large = (uint32_t)original_sum - (uint32_t)st[0] -
                           ((uint32_t)(p->num_free_32k + p->num_fixed_32k) << 15);
    const uint8_t a = (uint8_t)(large >> 6), c = (uint8_t)(count - free32k);
    uint8_t tc[16];
    const int len = (a == 0 || c >= 10) ? 0 : ad_combination((uint32_t)a << 6, c, tc);
    if (len == 0) return 0;
    if (c < 1 || (int)c >= (int)(p->target & 0xFFu) - 4 || npos > 15) return 0;  /* no slot */
    ad_walk w = {b, pos, tc, npos, c, len, len > 1 && tc[0] == tc[1], out, cap, 0};
    int cell_of[16] = {0};
    ad_walk_cells(&w, 0, 0, 0, cell_of);
    return w.total;
}
