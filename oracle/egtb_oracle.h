/*
 * CPU oracle for the classic endgame-tablebase build and lookup path, and
 * for the advanced algorithm's masked-board primitives.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm (game-difficulty/2048EndgameTablebase, native_core/) used by the
 * tests, smoke() and bench.py's CPU-baseline leg as the CHECKER. The product
 * (2048endgametablebase_b200/) never links, imports or calls it.
 *
 * Every function cites the reference file:line it restates. Parity of this
 * restatement against the reference's own compiled code is pinned by
 * tests/test_oracle_golden.py and tests/test_oracle_ad.py (digests and
 * vectors produced by the reference itself, tests/golden/make_golden.py).
 */
#ifndef EGTB_ORACLE_H
#define EGTB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* success-rate dtypes, same set as native_core/include/FormationRuntime.h:15,243-255 */
enum { OR_U32 = 0, OR_U64 = 1, OR_F32 = 2, OR_F64 = 3, OR_1F32 = 4, OR_1F64 = 5 };

/* symmetry modes, native_core/include/FormationRuntime.h:13 */
enum {
    OR_SYM_IDENTITY = 0, OR_SYM_FULL = 1, OR_SYM_DIAGONAL = 2, OR_SYM_HORIZONTAL = 3,
    OR_SYM_MIN33 = 4, OR_SYM_MIN24 = 5, OR_SYM_MIN34 = 6
};

typedef struct {
    const uint64_t *masks;
    int n_masks;
    const uint8_t *shifts;
    int n_shifts;
    int symm_mode;
    int is_variant; /* 1: the variant boards' wall-merge mover */
} or_spec;

/* board primitives */
void or_move_all_dir(uint64_t b, uint64_t out[4]);
void or_move_all_dir_variant_batch(const uint64_t *b, size_t n, uint64_t *out4);
void or_row_tables_variant(uint16_t *left_xor, uint16_t *right_xor);
uint64_t or_apply_sym(uint64_t b, int idx);
uint64_t or_canonical(uint64_t b, int mode);
int or_is_pattern(uint64_t b, const or_spec *s);
int or_is_success(uint64_t b, int target, const or_spec *s);
void or_row_tables(uint16_t *left_xor, uint16_t *right_xor);

/* batch wrappers for tests */
void or_move_all_dir_batch(const uint64_t *b, size_t n, uint64_t *out4);
void or_canonical_batch(const uint64_t *b, size_t n, int mode, uint64_t *out);

/* the advanced algorithm's masked-board primitives (AdvancedMaskParam,
 * native_core/include/FormationRuntime.h:98-104) */
typedef struct {
    uint64_t pos_fixed_32k_mask;
    uint32_t small_tile_sum_limit, target, num_free_32k, num_fixed_32k;
} or_ad_param;
void or_ad_move_all_dir_batch(const uint64_t *b, size_t n, uint64_t *out4, uint8_t *flags4);
uint64_t or_ad_mask_board(uint64_t b, int threshold);
void or_ad_tile_stats(uint64_t b, const or_ad_param *p, int kind, int64_t out8[8]);
int or_ad_validate(uint64_t b, uint32_t original_sum, const or_ad_param *p);
size_t or_ad_unmask(uint64_t b, uint32_t original_sum, const or_ad_param *p, uint64_t *out, size_t cap);

/* full build, layer-resident */
typedef struct or_build or_build;
or_build *or_generate(const uint64_t *seeds, size_t n_seeds, const or_spec *spec,
                      int target, int steps, int docheck_step);
int or_num_layers(const or_build *b);
size_t or_layer_len(const or_build *b, int t);
const uint64_t *or_layer_keys(const or_build *b, int t);
/* backward solve over every layer; rates stored with the dtype's element size */
int or_solve(or_build *b, int dtype, double spawn_rate4);
const void *or_layer_rates(const or_build *b, int t);
void or_free(or_build *b);

/* expand one parent layer: the two raw candidate streams (unsorted, with repeats) */
size_t or_expand(const uint64_t *parents, size_t n, const or_spec *spec, int target, int do_check,
                 uint64_t *out1, uint64_t *out2, size_t cap, size_t *n2);

/* backward solve of one layer from its two successor layers (keys sorted,
 * rates dtype-typed); rates0 receives n0 dtype-typed values */
void or_solve_layer(const uint64_t *keys0, size_t n0, void *rates0,
                    const uint64_t *k1, const void *r1, size_t n1,
                    const uint64_t *k2, const void *r2, size_t n2,
                    const or_spec *spec, int target, int do_check, int dtype, double spawn_rate4);

#ifdef __cplusplus
}
#endif
#endif
