// Thin C-ABI shim over the reference's masked-board primitives of the
// advanced algorithm (namespace FormationAD), linked with the reference's
// own BoardMoverAD.cpp and BoardMaskerAD.cpp compiled where they lie. Test
// infrastructure only: the golden-vector script and the CPU tests call it.
//
//   m_move_all_dir              native_core/src/BoardMoverAD.cpp:171-178
//   mask_board                  native_core/src/BoardMaskerAD.cpp:112-121
//   tile_sum_and_32k_count      native_core/src/BoardMaskerAD.cpp:123-144
//   tile_sum_and_32k_count2     native_core/src/BoardMaskerAD.cpp:169-190
//   tile_sum_and_32k_count4     native_core/src/BoardMaskerAD.cpp:219-257
//   validate                    native_core/src/BoardMaskerAD.cpp:409-443
//   init_masker                 native_core/src/BoardMaskerAD.cpp:514-533

#include <cstddef>
#include <cstdint>
#include <vector>

#include "BoardMaskerAD.h"
#include "BoardMoverAD.h"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

AdvancedPatternSpec make_spec(uint32_t small_limit, uint32_t target, const uint8_t *fixed_shifts,
                                           size_t n_fixed, uint32_t num_free_32k) {
    AdvancedPatternSpec s;
    s.small_tile_sum_limit = small_limit;
    s.target = (uint8_t)target;
    s.num_free_32k = (uint8_t)num_free_32k;
    s.fixed_32k_shifts.assign(fixed_shifts, fixed_shifts + n_fixed);
    return s;
}

}  // namespace

REF_API void ref_ad_move_all_dir_batch(const uint64_t *boards, size_t n, uint64_t *out4, uint8_t *flags4) {
    for (size_t i = 0; i < n; ++i) {
        const auto m = FormationAD::m_move_all_dir(boards[i]);
        for (int d = 0; d < 4; ++d) {
            out4[4 * i + d] = m[d].board;
            flags4[4 * i + d] = m[d].mask_new_tile ? 1 : 0;
        }
    }
}

REF_API void ref_ad_mask_board_batch(const uint64_t *boards, size_t n, int threshold, uint64_t *out) {
    for (size_t i = 0; i < n; ++i) out[i] = FormationAD::mask_board(boards[i], threshold);
}

// kind 1: tile_sum_and_32k_count, 2: tile_sum_and_32k_count2, 4: tile_sum_and_32k_count4.
// out8 per board: total_sum, count_32k, pos_bitmap low, pos_bitmap high,
// pos_rank, merged_tile_found, merged_tile, is_success (the last four: kind 4).
REF_API void ref_ad_tile_stats_batch(const uint64_t *boards, size_t n, uint32_t small_limit, uint32_t target,
                                     const uint8_t *fixed_shifts, size_t n_fixed, uint32_t num_free_32k, int kind,
                                     int64_t *out8) {
    const auto param = FormationAD::build_mask_param(make_spec(small_limit, target, fixed_shifts, n_fixed, num_free_32k));
    for (size_t i = 0; i < n; ++i) {
        int64_t *o = out8 + 8 * i;
        for (int k = 0; k < 8; ++k) o[k] = 0;
        if (kind == 4) {
            const auto r = FormationAD::tile_sum_and_32k_count4(boards[i], param);
            o[0] = r.total_sum;
            o[1] = r.count_32k;
            o[2] = (int64_t)(r.pos_bitmap & 0xFFFFFFFFull);
            o[3] = (int64_t)(r.pos_bitmap >> 32);
            o[4] = r.pos_rank;
            o[5] = r.merged_tile_found;
            o[6] = r.merged_tile;
            o[7] = r.is_success ? 1 : 0;
        } else {
            const auto r = kind == 1 ? FormationAD::tile_sum_and_32k_count(boards[i], param)
                                     : FormationAD::tile_sum_and_32k_count2(boards[i], param);
            o[0] = r.total_sum;
            o[1] = r.count_32k;
            o[2] = (int64_t)(r.pos_bitmap & 0xFFFFFFFFull);
            o[3] = (int64_t)(r.pos_bitmap >> 32);
        }
    }
}

REF_API void ref_ad_validate_batch(const uint64_t *boards, size_t n, const uint32_t *original_sums,
                                   uint32_t small_limit, uint32_t target, const uint8_t *fixed_shifts, size_t n_fixed,
                                   uint32_t num_free_32k, uint8_t *out) {
    const auto ctx = FormationAD::init_masker(make_spec(small_limit, target, fixed_shifts, n_fixed, num_free_32k));
    for (size_t i = 0; i < n; ++i)
        out[i] = FormationAD::validate(boards[i], original_sums[i], ctx.tiles_combination_table, ctx.param) ? 1 : 0;
}

// The tiles-combination table of init_masker: entry (a, b) = a + 256 b,
// a in 1..255, b in 1..9; lens[e] entries of at most 16 values in vals[16 e].
REF_API void ref_ad_tiles_combinations(uint8_t *lens, uint8_t *vals) {
    const auto ctx = FormationAD::init_masker(make_spec(96, 10, nullptr, 0, 0));
    for (size_t e = 0; e < ctx.tiles_combination_table.size(); ++e) {
        const auto &v = ctx.tiles_combination_table[e];
        lens[e] = (uint8_t)v.size();
        for (size_t j = 0; j < v.size() && j < 16; ++j) vals[16 * e + j] = v[j];
    }
}

// unmask_board (native_core/src/BoardMaskerAD.cpp:445-512) with init_masker's
// tables: counts[i] boards for boards[i], packed in order into out (room for
// cap); returns the total (boards past cap are counted, not written).
REF_API size_t ref_ad_unmask_batch(const uint64_t *boards, size_t n, const uint32_t *original_sums,
                                   uint32_t small_limit, uint32_t target, const uint8_t *fixed_shifts, size_t n_fixed,
                                   uint32_t num_free_32k, uint32_t *counts, uint64_t *out, size_t cap) {
    const auto ctx = FormationAD::init_masker(make_spec(small_limit, target, fixed_shifts, n_fixed, num_free_32k));
    size_t total = 0;
    std::vector<uint64_t> got;
    for (size_t i = 0; i < n; ++i) {
        FormationAD::unmask_board_into(boards[i], original_sums[i], ctx.tiles_combination_table,
                                       ctx.permutation_table, ctx.param, got);
        counts[i] = (uint32_t)got.size();
        for (uint64_t b : got) {
            if (total < cap) out[total] = b;
            ++total;
        }
    }
    return total;
}
