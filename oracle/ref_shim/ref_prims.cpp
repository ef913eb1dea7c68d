// Thin C-ABI shim over the reference's board primitives, compiled from the
// reference headers where they lie (native_core/include). Test
// infrastructure only: it exposes the reference's own move tables and
// symmetry functions to the parity tests and to the golden-vector script.
//
//   move_all_dir      native_core/include/CommonMover.h:136-139 (classic
//                     BoardMover and the variant VBoardMover,
//                     native_core/include/VBoardMover.h)
//   row tables        native_core/include/CommonMover.h:87-94,
//                     native_core/include/BoardMover.h:6-55
//   canonical_by_mode native_core/include/SymmetryUtils.h:31-49
//   apply_sym_like    native_core/include/SymmetryUtils.h:9-29
//   is_pattern        native_core/include/Formation.h:11-17

#include <cstddef>
#include <cstdint>
#include <vector>

#include "BoardMover.h"
#include "VBoardMover.h"
#include "Formation.h"
#include "SymmetryUtils.h"

extern "C" {

void ref_move_all_dir_batch(const uint64_t *boards, size_t n, uint64_t *out4) {
    for (size_t i = 0; i < n; ++i) {
        auto m = BoardMover::move_all_dir(boards[i]);
        out4[4 * i + 0] = std::get<0>(m);
        out4[4 * i + 1] = std::get<1>(m);
        out4[4 * i + 2] = std::get<2>(m);
        out4[4 * i + 3] = std::get<3>(m);
    }
}

void ref_canonical_batch(const uint64_t *boards, size_t n, int symm_mode, uint64_t *out) {
    for (size_t i = 0; i < n; ++i) {
        out[i] = canonical_by_mode(boards[i], symm_mode);
    }
}

void ref_apply_sym_batch(const uint64_t *boards, size_t n, int symm_index, uint64_t *out) {
    for (size_t i = 0; i < n; ++i) {
        out[i] = apply_sym_like(boards[i], symm_index);
    }
}

void ref_is_pattern_batch(const uint64_t *boards, size_t n, const uint64_t *masks, size_t n_masks, uint8_t *out) {
    std::vector<uint64_t> m(masks, masks + n_masks);
    for (size_t i = 0; i < n; ++i) {
        out[i] = is_pattern(boards[i], m) ? 1 : 0;
    }
}

void ref_row_tables(uint16_t *left_xor, uint16_t *right_xor) {
    for (uint32_t r = 0; r < 65536; ++r) {
        left_xor[r] = BoardMover::row_move_table[r].movel;
        right_xor[r] = BoardMover::row_move_table[r].mover;
    }
}

void ref_move_all_dir_variant_batch(const uint64_t *boards, size_t n, uint64_t *out4) {
    for (size_t i = 0; i < n; ++i) {
        auto m = VBoardMover::move_all_dir(boards[i]);
        out4[4 * i + 0] = std::get<0>(m);
        out4[4 * i + 1] = std::get<1>(m);
        out4[4 * i + 2] = std::get<2>(m);
        out4[4 * i + 3] = std::get<3>(m);
    }
}

void ref_row_tables_variant(uint16_t *left_xor, uint16_t *right_xor) {
    for (uint32_t r = 0; r < 65536; ++r) {
        left_xor[r] = VBoardMover::row_move_table[r].movel;
        right_xor[r] = VBoardMover::row_move_table[r].mover;
    }
}

}  // extern "C"
