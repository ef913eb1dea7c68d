/*
 * egtb_gpu.h — C ABI of libegtb_gpu.so, the B200 (sm_100a) implementation of
 * the classic endgame-tablebase table build and book lookup of
 * game-difficulty/2048EndgameTablebase.
 *
 * Plain C: fixed-size structs, pointers and sizes, int status codes. No
 * CUDA, C++ or torch types cross this boundary. Every entry point returns
 * EGTB_OK (0) or a negative EGTB_ERR_* code; egtb_last_error() gives the
 * message of the calling thread's last failure.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the reference project). The reference binds these from Python through
 * nanobind (native_core/src/bindings_formation.cpp:46-241); this library is
 * bound through ctypes by 2048endgametablebase_b200/native_core/formation_core.py.
 *
 * Threading: build entry points may run on any host thread; progress may be
 * read from another thread while a build runs (relaxed atomics, as
 * native_core/include/FormationRuntime.h:44-86). One device context is kept
 * per device; builds on the same device are serialised inside the library.
 */
#ifndef EGTB_GPU_H
#define EGTB_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define EGTB_API __attribute__((visibility("default")))
#else
#define EGTB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status ---- */
#define EGTB_OK 0
#define EGTB_ERR_ARG (-1)          /* invalid argument */
#define EGTB_ERR_CUDA (-2)         /* CUDA runtime error (no device, launch failure, ...) */
#define EGTB_ERR_NOMEM (-3)        /* device or pinned-host allocation failed */
#define EGTB_ERR_IO (-4)           /* file read/write failed */
#define EGTB_ERR_CAPACITY (-5)     /* a layer outgrew the largest buffer the device can hold */
#define EGTB_ERR_TIMEOUT (-6)      /* a bounded device wait gave up */
#define EGTB_ERR_UNSUPPORTED (-7)  /* option outside the implemented path */

/* ------------------------------------------------------------ types ----- */

/* SymmMode, native_core/include/FormationRuntime.h:13 */
enum egtb_symm_mode {
    EGTB_SYMM_IDENTITY = 0,
    EGTB_SYMM_FULL = 1,
    EGTB_SYMM_DIAGONAL = 2,
    EGTB_SYMM_HORIZONTAL = 3,
    EGTB_SYMM_MIN33 = 4,
    EGTB_SYMM_MIN24 = 5,
    EGTB_SYMM_MIN34 = 6
};

/* success_rate_dtype names, native_core/include/FormationRuntime.h:243-255 */
enum egtb_dtype {
    EGTB_DTYPE_UINT32 = 0,
    EGTB_DTYPE_UINT64 = 1,
    EGTB_DTYPE_FLOAT32 = 2,
    EGTB_DTYPE_FLOAT64 = 3,
    EGTB_DTYPE_1_FLOAT32 = 4, /* stores success - 1 */
    EGTB_DTYPE_1_FLOAT64 = 5
};

#define EGTB_MAX_MASKS 32
#define EGTB_MAX_PATH 4096

/* PatternSpec, native_core/include/FormationRuntime.h:17-22 */
typedef struct egtb_pattern_spec {
    char name[64];
    uint64_t pattern_masks[EGTB_MAX_MASKS];
    int32_t n_masks;
    uint8_t success_shifts[16];
    int32_t n_shifts;
    int32_t symm_mode; /* enum egtb_symm_mode */
} egtb_pattern_spec;

/* RunOptions, native_core/include/FormationRuntime.h:24-42, plus device fields */
typedef struct egtb_run_options {
    int32_t target;       /* log2 of the target tile */
    int32_t steps;
    int32_t docheck_step;
    char pathname[EGTB_MAX_PATH]; /* file prefix: layer t is <pathname><t>, book <pathname><t>.book */
    int32_t is_free;
    int32_t is_variant;
    double spawn_rate4;
    int32_t success_rate_dtype; /* enum egtb_dtype */
    double deletion_threshold;
    int32_t compress;     /* books of layer 3+ over 2 MiB -> <pathname><t>.z trie + xz directories (needs write_files) */
    int32_t compress_temp_files;
    int32_t optimal_branch_only;
    int32_t chunked_solve;
    int32_t num_threads;  /* host threads for file writing (0 = library default) */
    int32_t direct_io;
    int32_t direct_io_queue_depth;
    int32_t direct_io_chunk_mib;
    /* device fields (no reference counterpart) */
    int32_t device;       /* CUDA device ordinal */
    int32_t write_files;  /* egtb_build only: 0 keeps the books on the device (benchmarks) */
} egtb_run_options;

/* Per-build record filled by egtb_build / egtb_generate (no reference counterpart:
 * the reference logs the same quantities through Config.logger). */
typedef struct egtb_build_stats {
    uint64_t raw_boards;       /* sum of raw layer sizes */
    uint64_t book_entries;     /* sum of .book sizes (zero rates dropped) */
    uint64_t max_layer;        /* largest raw layer */
    uint64_t candidates;       /* children that reached the sort (after the device filter) */
    uint64_t lookups;          /* exact searches done by the backward pass */
    int32_t layers;            /* steps */
    int32_t retries;           /* capacity regrowths */
    double forward_ms;         /* device time */
    double backward_ms;        /* device time */
    double total_ms;           /* host wall time of the call */
    uint64_t kernel_launches;  /* kernels this call launched */
} egtb_build_stats;

/* Accumulated device time of one kind of kernel (egtb_profile_read). */
typedef struct egtb_kernel_time {
    char name[32];
    uint64_t launches;   /* timed units (one unit may be a short chain of kernels) */
    double total_ms;
} egtb_kernel_time;

/* ------------------------------------------------------------ errors ---- */

/* Message of the calling thread's last failure (empty when none). */
EGTB_API int egtb_last_error(char *buf, size_t len);

/* Library version string, e.g. "egtb_gpu 0.1 sm_100a". */
EGTB_API const char *egtb_version(void);

/* Number of visible CUDA devices (0 when none). */
EGTB_API int egtb_device_count(void);

/* Use the caller's CUDA stream (a cudaStream_t passed as void*) for all
 * device work of this device; NULL returns to the library's own stream.
 * No reference counterpart: lets a host framework order builds on its own
 * stream and time them with its own events. */
EGTB_API int egtb_set_stream(int device, void *stream);

/* Per-kernel-kind device timing with CUDA events on the launching stream
 * (no reference counterpart; the reference logs phase fractions through
 * Config.logger, BookGenerator.cpp:129-146). egtb_profile(device, 1) clears
 * and enables it; egtb_profile_read fills up to max_kinds entries. The layer
 * loops of the forward expand and of the solve are timed as one run each
 * (two events per loop, the gaps between their launches included, launches =
 * the loop's kernel count); other kinds one event pair per launch. */
EGTB_API int egtb_profile(int device, int enable);
EGTB_API int egtb_profile_read(int device, egtb_kernel_time *out, int max_kinds, int *n_kinds);

/* Free the device (and pinned host) memory the library keeps on `device`
 * between builds: the layer arena, sets, rate indexes, sort buffers and the
 * books of the last egtb_build / egtb_build_batch (egtb_book_layer_copy and
 * egtb_batch_book_copy have nothing to copy afterwards). Buffers grow to the
 * largest table built and stay for the next build otherwise. Open books and
 * servers keep theirs. No reference counterpart (the reference's buffers
 * live for one call); for long-lived processes that build tables of very
 * different sizes. */
EGTB_API int egtb_release(int32_t device);

/* Number of polls a bounded device wait (the sort's look-back on another
 * block's counts) makes before it gives up; 0 restores the default 2^22.
 * Process-wide, read at each launch. A wait that gives up makes the call
 * return EGTB_ERR_TIMEOUT (egtb_build, egtb_generate, egtb_solve,
 * egtb_build_batch) instead of hanging; the library stays usable. No
 * reference counterpart (the reference's CPU sort has no cross-block waits);
 * meant for tests of the timeout path and for callers that want a shorter
 * bound. */
EGTB_API int egtb_set_spin_limit(uint32_t polls);

/* ---------------------------------------------------------- progress ---- */

/* get_build_progress / reset_build_progress,
 * native_core/src/bindings_formation.cpp:140-155, FormationRuntime.h:57-84 */
EGTB_API int egtb_get_build_progress(uint32_t *current, uint32_t *total);
EGTB_API int egtb_reset_build_progress(uint32_t total);

/* ------------------------------------------------------------ build ----- */

/* run_pattern_build, native_core/src/BookSolver.cpp:823-832 (bound at
 * bindings_formation.cpp:220-229): forward layer generation then backward
 * solve, writing <pathname><t>.book for every layer and <pathname>stats.txt.
 * With no layer files present the whole build stays in device memory and
 * only books are written; with layer files present it resumes through
 * egtb_generate + egtb_solve like the reference. stats may be NULL. */
EGTB_API int egtb_build(const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec *spec,
               const egtb_run_options *options, egtb_build_stats *stats);

/* run_pattern_generate, native_core/src/BookSolver.cpp:766-782 (bound at
 * bindings_formation.cpp:200-208): writes raw layers <pathname>0 ..
 * <pathname><steps-3> and the success-only books of layers steps-2 and
 * steps-1 (final_steps, BookSolver.cpp:263-284). *started is 0 when every
 * step was already on disk. */
EGTB_API int egtb_generate(const uint64_t *seeds, size_t n_seeds, const egtb_pattern_spec *spec,
                  const egtb_run_options *options, int32_t *started, egtb_build_stats *stats);

/* run_pattern_solve, native_core/src/BookSolver.cpp:784-821 (bound at
 * bindings_formation.cpp:210-218): backward pass from the raw layer files.
 * d1/d2 are the packed book records of layers steps-2 and steps-1 (n1/n2
 * records; may be empty, then they are read from their .book files). */
EGTB_API int egtb_solve(const void *d1_records, size_t n1, const void *d2_records, size_t n2,
               const egtb_pattern_spec *spec, const egtb_run_options *options, egtb_build_stats *stats);

/* Copy the .book records of one layer of the last egtb_build on this device
 * (write_files = 0 keeps them in device memory) into dst; *bytes receives
 * their size (dst = NULL: size only). No reference counterpart: the
 * reference only writes books to files (write_layer_file,
 * native_core/src/BookSolver.cpp:206-231); the bytes are the same. */
EGTB_API int egtb_book_layer_copy(int device, int32_t layer, void *dst, size_t dst_bytes, uint64_t *bytes);

/* ------------------------------------------------------- primitives ----- */

/* Batched board primitives on the device, host buffers in and out
 * (move_all_dir native_core/include/CommonMover.h:136-139; canonical_by_mode
 * SymmetryUtils.h:31-49; apply_sym_like SymmetryUtils.h:9-29). */
EGTB_API int egtb_move_all_dir(int device, const uint64_t *boards, size_t n, uint64_t *out4);
/* move_all_dir of the variant boards' mover (VBoardMover,
 * native_core/include/VBoardMover.h:79 over CommonMover.h:136-139): 0xF cells
 * are walls, tiles slide and merge between them. */
EGTB_API int egtb_move_all_dir_variant(int device, const uint64_t *boards, size_t n, uint64_t *out4);
/* symm_mode 0-6: identity, full, diagonal, horizontal, min33, min24, min34. */
EGTB_API int egtb_canonical(int device, const uint64_t *boards, size_t n, int32_t symm_mode, uint64_t *out);
EGTB_API int egtb_apply_sym(int device, const uint64_t *boards, size_t n, int32_t symm_index, uint64_t *out);

/* ------------------------- masked-board primitives (advanced algorithm) --- */

/* The masked boards of the reference's advanced algorithm (namespace
 * FormationAD): tiles of 64 and up are held as 0xF ("32k") nibbles.
 * AdvancedMaskParam, native_core/include/FormationRuntime.h:98-104. */
typedef struct egtb_ad_param {
    uint64_t pos_fixed_32k_mask;   /* 0xF nibbles at the pattern's fixed 32k cells */
    uint32_t small_tile_sum_limit; /* default 96 */
    uint32_t target;               /* log2 of the target tile */
    uint32_t num_free_32k;
    uint32_t num_fixed_32k;
} egtb_ad_param;

/* TileCountResult / TileCount4Result, native_core/include/BoardMaskerAD.h:51-79. */
typedef struct egtb_ad_tile_count {
    uint64_t pos_bitmap;        /* 0xF at every cell counted as 32k */
    uint32_t total_sum;         /* sum of the other tiles */
    int32_t count_32k;
    uint32_t pos_rank;          /* kind 4 only: 32k cells before the first merged tile */
    uint32_t merged_tile_found; /* kind 4: large tiles that are not 0xF */
    uint32_t merged_tile;       /* kind 4: xor of those tiles */
    uint32_t is_success;        /* kind 4: one merged tile, equal to the target */
} egtb_ad_tile_count;

/* Masked mover, batched (host buffers): out4[4i..4i+3] = left, right, up,
 * down of boards[i]; flags4 likewise = 1 where a merge made a tile of 64 or
 * more, which the masked board holds as 0xF (mask_new_tile; left and right
 * report the left merge's flag, up and down the up merge's). 0xF never
 * merges. m_move_all_dir, native_core/src/BoardMoverAD.cpp:171-178, rows by
 * merge_line, :49-89. */
EGTB_API int egtb_ad_move_all_dir(int device, const uint64_t *boards, size_t n, uint64_t *out4, uint8_t *flags4);
/* mask_board, native_core/src/BoardMaskerAD.cpp:112-121: every nibble >=
 * threshold becomes 0xF (the reference's default threshold is 6). */
EGTB_API int egtb_ad_mask_board(int device, const uint64_t *boards, size_t n, int32_t threshold, uint64_t *out);
/* Tile statistics after clearing the fixed 32k cells: kind 1 counts only 0xF
 * as 32k (tile_sum_and_32k_count, BoardMaskerAD.cpp:123-144), kind 2 counts
 * every tile of 64 and up (tile_sum_and_32k_count2, :169-190), kind 4 is kind
 * 2 plus the merged-tile fields (tile_sum_and_32k_count4, :219-257). */
EGTB_API int egtb_ad_tile_stats(int device, const uint64_t *boards, size_t n, const egtb_ad_param *param,
                                int32_t kind, egtb_ad_tile_count *out);
/* validate, native_core/src/BoardMaskerAD.cpp:409-443: out[i] = 1 when
 * boards[i] (tile sum original_sums[i] before masking) can stand for a real
 * board of the pattern. The reference reads its tiles-combination table at
 * (count_32k - num_free_32k) < 10 only; boards past that give 0 here. */
EGTB_API int egtb_ad_validate(int device, const uint64_t *boards, size_t n, const uint32_t *original_sums,
                              const egtb_ad_param *param, uint8_t *out);
/* unmask_board, native_core/src/BoardMaskerAD.cpp:445-512 (tables of
 * init_masker, :514-533): every board that masked board boards[i] (tile sum
 * original_sums[i] before masking) stands for, in the reference's order:
 * counts[i] of them, all boards' packed one after another into out (room for
 * cap). *total = their sum; above cap the call fails with EGTB_ERR_CAPACITY
 * after filling counts and *total, so the caller can size out and call again.
 * Boards whose 32k count is below num_free_32k or 10 or more above it (where
 * the reference reads past its tables) give none. */
EGTB_API int egtb_ad_unmask(int device, const uint64_t *boards, size_t n, const uint32_t *original_sums,
                            const egtb_ad_param *param, uint32_t *counts, uint64_t *out, size_t cap,
                            uint64_t *total);
/* The host tables behind the kernels above (no device needed): the masked row
 * moves (moves[r] = left xor | right xor << 16, flags[r] = mask_new_tile of
 * the left merge; BoardMoverAD.cpp:27-45) and the tiles-combination table of
 * init_masker (BoardMaskerAD.cpp:524-531: entry a + 256 b, a < 256, b < 10;
 * lens[e] values in vals16[16 e ..]). */
EGTB_API int egtb_ad_row_tables(uint32_t *moves, uint8_t *flags);
EGTB_API int egtb_ad_tiles_combinations(uint8_t *lens, uint8_t *vals16);

/* Sort the n keys at d_keys (device memory) ascending, drop repeats, write
 * the unique keys to d_out (device, room for n keys, must not alias d_keys)
 * and their count to *d_n_out (device). Enqueued on `stream`
 * (cudaStream_t as void*, NULL = legacy default stream); scratch is taken
 * and returned stream-ordered. The device counterpart of the reference's
 * sort/unique plug-in seam (sort_uint64, native_core/xss_wrapper.cpp:14-31;
 * unique_sorted_u64_inplace, native_core/src/unique_wrapper.cpp:12-14). */
EGTB_API int egtb_sort_unique_u64(int device, const uint64_t *d_keys, size_t n, uint64_t *d_out,
                                  uint64_t *d_n_out, void *stream);

/* egtb_sort_unique_u64 for callers that cannot have the library allocate
 * device memory (their pool holds all of it, or cudaMalloc/cudaFree would
 * stall a latency-critical path). No counterpart in the reference. Same
 * arguments and result; n <= 1048576 keys (larger n: EGTB_ERR_ARG). Its
 * scratch is a static device array of about 8.6 MB that every GPU loading
 * the library holds until exit; the first call on a device looks up that
 * array's address, so make the first call before any stream capture. All
 * calls share the array: calls that overlap on the GPU race. The address is
 * kept for the life of the process: after a cudaDeviceReset of a device
 * (which unloads the library's device code there) do not call this entry
 * point on that device again. */
EGTB_API int egtb_sort_unique_u64_noalloc(int device, const uint64_t *d_keys, size_t n, uint64_t *d_out,
                                          uint64_t *d_n_out, void *stream);

/* ------------------------------------------------------------ books ----- */

typedef struct egtb_book egtb_book;

/* Open the books <dir>/<pattern_full>_<t>.book of one table and keep them
 * resident in device memory as sorted keys + rates (the reader side of
 * ClassicBookReader, native_core/src/ReaderRuntime.cpp:1050-1067).
 * nums_adjust is the pattern's -(seed tile sum) (Config.py:265). Layers
 * are loaded on first use; max_layers bounds the layer index scanned. A
 * layer without a .book file is read from its compressed directory
 * <pattern_full>_<t>.z when there is one (trie + xz blocks,
 * TrieCompression.cpp:326-354): its blocks are decoded on the host and
 * searched on the device as trie_search_with_context does
 * (ReaderRuntime.cpp:318-477). */
EGTB_API int egtb_book_open(const char *dir, const char *pattern_full, int32_t dtype, const egtb_pattern_spec *spec,
                   int64_t nums_adjust, int32_t device, egtb_book **out);
EGTB_API int egtb_book_close(egtb_book *book);

/* Mark the book as one of variant boards (ClassicBookReader(spec, is_variant),
 * native_core/src/ReaderRuntime.cpp:1050-1067): its lookups move with the
 * wall-merge rule (VBoardMover, native_core/include/VBoardMover.h) and try
 * the board as given only (operation_sequence, ReaderRuntime.cpp:171-182),
 * whatever last_op says. */
EGTB_API int egtb_book_set_variant(egtb_book *book, int32_t is_variant);

/* Load every book layer of the table now (otherwise loaded on first lookup). */
EGTB_API int egtb_book_load_all(egtb_book *book, int32_t *layers_loaded);

/* Batched move_on_dic on encoded positions (encode_board_matrix,
 * native_core/include/BoardCodec.h:20-30), host buffers, op order
 * [last_op, 0..7] as evaluate_classic_result_candidates
 * (ReaderRuntime.cpp:739-840). Per position writes 4 values in direction
 * order up, right, down, left (kDirectionNames, ReaderRuntime.cpp:32) already
 * normalised and rounded like maybe_round_value (:208-214), a validity mask
 * (bit d set when direction d has a numeric value) and the operation index
 * that matched (-1 when none; -2 when the layer index is negative; -3 when
 * the layer's book file does not exist). */
EGTB_API int egtb_book_lookup(egtb_book *book, const uint64_t *positions, size_t n, int32_t last_op,
                     double *values4, uint8_t *valid_mask, int8_t *op_used);

/* Same on device memory and a caller stream (cudaStream_t passed as void*),
 * float32 values; used by the serving loop. Layers must be loaded. */
EGTB_API int egtb_book_lookup_device(egtb_book *book, const uint64_t *d_positions, size_t n, int32_t last_op,
                            float *d_values4, uint8_t *d_valid_mask, void *stream);

/* find_classic_value, native_core/src/ReaderRuntime.cpp:1107-1133 (bound at
 * bindings_formation.cpp:180-194): the normalised value of one key in one
 * book file; *found = 0 when the file does not exist (value 0 then). */
EGTB_API int egtb_find_classic_value(const char *pathname, const char *filename, uint64_t key, int32_t dtype,
                            int32_t device, double *value, int32_t *found);

/* ---- batched build -----------------------------------------------------
 * Many tables of uneven size built together: no counterpart in the
 * reference, which builds one table per run_pattern_build call
 * (native_core/src/BookSolver.cpp:823-832; engine_core/BookBuilder.py:264).
 * Every table gives the same inputs as egtb_build (seeds, spec, options) and
 * gets the same books, byte for byte; all tables advance one global layer
 * step per kernel launch (forward: expand + dedup of layer t of every table;
 * backward: solve + rate index of layer t of every table), the per-step
 * loops replayed as CUDA graphs, one radix sort pass at a time over every
 * table's layers, each layer in its own region. */
typedef struct egtb_batch_params {
    int32_t expand_chunk;         /* parents per work item of the forward step: multiple of 32 in 32..4096 (0: tuned, else 128) */
    int32_t expand_blocks_per_sm; /* blocks per SM of the forward step, 1..8 (0: tuned, else 3) */
    int32_t digit_nibbles;        /* radix digit of the layer sort in nibbles, 1 or 2 (0: tuned, else 2) */
    int32_t index_load;           /* rate-index slots per key of a table's largest layer, 2 or 4 (0: tuned, else 2) */
    int32_t use_graphs;           /* 1: per-step loops replayed as CUDA graphs, -1: direct launches (0: tuned, else 1) */
    int32_t reserved[3];
} egtb_batch_params;

typedef struct egtb_batch_stats {
    uint64_t raw_boards;      /* all tables, as egtb_build_stats */
    uint64_t book_entries;
    uint64_t candidates;
    uint64_t lookups;
    int32_t tables;
    int32_t max_steps;        /* global layer steps */
    int32_t retries;          /* forward re-runs after capacity regrowth */
    int32_t graphs_used;      /* 1 when the per-step loops ran as CUDA graphs */
    double forward_ms;        /* device time of the phases */
    double sort_ms;
    double backward_ms;
    double pack_ms;
    double total_ms;          /* host wall time of the call */
    uint64_t kernel_launches; /* kernels run (graph nodes counted one by one) */
    uint64_t graph_launches;
    egtb_batch_params params; /* the parameters used */
} egtb_batch_stats;

/* Build n_tables tables on options[0].device (all tables: same device and
 * success_rate_dtype). Table i: seeds[i][0..n_seeds[i]), specs[i],
 * options[i] (write_files per table). params may be NULL (tuned values for
 * this set of tables when egtb_batch_autotune ran, else defaults).
 * table_stats (n_tables entries) and stats may be NULL. The books of the last
 * batch stay on the device for egtb_batch_book_copy. */
EGTB_API int egtb_build_batch(int32_t n_tables, const uint64_t *const *seeds, const uint64_t *n_seeds,
                              const egtb_pattern_spec *specs, const egtb_run_options *options,
                              const egtb_batch_params *params, egtb_build_stats *table_stats, egtb_batch_stats *stats);

/* Autotuner: builds the batch (books kept on the device) under candidate
 * parameters, one parameter at a time (forward work-item size and blocks per
 * SM, radix digit width, rate-index load), keeps the fastest by device time,
 * remembers it for this set of tables and returns it in *best (*best_ms: its
 * device time). */
EGTB_API int egtb_batch_autotune(int32_t n_tables, const uint64_t *const *seeds, const uint64_t *n_seeds,
                                 const egtb_pattern_spec *specs, const egtb_run_options *options,
                                 egtb_batch_params *best, double *best_ms);

/* Copy book layer `layer` of table `table` of the device's last batch (packed
 * records) to host memory; *bytes = its size (dst may be NULL to ask). */
EGTB_API int egtb_batch_book_copy(int device, int32_t table, int32_t layer, void *dst, size_t dst_bytes,
                                  size_t *bytes);

/* ---- serving loop ------------------------------------------------------
 * Answers move_on_dic queries (last_op 0) against books resident in device
 * memory, for many concurrent clients. No counterpart in the reference,
 * which answers one position per Python call from files
 * (ClassicBookReader.move_on_dic, native_core/src/ReaderRuntime.cpp:1050-1067;
 * engine_core/BookReader.py:96-118); each answer equals that call's answer
 * as float32 (egtb_book_lookup_device).
 *
 * A scheduler thread batches queued requests into `slots` in-flight batches
 * (one CUDA stream, pinned buffers and device buffers of slot_positions
 * positions each): a free slot takes queued requests in arrival order while
 * they fit (continuous batching; admission by slot memory), so batches
 * overlap on the GPU and a request waits for a running batch only when every
 * slot is busy. max_requests_per_batch > 0 caps requests per batch (1 = one
 * request per launch). Books must be loaded (egtb_book_load_all) and stay
 * open while the server runs. */
typedef struct egtb_server egtb_server;

EGTB_API int egtb_serve_start(egtb_book *const *books, int32_t n_books, int32_t slots, uint64_t slot_positions,
                              int32_t max_requests_per_batch, egtb_server **out);

/* Queue one request of n (1..slot_positions) positions for books[book];
 * positions, values4 (4 floats per position) and valid_mask (may be NULL)
 * must stay valid until egtb_serve_wait returns for the ticket. */
EGTB_API int egtb_serve_submit(egtb_server *server, int32_t book, const uint64_t *positions, uint64_t n,
                               float *values4, uint8_t *valid_mask, uint64_t *ticket);

/* Register caller memory with the server (page-locked and mapped into the
 * device's address space until egtb_serve_unregister or egtb_serve_stop). A
 * request whose positions, values4 and valid_mask all lie in registered
 * memory is answered in place: the lookup kernel reads its positions and
 * writes its answers there, with no staging copy on the host.
 * egtb_serve_replay registers its own buffers. */
EGTB_API int egtb_serve_register(egtb_server *server, void *ptr, uint64_t bytes);
/* Refused (EGTB_ERR_ARG) while a request answered in place that is not done
 * yet (queued or on the GPU) has its positions, values4 or valid_mask in the
 * range: the GPU still reads or writes it there. */
EGTB_API int egtb_serve_unregister(egtb_server *server, void *ptr);

/* Wait for a ticket (timeout_ms < 0: one hour); *latency_us = submit to
 * answer. Every ticket must be waited for once. On EGTB_ERR_TIMEOUT the
 * request is still live and its buffers stay in use until it is answered:
 * wait for the ticket again before freeing or unregistering them. */
EGTB_API int egtb_serve_wait(egtb_server *server, uint64_t ticket, int32_t timeout_ms, double *latency_us);

EGTB_API int egtb_serve_stats(egtb_server *server, uint64_t *requests, uint64_t *positions, uint64_t *batches,
                              uint64_t *launches);

/* Replay a recorded request stream: request i arrives arrival_us[i]
 * microseconds after the call, reads sizes[i] positions at pool + offsets[i]
 * for books[book_of[i]] and answers into values4 + 4*offsets[i] and
 * valid + offsets[i] (valid may be NULL); latency_us[i] gets its latency,
 * measured from its scheduled arrival (time the submitting thread fell
 * behind the schedule counts as queueing), and *wall_us the time until the
 * last answer. On a timeout the replay stops submitting and waits (bounded)
 * for what it submitted; buffers of requests still unanswered stay
 * registered (the GPU may still write them). */
EGTB_API int egtb_serve_replay(egtb_server *server, const uint64_t *pool, const double *arrival_us,
                               const uint32_t *sizes, const uint64_t *offsets, const int32_t *book_of, uint64_t n_req,
                               float *values4, uint8_t *valid, double *latency_us, double *wall_us);

/* Stop the scheduler and free the slots (books stay open). */
EGTB_API int egtb_serve_stop(egtb_server *server);

#ifdef __cplusplus
}
#endif
#endif /* EGTB_GPU_H */
