// Host-side helpers of libegtb_gpu: error state, CUDA checking, file I/O,
// row tables, pattern conversion. Shared by the build and book modules.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/egtb_gpu.h"
#include "egtb_device.cuh"

namespace egtb {

// Exception carrying an EGTB_ERR_* status; caught at the C boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &msg);
void clear_last_error();

#define EGTB_CUDA(call)                                                                              \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            throw ::egtb::Error(e_ == cudaErrorMemoryAllocation ? EGTB_ERR_NOMEM : EGTB_ERR_CUDA,     \
                                std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

// Run f and translate exceptions into a status code + thread-local message.
template <typename F>
int guarded(F &&f) {
    try {
        clear_last_error();
        f();
        return EGTB_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return EGTB_ERR_NOMEM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return EGTB_ERR_IO;
    }
}

// Row-move XOR delta table (low 16 bits toward column 0, high 16 toward
// column 3) from the classic merge rule (native_core/include/BoardMover.h:6-55)
// or, with variant, the wall-merge rule of the variant boards
// (native_core/include/VBoardMover.h:7-76).
const std::vector<uint32_t> &host_row_tables(bool variant = false);

// Device copy of a row table on the current device (created once per device).
const uint32_t *device_row_table(bool variant = false);

DevSpec make_dev_spec(const egtb_pattern_spec &s, int target);

size_t dtype_size(int dtype);
bool dtype_is_one_minus(int dtype);
double dtype_zero(int dtype);
double dtype_max(int dtype);
std::string dtype_name(int dtype);

// Files
bool file_valid(const std::string &path, uint64_t alignment);
void remove_invalid(const std::string &path, uint64_t alignment);
bool file_exists(const std::string &path);
uint64_t file_size(const std::string &path);
void write_file(const std::string &path, const void *data, size_t bytes);   // via <path>.tmp + rename
std::vector<unsigned char> read_file(const std::string &path);
void read_file_into(const std::string &path, void *dst, size_t bytes);
void remove_file(const std::string &path);
std::string parent_dir(const std::string &path);
std::string now_string();
double round_to_2(double v);

// Polls a sort look-back wait makes before it gives up (egtb_set_spin_limit;
// process-wide, read at every launch).
unsigned look_back_spin_limit();

// Byte size of SuccessEntry<T> records, native_core/include/FormationRuntime.h:191-205.
inline size_t record_size(int dtype) { return 8 + dtype_size(dtype); }

// The per-device build engine (egtb_build.cu) as the batched build sees it:
// its lock (builds on one device run one at a time), the stream in use, the
// row table and the SM count.
struct EngineRef {
    std::mutex *mu;
    int device;
    cudaStream_t *stream;
    const uint32_t *tab;
    int sm_count;
    int sweep_grid;
    int seg_grid;  // resident blocks of the per-layer onesweep kernel (kSegSweepSmem of shared memory each)
};
EngineRef engine_ref(int device);
// Free the batched build's buffers on a device (egtb_release; the caller holds the build lock).
void batch_release_buffers(int device);
// Nibbles that are 0xF in every canonical key of the pattern.
uint64_t pattern_pinned_nibbles(const egtb_pattern_spec &s);
// Build progress (get_build_progress): the mapped word kernels write, and the host setter.
unsigned *build_progress_ptr();
void build_progress_set(uint32_t cur, uint32_t total);
// stats.txt lines (ensure_stats_header + recalculate_process_impl,
// native_core/src/BookSolver.cpp:286-293,569-581).
void write_stats_file(const egtb_run_options &o, int dtype, const std::vector<int> &layers,
                      const std::vector<unsigned long long> &raw_len, const std::vector<unsigned long long> &book_len,
                      const std::vector<unsigned long long> &maxbits, double seconds_per_layer);

// One request of the serving loop for the request-list lookup kernel: device
// addresses of its positions and answers (registered caller memory) and its
// first work item; one extra entry closes a list.
struct ServeReq {
    const uint64_t *pos;
    float *out;
    uint8_t *valid;
    unsigned long long at;
};

// Simple fixed-size thread pool for file writes.
class WriterPool {
public:
    explicit WriterPool(int threads);
    ~WriterPool();
    // ready (optional): the job waits for this event (on `device`) before writing
    void submit(std::string path, const void *data, size_t bytes, cudaEvent_t ready = nullptr, int device = 0);
    void wait();  // rethrows the first failure

private:
    struct Impl;
    Impl *impl_;
};

}  // namespace egtb
