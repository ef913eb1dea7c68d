// Host helpers of libegtb_gpu (see egtb_host.h).
#include "egtb_host.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <cerrno>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <ctime>
#include <deque>
#include <mutex>
#include <thread>

namespace egtb {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }
void clear_last_error() { g_last_error.clear(); }

static std::atomic<unsigned> g_spin_limit{0};  // 0: kSpinLimit

unsigned look_back_spin_limit() {
    const unsigned v = g_spin_limit.load(std::memory_order_relaxed);
    return v ? v : kSpinLimit;
}

}  // namespace egtb

extern "C" int egtb_set_spin_limit(uint32_t polls) {
    egtb::g_spin_limit.store(polls, std::memory_order_relaxed);
    return EGTB_OK;
}

extern "C" int egtb_last_error(char *buf, size_t len) {
    if (!buf || len == 0) return EGTB_ERR_ARG;
    const std::string &m = egtb::g_last_error;
    size_t n = m.size() < len - 1 ? m.size() : len - 1;
    std::memcpy(buf, m.data(), n);
    buf[n] = 0;
    return EGTB_OK;
}

namespace egtb {

// One row moved toward column 0 (reverse = false) or column 3.
// Classic (walls = false): slide the tiles, merge each adjacent equal pair
// once, first pair first; 0xF (32768) slides but never merges
// (native_core/include/BoardMover.h:6-55).
// Variant (walls = true): 0xF cells are walls that stay put; the tiles of
// each stretch between walls slide and merge within it the same way
// (WallMergePolicy, native_core/include/VBoardMover.h:7-76).
static uint32_t row_after_move(uint32_t row, bool reverse, bool walls) {
    int cell[4];
    for (int i = 0; i < 4; ++i) cell[i] = (row >> (12 - 4 * i)) & 0xF;  // column 0 first
    if (reverse) {
        std::swap(cell[0], cell[3]);
        std::swap(cell[1], cell[2]);
    }
    int out[4] = {0, 0, 0, 0};
    int seg = 0;  // first cell of the current stretch
    while (seg < 4) {
        if (walls && cell[seg] == 0xF) {
            out[seg] = 0xF;
            ++seg;
            continue;
        }
        int end = seg;
        while (end < 4 && !(walls && cell[end] == 0xF)) ++end;
        int m = seg, pending = 0;
        for (int i = seg; i < end; ++i) {
            if (!cell[i]) continue;
            if (pending && pending == cell[i] && pending != 0xF) {
                out[m++] = pending + 1;
                pending = 0;
            } else {
                if (pending) out[m++] = pending;
                pending = cell[i];
            }
        }
        if (pending) out[m++] = pending;
        seg = end;
    }
    if (reverse) {
        std::swap(out[0], out[3]);
        std::swap(out[1], out[2]);
    }
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) r |= (uint32_t)(out[i] & 0xF) << (12 - 4 * i);
    return r;
}

const std::vector<uint32_t> &host_row_tables(bool variant) {
    auto make = [](bool walls) {
        std::vector<uint32_t> t(65536);
        for (uint32_t r = 0; r < 65536; ++r) {
            const uint32_t l = row_after_move(r, false, walls) ^ r;
            const uint32_t rr = row_after_move(r, true, walls) ^ r;
            t[r] = l | (rr << 16);
        }
        return t;
    };
    static const std::vector<uint32_t> classic = make(false), walled = make(true);
    return variant ? walled : classic;
}

const uint32_t *device_row_table(bool variant) {
    static std::mutex mu;
    static std::vector<uint32_t *> per_device[2];
    int dev = 0;
    EGTB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    std::vector<uint32_t *> &v = per_device[variant ? 1 : 0];
    if ((int)v.size() <= dev) v.resize(dev + 1, nullptr);
    if (!v[dev]) {
        uint32_t *p = nullptr;
        EGTB_CUDA(cudaMalloc(&p, 65536 * sizeof(uint32_t)));
        EGTB_CUDA(cudaMemcpy(p, host_row_tables(variant).data(), 65536 * sizeof(uint32_t), cudaMemcpyHostToDevice));
        v[dev] = p;
    }
    return v[dev];
}

DevSpec make_dev_spec(const egtb_pattern_spec &s, int target) {
    DevSpec d;
    std::memset(&d, 0, sizeof d);
    if (s.n_masks < 0 || s.n_masks > kMaxMasks) throw Error(EGTB_ERR_ARG, "n_masks out of range");
    if (s.n_shifts < 0 || s.n_shifts > 16) throw Error(EGTB_ERR_ARG, "n_shifts out of range");
    if (s.symm_mode < 0 || s.symm_mode > 6)
        throw Error(EGTB_ERR_ARG, "symmetry mode " + std::to_string(s.symm_mode) + " out of range");
    d.n_masks = s.n_masks;
    for (int i = 0; i < s.n_masks; ++i) d.masks[i] = s.pattern_masks[i];
    d.symm = s.symm_mode;
    d.has_success = s.n_shifts > 0;
    d.target = target;
    d.target_rep = (uint64_t)(target & 0xF) * 0x1111111111111111ull;
    d.succ_hi = 0;
    for (int i = 0; i < s.n_shifts; ++i) {
        const int sh = s.success_shifts[i];
        if (sh % 4 != 0 || sh > 60) throw Error(EGTB_ERR_UNSUPPORTED, "success shift not on a nibble boundary");
        d.succ_hi |= 8ull << sh;
    }
    if (target < 0 || target > 15) {
        // a nibble can never equal it: nothing is a success (unless no shifts)
        d.succ_hi = d.has_success ? 0 : d.succ_hi;
    }
    return d;
}

size_t dtype_size(int dtype) {
    switch (dtype) {
        case EGTB_DTYPE_UINT64: case EGTB_DTYPE_FLOAT64: case EGTB_DTYPE_1_FLOAT64: return 8;
        case EGTB_DTYPE_UINT32: case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_1_FLOAT32: return 4;
        default: throw Error(EGTB_ERR_ARG, "unknown success_rate_dtype " + std::to_string(dtype));
    }
}
bool dtype_is_one_minus(int dtype) { return dtype == EGTB_DTYPE_1_FLOAT32 || dtype == EGTB_DTYPE_1_FLOAT64; }
// zero_value_for_dtype / max_scale_value_for_dtype, native_core/include/FormationRuntime.h:257-312
double dtype_zero(int dtype) { return dtype_is_one_minus(dtype) ? -1.0 : 0.0; }
double dtype_max(int dtype) {
    switch (dtype) {
        case EGTB_DTYPE_UINT32: return 4000000000.0;
        case EGTB_DTYPE_UINT64: return 1600000000000000000.0;
        case EGTB_DTYPE_FLOAT32: case EGTB_DTYPE_FLOAT64: return 1.0;
        default: return 0.0;
    }
}
std::string dtype_name(int dtype) {
    static const char *names[] = {"uint32", "uint64", "float32", "float64", "1-float32", "1-float64"};
    return (dtype >= 0 && dtype < 6) ? names[dtype] : "uint32";
}

bool file_exists(const std::string &path) {
    struct stat st;
    return ::stat(path.c_str(), &st) == 0;
}

uint64_t file_size(const std::string &path) {
    struct stat st;
    if (::stat(path.c_str(), &st) != 0) return 0;
    return (uint64_t)st.st_size;
}

// is_valid_restart_file, native_core/src/BookGenerator.cpp:71-84
bool file_valid(const std::string &path, uint64_t alignment) {
    struct stat st;
    if (::stat(path.c_str(), &st) != 0 || !S_ISREG(st.st_mode) || st.st_size == 0) return false;
    return alignment == 0 || ((uint64_t)st.st_size % alignment) == 0;
}

// remove_invalid_restart_file, native_core/src/BookGenerator.cpp:86-99
void remove_invalid(const std::string &path, uint64_t alignment) {
    if (!file_exists(path) || file_valid(path, alignment)) return;
    if (::unlink(path.c_str()) != 0) throw Error(EGTB_ERR_IO, "failed to remove invalid restart file: " + path);
}

void remove_file(const std::string &path) { ::unlink(path.c_str()); }

void write_file(const std::string &path, const void *data, size_t bytes) {
    const std::string tmp = path + ".tmp";
    int fd = ::open(tmp.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) throw Error(EGTB_ERR_IO, "cannot open " + tmp + ": " + std::strerror(errno));
    const char *p = static_cast<const char *>(data);
    size_t left = bytes;
    while (left > 0) {
        ssize_t w = ::write(fd, p, left > (1u << 30) ? (1u << 30) : left);
        if (w < 0) {
            if (errno == EINTR) continue;
            ::close(fd);
            throw Error(EGTB_ERR_IO, "write failed " + tmp + ": " + std::strerror(errno));
        }
        p += w;
        left -= (size_t)w;
    }
    if (::close(fd) != 0) throw Error(EGTB_ERR_IO, "close failed " + tmp);
    if (::rename(tmp.c_str(), path.c_str()) != 0) throw Error(EGTB_ERR_IO, "rename failed " + path);
}

void read_file_into(const std::string &path, void *dst, size_t bytes) {
    int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) throw Error(EGTB_ERR_IO, "cannot open " + path + ": " + std::strerror(errno));
    char *p = static_cast<char *>(dst);
    size_t left = bytes;
    while (left > 0) {
        ssize_t r = ::read(fd, p, left > (1u << 30) ? (1u << 30) : left);
        if (r < 0) {
            if (errno == EINTR) continue;
            ::close(fd);
            throw Error(EGTB_ERR_IO, "read failed " + path);
        }
        if (r == 0) break;
        p += r;
        left -= (size_t)r;
    }
    ::close(fd);
    if (left) throw Error(EGTB_ERR_IO, "short read " + path);
}

std::vector<unsigned char> read_file(const std::string &path) {
    std::vector<unsigned char> v(file_size(path));
    if (!v.empty()) read_file_into(path, v.data(), v.size());
    return v;
}

std::string parent_dir(const std::string &path) {
    const size_t p = path.find_last_of('/');
    return p == std::string::npos ? std::string(".") : path.substr(0, p);
}

std::string now_string() {
    std::time_t now = std::time(nullptr);
    std::tm lt{};
    localtime_r(&now, &lt);
    char buf[32];
    std::strftime(buf, sizeof buf, "%Y-%m-%d %H:%M:%S", &lt);
    return buf;
}

double round_to_2(double v) { return std::round(v * 100.0) / 100.0; }

// ------------------------------------------------------------ writer pool ---

struct WriterPool::Impl {
    struct Job {
        std::string path;
        const void *data;
        size_t bytes;
        cudaEvent_t ready;  // when set: the data is complete once this event has completed
        int device;
    };
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<Job> q;
    std::vector<std::thread> threads;
    int active = 0;
    bool stop = false;
    std::string error;
    int error_code = 0;
};

WriterPool::WriterPool(int threads) : impl_(new Impl) {
    if (threads < 1) threads = 1;
    for (int i = 0; i < threads; ++i) {
        impl_->threads.emplace_back([this] {
            Impl &s = *impl_;
            for (;;) {
                Impl::Job job;
                {
                    std::unique_lock<std::mutex> lk(s.mu);
                    s.cv.wait(lk, [&] { return s.stop || !s.q.empty(); });
                    if (s.q.empty()) return;
                    job = std::move(s.q.front());
                    s.q.pop_front();
                    ++s.active;
                }
                try {
                    if (job.ready) {
                        EGTB_CUDA(cudaSetDevice(job.device));
                        EGTB_CUDA(cudaEventSynchronize(job.ready));
                    }
                    write_file(job.path, job.data, job.bytes);
                } catch (const Error &e) {
                    std::lock_guard<std::mutex> lk(s.mu);
                    if (s.error.empty()) {
                        s.error = e.what();
                        s.error_code = e.code;
                    }
                }
                {
                    std::lock_guard<std::mutex> lk(s.mu);
                    --s.active;
                }
                s.done_cv.notify_all();
            }
        });
    }
}

WriterPool::~WriterPool() {
    {
        std::lock_guard<std::mutex> lk(impl_->mu);
        impl_->stop = true;
    }
    impl_->cv.notify_all();
    for (auto &t : impl_->threads) t.join();
    delete impl_;
}

void WriterPool::submit(std::string path, const void *data, size_t bytes, cudaEvent_t ready, int device) {
    {
        std::lock_guard<std::mutex> lk(impl_->mu);
        impl_->q.push_back({std::move(path), data, bytes, ready, device});
    }
    impl_->cv.notify_one();
}

void WriterPool::wait() {
    std::unique_lock<std::mutex> lk(impl_->mu);
    impl_->done_cv.wait(lk, [&] { return impl_->q.empty() && impl_->active == 0; });
    if (!impl_->error.empty()) {
        std::string e = impl_->error;
        int c = impl_->error_code;
        impl_->error.clear();
        throw Error(c, e);
    }
}

}  // namespace egtb
